"""The launch-shape tuner: candidate search and cache on the CPU with a stand-in timer, the
settings' validation through the C ABI, and on the GPU that results do not depend on them."""

from __future__ import annotations

import numpy as np
import pytest

from larmor_b200 import autotune


def test_settings_round_trip_and_validation():
    autotune.set_setting("sd.nnls.ctas_per_sm", 3)
    assert autotune.get_setting("sd.nnls.ctas_per_sm") == 3
    autotune.set_setting("sd.nnls.ctas_per_sm", 0)
    assert autotune.get_setting("sd.nnls.ctas_per_sm") == 0
    with pytest.raises(ValueError):
        autotune.set_setting("no.such.setting", 1)
    with pytest.raises(ValueError):
        autotune.set_setting("dti.voxels_per_cta", 1000)
    with pytest.raises(ValueError):
        autotune.set_setting("lsi.ctas_per_sm", -1)


def test_tuner_picks_the_fastest_value_per_setting_and_caches_it(tmp_path):
    cost = {("lsi.ctas_per_sm", 0): 5.0, ("lsi.ctas_per_sm", 2): 3.0, ("lsi.ctas_per_sm", 3): 4.0}

    def timer(run):
        run()
        return cost[("lsi.ctas_per_sm", autotune.get_setting("lsi.ctas_per_sm"))]

    calls = []
    tuner = autotune.LaunchTuner(tmp_path / "cache.json", timer=timer, device="test-gpu")
    chosen = tuner.tune("msmt:n=280", {"lsi.ctas_per_sm": [2, 3]}, lambda: calls.append(1))
    assert chosen == {"lsi.ctas_per_sm": 2}
    assert autotune.get_setting("lsi.ctas_per_sm") == 2
    assert len(calls) == 3
    # A new tuner reads the cache and measures nothing.
    autotune.set_setting("lsi.ctas_per_sm", 0)
    again = autotune.LaunchTuner(tmp_path / "cache.json", timer=lambda run: pytest.fail("measured"),
                                 device="test-gpu")
    assert again.tune("msmt:n=280", {"lsi.ctas_per_sm": [2, 3]}, lambda: None) == {"lsi.ctas_per_sm": 2}
    assert autotune.get_setting("lsi.ctas_per_sm") == 2
    autotune.set_setting("lsi.ctas_per_sm", 0)


@pytest.mark.gpu
def test_results_do_not_depend_on_the_launch_settings(cuda):
    import torch

    from larmor_b200.batch import generate_jobs, job_handles, job_inputs_host, job_outputs, launch_job

    jobs = generate_jobs(seed=8, n_volumes=6, min_voxels=2000, max_voxels=6000, mix=(1, 1, 1))
    dev = torch.device("cuda")
    shapes = [{}, {"dti.voxels_per_cta": 16, "log.warp.waves": 1, "dki.refit.ctas_per_sm": 2,
                   "sd.nnls.ctas_per_sm": 2, "sd.fractions.ctas_per_sm": 2},
              {"dti.voxels_per_cta": 32, "log.warp.waves": 8, "dki.refit.ctas_per_sm": 3,
               "sd.nnls.ctas_per_sm": 5, "sd.fractions.ctas_per_sm": 3}]
    results = []
    try:
        for shape in shapes:
            for name in ("dti.voxels_per_cta", "log.warp.waves", "dki.refit.ctas_per_sm", "sd.nnls.ctas_per_sm",
                         "sd.fractions.ctas_per_sm"):
                autotune.set_setting(name, shape.get(name, 0))
            run = []
            for j in jobs:
                h = job_handles(j)
                d_in = tuple(torch.from_numpy(a).to(dev) for a in job_inputs_host(j))
                out = job_outputs(j, h, dev)
                launch_job(j, h, d_in, out)
                torch.cuda.synchronize()
                run.append({k: t.cpu().numpy() for k, t in out.items()})
            results.append(run)
    finally:
        for name in ("dti.voxels_per_cta", "log.warp.waves", "dki.refit.ctas_per_sm", "sd.nnls.ctas_per_sm",
                     "sd.fractions.ctas_per_sm"):
            autotune.set_setting(name, 0)
    for other in results[1:]:
        for j, a, b in zip(jobs, results[0], other):
            for k in a:
                np.testing.assert_array_equal(a[k], b[k], err_msg=f"{j.kind} {k}")
