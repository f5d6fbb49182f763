"""The batched uneven fit (many volumes, one CUDA graph): the job generator and branch plan on
the CPU, and on the GPU every job's result from the per-family work queues (captured in a graph)
and from the per-job kernel chains against the same job fitted alone and, for mFOD, against the
public fit_multi_tissue, bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

from larmor_b200.batch import assign_branches, generate_jobs


def test_generated_jobs_follow_the_spec():
    jobs = generate_jobs(seed=9, n_volumes=12, min_voxels=100, max_voxels=400)
    again = generate_jobs(seed=9, n_volumes=12, min_voxels=100, max_voxels=400)
    for a, b in zip(jobs, again):
        assert a.kind == b.kind and np.array_equal(a.signals, b.signals)
    for j in jobs:
        assert 100 <= j.voxels <= 400
        b = np.round(j.gtab.bvals, -1)  # the table rescales b by |g|^2, within rounding
        shells = sorted(set(b[b > 0]))
        assert 1 <= len(shells) <= 3
        for s in shells:
            assert 30 <= int((b == s).sum()) <= 90
        if j.kind in ("dki", "mfod"):
            assert len(shells) >= 2
        assert j.signals.shape == (j.voxels, len(b))


def test_branches_balance_longest_first():
    plan = assign_branches([5.0, 1.0, 4.0, 3.0, 3.0], 2)
    assert sorted(i for b in plan for i in b) == [0, 1, 2, 3, 4]
    loads = [sum([5.0, 1.0, 4.0, 3.0, 3.0][i] for i in b) for b in plan]
    assert max(loads) - min(loads) <= 2.0
    assert plan[0][0] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("queue", [True, False], ids=["family_queues", "job_chains"])
def test_graph_batch_equals_eager_fits(cuda, queue):
    import torch

    from larmor_b200 import _core
    from larmor_b200.batch import Batch
    from larmor_b200.sd.solvers import FINAL_FRACTION_TOL_X, MAX_ROUNDS

    jobs = generate_jobs(seed=5, n_volumes=9, min_voxels=300, max_voxels=3000, mix=(1, 1, 1))
    assert {j.kind for j in jobs} == {"dti", "dki", "mfod"}
    # An odd number of DKI voxels in all, as in the 64-volume workload: the scratch that follows
    # the queue's violator list must stay 8-byte aligned.
    if sum(j.voxels for j in jobs if j.kind == "dki") % 2 == 0:
        dki = next(j for j in jobs if j.kind == "dki")
        dki.signals, dki.s0, dki.floor = dki.signals[:-1], dki.s0[:-1], dki.floor[:-1]
    assert sum(j.voxels for j in jobs if j.kind == "dki") % 2 == 1
    graph = Batch(jobs, branches=3, queue=queue)
    graph.capture()
    for o in (j.out for j in jobs):
        for t in o.values():
            t.zero_()
    graph.run()
    torch.cuda.synchronize()
    got = [{k: t.cpu().numpy().copy() for k, t in j.out.items()} for j in jobs]
    eager = Batch(jobs, branches=1, queue=False)
    eager.run_eager()
    torch.cuda.synchronize()
    for j, g in zip(jobs, got):
        for k, t in j.out.items():
            np.testing.assert_array_equal(g[k], t.cpu().numpy(), err_msg=f"{j.kind} {k}")
        if j.kind == "mfod":
            h = j.handles
            fods, fr = _core.fit_multi_tissue(np.ascontiguousarray(j.signals), h["weights"], h["k_lr"],
                                              h["lr_solver"], h["k_hr"], h["hr_solver"], MAX_ROUNDS, 1e-7,
                                              FINAL_FRACTION_TOL_X, 1)
            np.testing.assert_array_equal(g["fods"], fods)
            np.testing.assert_array_equal(g["fractions"], fr)
