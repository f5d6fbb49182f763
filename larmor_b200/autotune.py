"""Autotuning of the kernels' launch shapes.

The library's kernels read a few launch settings (lar_set_launch_setting): how many voxels a
CTA of the shared-memory DTI fit takes, how many waves of CTAs the warp-per-voxel log fit
launches, and how many CTAs per SM the persistent grids of the constrained DKI re-fit, the LSI,
the ridge NNLS and the fraction fits keep resident (fewer than occupancy allows can win when
their per-warp scratch then stays in L2). Results never depend on them, only the time does.

A `LaunchTuner` times the candidates of each setting on a sample fit, one setting after the
other (coordinate descent, each at its best value once chosen), with CUDA events on the current
stream, keeps the fastest and remembers it in a JSON cache keyed by the GPU's name and a
signature of the workload (model, measurements, directions), so that a later process applies
the choice without measuring again. `tune_jobs` tunes the models of a batch on a sample of its
largest volume of each model.
"""

from __future__ import annotations

import json
import os
import statistics
from pathlib import Path

from larmor_b200 import _lib

# The settings each model's kernels read, with the values worth trying.
CANDIDATES = {
    "dti": {"dti.voxels_per_cta": [16, 32, 64]},
    "dki": {"log.warp.waves": [1, 2, 4, 8], "dki.refit.ctas_per_sm": [2, 3, 4]},
    "mfod": {"sd.nnls.ctas_per_sm": [2, 4, 6, 8], "sd.fractions.ctas_per_sm": [2, 3, 4]},
    "msmt": {"lsi.ctas_per_sm": [2, 3, 4, 5]},
}


def set_setting(name: str, value: int) -> None:
    """Sets one launch setting (0 restores the library's choice)."""
    _lib.check(_lib.lib().lar_set_launch_setting(name.encode(), int(value)))


def get_setting(name: str) -> int:
    import ctypes

    v = ctypes.c_int64(0)
    _lib.check(_lib.lib().lar_get_launch_setting(name.encode(), ctypes.byref(v)))
    return v.value


def default_cache_path() -> Path:
    env = os.environ.get("LARMOR_B200_TUNE_CACHE")
    return Path(env) if env else Path.home() / ".cache" / "larmor_b200" / "launch_settings.json"


def gpu_name() -> str:
    import torch

    return torch.cuda.get_device_name(torch.cuda.current_device())


def event_timer(run, repeats: int = 3) -> float:
    """Median device time (ms) of `repeats` calls of run() after one warm-up call."""
    import torch

    run()
    times = []
    stream = torch.cuda.current_stream()
    for _ in range(repeats):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        run()
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    return statistics.median(times)


class LaunchTuner:
    """See the module docstring. `timer(run)` returns a run's time (ms); `device` names the GPU
    in the cache keys (both replaceable, e.g. in tests)."""

    def __init__(self, cache_path=None, timer=event_timer, device: str | None = None) -> None:
        self.cache_path = Path(cache_path) if cache_path is not None else default_cache_path()
        self.timer = timer
        self.device = device
        self.cache = self._load()
        self.measured: dict = {}

    def _load(self) -> dict:
        try:
            return json.loads(self.cache_path.read_text())
        except (OSError, ValueError):
            return {}

    def _save(self) -> None:
        try:
            self.cache_path.parent.mkdir(parents=True, exist_ok=True)
            self.cache_path.write_text(json.dumps(self.cache, indent=1, sort_keys=True))
        except OSError:
            pass  # a read-only home: the choice still holds for this process

    def key(self, signature: str) -> str:
        return f"{self.device or gpu_name()}|{signature}"

    def tune(self, signature: str, candidates: dict, run) -> dict:
        """The best value of each setting for run() (from the cache when it is there), applied."""
        key = self.key(signature)
        if key in self.cache:
            chosen = self.cache[key]
            for name, value in chosen.items():
                set_setting(name, value)
            return dict(chosen)
        chosen, times = {}, {}
        for name, values in candidates.items():
            best, best_ms = 0, None
            times[name] = {}
            for value in [0] + [v for v in values if v != 0]:
                set_setting(name, value)
                ms = self.timer(run)
                times[name][value] = ms
                if best_ms is None or ms < best_ms:
                    best, best_ms = value, ms
            set_setting(name, best)
            chosen[name] = best
        self.cache[key] = chosen
        self.measured[key] = times
        self._save()
        return dict(chosen)


def job_signature(job) -> str:
    """What a model's best launch shape depends on: the model, the measurements and, for the
    spherical deconvolution, the directions."""
    return f"{job.kind}:n={job.signals.shape[1]}"


def tune_jobs(jobs, tuner: LaunchTuner | None = None, sample_voxels: int = 65536) -> dict:
    """Tunes the launch settings of every model in `jobs` on up to `sample_voxels` voxels of its
    largest volume; returns {model: chosen settings}."""
    import dataclasses

    import torch

    from larmor_b200.batch import job_handles, job_inputs_host, job_outputs, launch_job

    tuner = tuner or LaunchTuner()
    dev = torch.device("cuda", torch.cuda.current_device())
    chosen = {}
    for kind in sorted({j.kind for j in jobs}):
        largest = max((j for j in jobs if j.kind == kind), key=lambda j: j.voxels)
        n = min(largest.voxels, sample_voxels)
        fields = {"signals": largest.signals[:n]}
        for name in ("floor", "s0"):
            if hasattr(largest, name):
                fields[name] = getattr(largest, name)[:n]
        sample = dataclasses.replace(largest, **fields, out={})
        handles = job_handles(sample)
        d_in = tuple(torch.from_numpy(a).to(dev) for a in job_inputs_host(sample))
        out = job_outputs(sample, handles, dev)
        chosen[kind] = tuner.tune(job_signature(sample), CANDIDATES[kind],
                                  lambda: launch_job(sample, handles, d_in, out))
    return chosen
