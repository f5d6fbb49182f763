"""Batched fits of many volumes in one CUDA graph.

A batch holds jobs of different models (DTI, DKI, mFOD), gradient tables and voxel counts. Each
job gets its own device inputs, outputs and design handles. By default (`queue=True`) the jobs
of each model family are fitted through one device work queue (lar_batch_*): every stage of the
family is one launch over all of the family's volumes, whose CTAs or warps take (volume,
voxel-block) tickets from one counter, so uneven volumes and uneven per-voxel NNLS costs are
absorbed across the whole batch; the three families run on parallel branches. With
`queue=False` each job runs its own chain of kernels, the jobs spread over parallel branches
(longest first onto the least-loaded branch).

`Batch.capture()` runs the batch once eagerly (which sizes the per-job scratch of the chained
mode and uploads shell weights), then records it into one CUDA graph; `Batch.run()` replays
it: one launch for the whole batch. With `tune=True` the launch shapes of each model's kernels
are first chosen by measurement (larmor_b200.autotune). The results stay on the device in each
job's output tensors.

The per-voxel work is the same device code as the single fits (larmor_b200._core), so a job's
result in the batch equals its result alone, bit for bit.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from larmor_b200 import _core, _lib
from larmor_b200.types import GradientTable


@dataclass
class DtiJob:
    """A DTI WLS fit of float32 signals (v, n) with per-voxel floors (v,): 16 maps (16, v)."""

    gtab: GradientTable
    signals: np.ndarray
    floor: np.ndarray
    kind: str = "dti"
    out: dict = field(default_factory=dict)

    @property
    def voxels(self) -> int:
        return len(self.signals)

    def cost(self) -> float:
        return self.voxels * self.signals.shape[1] * 1.0


@dataclass
class DkiJob:
    """A constrained DKI WLS fit of float32 signals (v, n) with S0 and floors (v,): 36 maps."""

    gtab: GradientTable
    signals: np.ndarray
    s0: np.ndarray
    floor: np.ndarray
    kind: str = "dki"
    out: dict = field(default_factory=dict)

    @property
    def voxels(self) -> int:
        return len(self.signals)

    def cost(self) -> float:
        return self.voxels * self.signals.shape[1] * 60.0


@dataclass
class MfodJob:
    """A three-tissue mFOD fit of S0-normalised signals (v, n): amplitudes on the 300-direction
    grid and the fractions (WM, GM, CSF)."""

    gtab: GradientTable
    signals: np.ndarray
    responses: list
    kind: str = "mfod"
    out: dict = field(default_factory=dict)

    @property
    def voxels(self) -> int:
        return len(self.signals)

    def cost(self) -> float:
        return self.voxels * self.signals.shape[1] * 150.0


def assign_branches(costs, n: int) -> list[list[int]]:
    """Job indices per graph branch: longest job first onto the least-loaded branch (ties to
    the lowest branch index)."""
    loads = [0.0] * n
    out: list[list[int]] = [[] for _ in range(n)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        b = min(range(n), key=lambda k: (loads[k], k))
        out[b].append(i)
        loads[b] += costs[i]
    return out


def job_key(job) -> bytes:
    """What a job's design handles depend on: its model and gradient table (and, for mFOD, its
    responses); jobs with equal keys can share handles when they never run at the same time."""
    import hashlib

    h = hashlib.blake2b(digest_size=20)
    h.update(job.kind.encode())
    h.update(np.ascontiguousarray(job.gtab.bvals).tobytes())
    h.update(np.ascontiguousarray(job.gtab.bvecs).tobytes())
    if job.kind == "mfod":
        h.update(repr(job.responses).encode())
    return h.digest()


def job_handles(job) -> dict:
    """The device design handles of a job: the log-fit design (DTI, DKI), or the two
    deconvolution kernels, their L2NNLS solvers and the shell weights (mFOD)."""
    if job.kind == "dti":
        from larmor_b200.dwi.dti import dti_design

        return {"design": _core.LogDesign(dti_design(job.gtab), np.zeros((0, 7)))}
    if job.kind == "dki":
        from larmor_b200.dwi.dki import dki_constraints, dki_design

        return {"design": _core.LogDesign(dki_design(job.gtab), dki_constraints(job.gtab))}
    if job.kind == "mfod":
        from larmor_b200.sd.kernel import Kernel
        from larmor_b200.sd.model import compute_shell_weights, low_resolution_dirs
        from larmor_b200.sd.solvers import L2NNLS, Stage, _deconv_kernel
        from larmor_b200.sd.sphere import DIRS_300

        b, g = job.gtab.bvals, job.gtab.bvecs
        weights = compute_shell_weights(b, 1.0)
        hr = Kernel(job.responses, b, g, dirs=DIRS_300, weights=weights)
        lr = Kernel(job.responses, b, g, dirs=low_resolution_dirs(job.responses, len(b)), weights=weights)
        return {"weights": np.ascontiguousarray(lr.weights, dtype=np.float64),
                "k_lr": _deconv_kernel(lr), "k_hr": _deconv_kernel(hr),
                "lr_solver": L2NNLS()._prepare(lr, b, Stage.LOW_RES),
                "hr_solver": L2NNLS()._prepare(hr, b, Stage.HIGH_RES)}
    raise ValueError(f"unknown job kind {job.kind!r}")


def job_outputs(job, handles: dict, dev) -> dict:
    """Device tensors for a job's results."""
    import torch

    v = job.voxels
    if job.kind == "dti":
        return {"maps": torch.empty((16, v), dtype=torch.float32, device=dev),
                "npd": torch.empty((v,), dtype=torch.uint8, device=dev)}
    if job.kind == "dki":
        return {"maps": torch.empty((36, v), dtype=torch.float32, device=dev),
                "npd": torch.empty((v,), dtype=torch.uint8, device=dev),
                "broke": torch.empty((v,), dtype=torch.uint8, device=dev),
                "params": torch.empty((v, 22), dtype=torch.float64, device=dev)}
    k_hr = handles["k_hr"]
    return {"fods": torch.empty((v, k_hr.ca), dtype=torch.float64, device=dev),
            "fractions": torch.empty((v, k_hr.nb + k_hr.ci), dtype=torch.float64, device=dev),
            "rounds": torch.empty((v,), dtype=torch.int32, device=dev),
            "status": torch.empty((v,), dtype=torch.uint8, device=dev)}


def job_inputs_host(job) -> tuple:
    """The host arrays a job's fit reads, in the order launch_job takes them on the device."""
    if job.kind == "dti":
        return (np.ascontiguousarray(job.signals, dtype=np.float32), np.ascontiguousarray(job.floor, dtype=np.float64))
    if job.kind == "dki":
        return (np.ascontiguousarray(job.signals, dtype=np.float32), np.ascontiguousarray(job.s0, dtype=np.float64),
                np.ascontiguousarray(job.floor, dtype=np.float64),
                np.ascontiguousarray(job.gtab.b0_mask, dtype=np.uint8))
    return (np.ascontiguousarray(job.signals, dtype=np.float64),)


def launch_job(job, handles: dict, d_in: tuple, out: dict, asynchronous: bool = False) -> None:
    """Enqueues one job's fit on the current stream (the mFOD fit waits on the host for each
    round's voxel count unless the stream is being captured or `asynchronous` is set)."""
    import torch

    if job.kind == "dti":
        s, floor = d_in
        _core.fit_dti_maps_device(handles["design"], s, floor, True, out["maps"], out["npd"])
    elif job.kind == "dki":
        s, s0, floor, b0 = d_in
        _lib.check(_lib.lib().lar_fit_dki_maps(
            handles["design"].handle, _lib.ptr(s), _lib.ptr(s0), _lib.ptr(floor), _lib.ptr(b0), job.voxels, 1, 20,
            1e-6, _lib.LAR_FP64, _lib.ptr(out["maps"]), _lib.ptr(out["npd"]), _lib.ptr(out["broke"]),
            _lib.ptr(out["params"]), _core._stream(torch)))
    else:
        from larmor_b200.sd.solvers import FINAL_FRACTION_TOL_X, MAX_ROUNDS

        h = handles
        _core.fit_multi_tissue_device(d_in[0], h["weights"], h["k_lr"], h["lr_solver"], h["k_hr"], h["hr_solver"],
                                      MAX_ROUNDS, 1e-7, FINAL_FRACTION_TOL_X, out["fods"], out["fractions"],
                                      out["rounds"], out["status"], asynchronous=asynchronous)


def job_device_bytes(job) -> int:
    """Device memory a job's fit needs beyond its handles: inputs, outputs and the per-voxel
    state of its call."""
    v = job.voxels
    n = job.signals.shape[1]
    if job.kind == "dti":
        return v * (4 * n + 8 + 16 * 4 + 1)
    if job.kind == "dki":
        return v * (4 * n + 16 + 36 * 4 + 2 + 22 * 8) + v * (8 + 22 * 8) + n
    # signals, 300 amplitudes, 3 fractions, rounds and status; correlations, the 44-direction
    # FOD, f_iso, previous fractions, two list entries.
    return v * (8 * n + 8 * 303 + 5) + v * (8 * (300 + 44 + 2 + 3) + 12)


class FamilyQueues:
    """The jobs of a batch fitted through one device work queue per model family: a lar_batch
    holding every job's inputs, outputs and handles (which must outlive it). run(family)
    enqueues the family's stages on the current stream."""

    FAMILIES = {"dti": _lib.LAR_BATCH_DTI, "dki": _lib.LAR_BATCH_DKI, "mfod": _lib.LAR_BATCH_MFOD}

    def __init__(self, jobs) -> None:
        import ctypes

        from larmor_b200.sd.solvers import FINAL_FRACTION_TOL_X, MAX_ROUNDS

        lib = _lib.lib()
        handle = ctypes.c_void_p()
        _lib.check(lib.lar_batch_create(ctypes.byref(handle)))
        self.handle = handle
        self.kinds = []
        try:
            for job in jobs:
                h, d_in, out = job.handles, job.d_in, job.out
                if job.kind == "dti":
                    s, floor = d_in
                    _lib.check(lib.lar_batch_add_dti(
                        handle, h["design"].handle, _lib.ptr(s), _lib.ptr(floor), job.voxels, 1, 20, 1e-6,
                        _lib.ptr(out["maps"]), _lib.ptr(out["npd"])))
                elif job.kind == "dki":
                    s, s0, floor, b0 = d_in
                    _lib.check(lib.lar_batch_add_dki(
                        handle, h["design"].handle, _lib.ptr(s), _lib.ptr(s0), _lib.ptr(floor), _lib.ptr(b0),
                        job.voxels, 1, 20, 1e-6, _lib.ptr(out["maps"]), _lib.ptr(out["npd"]),
                        _lib.ptr(out["broke"]), _lib.ptr(out["params"])))
                else:
                    _lib.check(lib.lar_batch_add_mfod(
                        handle, _lib.ptr(d_in[0]), job.voxels, _lib.ptr(h["weights"]), h["k_lr"].handle,
                        h["lr_solver"].handle, h["k_hr"].handle, h["hr_solver"].handle, MAX_ROUNDS, 1e-7,
                        FINAL_FRACTION_TOL_X, _lib.ptr(out["fods"]), _lib.ptr(out["fractions"]),
                        _lib.ptr(out["rounds"]), _lib.ptr(out["status"])))
                if job.kind not in self.kinds:
                    self.kinds.append(job.kind)
            _lib.check(lib.lar_batch_finalize(handle))
        except Exception:
            lib.lar_batch_destroy(handle)
            raise

    def run(self, kind: str) -> None:
        """Enqueues the stages of one family ("dti", "dki" or "mfod") on the current stream."""
        import torch

        _lib.check(_lib.lib().lar_batch_run(self.handle, self.FAMILIES[kind], _core._stream(torch)))

    def __del__(self) -> None:
        handle = getattr(self, "handle", None)
        if handle is not None and handle.value:
            _lib.lib().lar_batch_destroy(handle)
            self.handle = None


class Batch:
    """Jobs fitted together, replayed as one CUDA graph (see the module docstring)."""

    def __init__(self, jobs, branches: int = 4, tune: bool = False, tuner=None, queue: bool = True) -> None:
        """tune: first pick each model's launch settings on a sample of its largest volume
        (larmor_b200.autotune; the choice is cached per GPU and workload signature). queue: one
        work queue per model family (else a chain of kernels per job on `branches` branches)."""
        import torch

        self.torch = torch
        self.jobs = list(jobs)
        self.launch_settings = {}
        if tune:
            from larmor_b200.autotune import tune_jobs

            self.launch_settings = tune_jobs(self.jobs, tuner)
        self.dev = torch.device("cuda", torch.cuda.current_device())
        self.graph = None
        for job in self.jobs:
            job.handles = job_handles(job)
            job.d_in = tuple(torch.from_numpy(a).to(self.dev) for a in job_inputs_host(job))
            job.out = job_outputs(job, job.handles, self.dev)
        self.queues = FamilyQueues(self.jobs) if queue else None
        n_streams = len(self.queues.kinds) if queue else branches
        self.streams = [torch.cuda.Stream(self.dev) for _ in range(max(1, n_streams))]
        self.assignment = assign_branches([j.cost() for j in self.jobs], len(self.streams))

    def _enqueue(self) -> None:
        torch = self.torch
        root = torch.cuda.current_stream(self.dev)
        if self.queues is not None:
            for stream, kind in zip(self.streams, self.queues.kinds):
                stream.wait_stream(root)
                with torch.cuda.stream(stream):
                    self.queues.run(kind)
                root.wait_stream(stream)
            return
        for stream, idx in zip(self.streams, self.assignment):
            stream.wait_stream(root)
            with torch.cuda.stream(stream):
                for i in idx:
                    job = self.jobs[i]
                    launch_job(job, job.handles, job.d_in, job.out)
            root.wait_stream(stream)

    def run_eager(self) -> None:
        """Every job on its branch's stream, without a graph (also the warm-up of capture())."""
        self._enqueue()

    def capture(self) -> None:
        """Runs the batch once eagerly, then records it into one CUDA graph."""
        torch = self.torch
        self.run_eager()
        torch.cuda.synchronize(self.dev)
        graph = torch.cuda.CUDAGraph()
        before = _core.launch_count()
        with torch.cuda.graph(graph, stream=torch.cuda.Stream(self.dev)):
            self._enqueue()
        self.graph = graph
        # The library's kernels recorded in the graph (each replay launches them all).
        self.graph_kernels = _core.launch_count() - before

    def run(self) -> None:
        """Replays the captured graph on the current stream (capture() first)."""
        if self.graph is None:
            raise RuntimeError("capture() the batch before run()")
        self.graph.replay()

    @property
    def voxels(self) -> int:
        return sum(j.voxels for j in self.jobs)


# ---- the batched-uneven workload (seeded) ----------------------------------------------------

def _table(rng: np.random.Generator, shells: int) -> GradientTable:
    """1-3 shells (b = 1000, 2000, 3000) of U[30, 90] directions each, with one b0 per 15."""
    from larmor_b200.synthetic import unit_directions

    counts = [int(rng.integers(30, 91)) for _ in range(shells)]
    n_b0 = max(1, sum(counts) // 15)
    bvals = np.concatenate([np.zeros(n_b0)] + [np.full(c, 1000.0 * (k + 1)) for k, c in enumerate(counts)])
    bvecs = np.vstack([np.zeros((n_b0, 3))] + [unit_directions(rng, c) for c in counts])
    return GradientTable(bvals, bvecs)


def generate_jobs(seed: int = 4, n_volumes: int = 64, min_voxels: int = 10_000, max_voxels: int = 400_000,
                  mix=(0.4, 0.2, 0.4)) -> list:
    """Seeded uneven jobs: voxel counts log-uniform in [min_voxels, max_voxels], 1-3 shells of
    30-90 directions, models DTI/DKI/mFOD drawn with probabilities `mix`; a DKI or mFOD draw
    with one shell (which those models cannot fit) draws its table again. Signals follow the
    single-volume generators (tensor for DTI, stick-zeppelin for DKI, 1-3 fibres with GM/CSF
    for mFOD) with Rician noise."""
    from larmor_b200.synthetic import (_stick_zeppelin, mfod_model_responses, mfod_signals, random_rotations,
                                       rician, unit_directions)

    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(n_volumes):
        kind = ["dti", "dki", "mfod"][int(rng.choice(3, p=np.asarray(mix) / np.sum(mix)))]
        v = int(round(math.exp(rng.uniform(math.log(min_voxels), math.log(max_voxels)))))
        shells = int(rng.integers(1, 4))
        while kind != "dti" and shells < 2:
            shells = int(rng.integers(1, 4))
        gtab = _table(rng, shells)
        b, g = gtab.bvals, gtab.bvecs
        s0 = 1000.0
        if kind == "dti":
            l1, l23 = rng.uniform(1.2e-3, 2.0e-3, v), rng.uniform(0.2e-3, 0.6e-3, v)
            rot = random_rotations(rng, v)
            tensors = np.einsum("vij,vj,vkj->vik", rot, np.stack([l1, l23, l23], axis=1), rot)
            adc = np.einsum("ni,vij,nj->vn", g, tensors, g)
            sig = rician(rng, s0 * np.exp(-b[None, :] * adc), s0 / 20.0).astype(np.float32)
            jobs.append(DtiJob(gtab, sig, np.full(v, 1e-3 * s0)))
        elif kind == "dki":
            axis = unit_directions(rng, v)
            sig = s0 * _stick_zeppelin(b, g, axis, rng.uniform(0.3, 0.7, v), 2.0e-3, rng.uniform(0.4e-3, 0.8e-3, v))
            sig = rician(rng, sig, s0 / 30.0).astype(np.float32)
            est = np.maximum(sig[:, b == 0].mean(axis=1).astype(np.float64), 1e-3 * s0)
            jobs.append(DkiJob(gtab, sig, est, 1e-3 * est))
        else:
            sig = mfod_signals(rng, gtab, v)
            est = np.maximum(sig[:, b == 0].mean(axis=1), 1e-3 * s0)
            jobs.append(MfodJob(gtab, np.minimum(sig / est[:, None], 1.0), mfod_model_responses()))
    return jobs
