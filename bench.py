"""Benchmark of the voxelwise fitting hot path on B200: voxel fits per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload dti|...] [--impl reference]

A step is one pass of the fit over one synthetic volume of the chosen configuration (seeded
generators in larmor_b200/synthetic.py; no public dataset is named for these shapes). The
timed region of `value` holds K steps with the inputs resident in device memory, timed with
CUDA events on the launching stream; L2 is flushed (a 256 MiB write) before every step, outside
the events. `e2e` times the same steps through the public C-ABI path with host buffers: the
pinned float32 signals and floors are copied to the device, fitted, and the maps copied back.

With N > 1 (torchrun, one process per GPU) every rank fits its own volume (weak scaling, no
data-path collective); the time is the maximum over ranks.

`--impl reference` times the reference's algorithm on the host's cores instead: the FP64 C++
restatement in oracle/ (the reference's own C++ core needs Eigen and nanobind, absent here), with
every host thread, on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "voxel fits/sec (DTI, mFOD) at stated FP64 error vs plain GPU; serve p50/p99 ms"
FALLBACK_HBM_GBS = 6650.0


def peaks() -> tuple[dict, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        return json.loads(path.read_text()), "measured"
    return {"hbm_gbs": FALLBACK_HBM_GBS, "bf16_tflops": 1590.0}, "fallback"


# Nominal dense FP64 tensor-core rate of one B200 (NVIDIA's HGX B200 figure, TFLOP/s): the
# denominator for the FP64 tensor-core kernels, which the measured peaks (an HBM copy and a bf16
# GEMM) do not cover.
NOMINAL_FP64_TENSOR_TFLOPS = 37.0


def fp64_tensor_roofline(flops_per_launch: float, avg_launch_s: float) -> dict:
    """The roofline fields of a kernel bound by the FP64 tensor cores."""
    achieved = flops_per_launch / avg_launch_s / 1e12 if avg_launch_s > 0 else 0.0
    return {"bound": "tensor", "achieved": achieved, "peak": NOMINAL_FP64_TENSOR_TFLOPS, "unit": "TFLOP/s",
            "frac": achieved / NOMINAL_FP64_TENSOR_TFLOPS, "peak_source": "nominal FP64 tensor rate",
            "algorithmic_flops_per_launch": flops_per_launch}


def tf32_tensor_roofline(hw_flops_per_launch: float, useful_flops_per_launch: float, avg_launch_s: float,
                         pk: dict) -> dict:
    """The roofline fields of a kernel bound by the TF32 tensor cores: the tensor FLOP it issues
    (three TF32 products over the padded tiles) against half the measured bf16 GEMM rate, TF32's
    dense rate being half of bf16's on this part (1.1 vs 2.25 PFLOP/s nominal)."""
    peak = pk["bf16_tflops"] / 2.0
    achieved = hw_flops_per_launch / avg_launch_s / 1e12 if avg_launch_s > 0 else 0.0
    return {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_source": "half the measured bf16 GEMM rate (TF32 dense rate)",
            "tensor_flops_per_launch": hw_flops_per_launch, "algorithmic_flops_per_launch": useful_flops_per_launch,
            "useful_tflops": useful_flops_per_launch / avg_launch_s / 1e12 if avg_launch_s > 0 else 0.0}


def committed_traffic(kernel: str, workload: str, algorithmic_bytes: float) -> float | None:
    """Per-launch DRAM bytes of a kernel: the measured DRAM bytes per algorithmic byte of its
    committed ncu capture (profiles/traffic.json, a smaller case of the same workload) times
    this launch's algorithmic bytes."""
    path = ROOT / "profiles" / "traffic.json"
    if not path.exists():
        return None
    entry = json.loads(path.read_text()).get("kernels", {}).get(f"{workload}:{kernel}")
    return None if entry is None else float(entry["dram_per_algorithmic_byte"]) * algorithmic_bytes


# The GPU arm prepares each synthetic volume's inputs with the product's device staging
# (stage_dwi); the CPU reference arm, which runs no GPU code, with the oracle's numpy staging.
# Both give the same float32 signals, and S0 and floors to 1e-13.
REFERENCE_ARM = False
# dRL's arithmetic in the drl and grl workloads: "fp64" (the reference's) or "tf32x3" (the
# 300-direction solves on the tcgen05 tensor cores).
DRL_PRECISION = "fp64"


def staged_inputs(w):
    """The mask voxels' float32 signals (v, N), S0 (v) and floors (v) of a synthetic volume."""
    if REFERENCE_ARM:
        from oracle import staging

        st = staging.stage(w.volume.data, w.volume.slope, w.volume.intercept, w.gtab.b0_mask, w.mask)
        return st["signals"], st["s0"], st["floor"]
    from larmor_b200.dwi.inputs import stage_dwi

    st = stage_dwi(w.volume, w.gtab, w.mask)
    return st.signals.cpu().numpy(), st.s0.cpu().numpy(), st.floor.cpu().numpy()


def strided(v: int, n: int) -> np.ndarray:
    """n voxel indices spread evenly over the whole volume (every voxel when v <= n)."""
    return np.arange(v) if v <= n else np.linspace(0, v - 1, n).round().astype(np.int64)


def tensor_fa_md(dt: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """FA and MD of tensors given as (v, 6) in the order xx, xy, xz, yy, yz, zz, by numpy's eigh
    (the reference's compute_dti_metrics, src/larmor/dwi/dti.py:170-235)."""
    xx, xy, xz, yy, yz, zz = dt.T
    t = np.stack([np.stack([xx, xy, xz], -1), np.stack([xy, yy, yz], -1), np.stack([xz, yz, zz], -1)], -2)
    ev = np.linalg.eigvalsh(t)
    md = ev.mean(axis=1)
    num = np.sqrt(((ev[:, 0] - ev[:, 1]) ** 2 + (ev[:, 1] - ev[:, 2]) ** 2 + (ev[:, 2] - ev[:, 0]) ** 2))
    den = np.sqrt((ev ** 2).sum(axis=1))
    fa = np.where(den > 1e-12, np.sqrt(0.5) * num / np.where(den > 1e-12, den, 1.0), 0.0)
    return np.clip(fa, 0.0, 1.0), md


def committed_issue(kernel: str, workload: str, algorithmic_bytes: float) -> dict | None:
    """Warp instructions per launch of a kernel: the measured warp instructions per algorithmic
    byte of its committed ncu capture (profiles/issue.json) times this launch's algorithmic
    bytes, with the capture's issue-active fraction and active lanes per instruction."""
    path = ROOT / "profiles" / "issue.json"
    if not path.exists():
        return None
    entry = json.loads(path.read_text()).get("kernels", {}).get(f"{workload}:{kernel}")
    if entry is None:
        return None
    return {"warp_instructions": float(entry["warp_instructions_per_algorithmic_byte"]) * algorithmic_bytes,
            "issue_active_pct_ncu": entry["issue_active_pct"], "threads_per_instruction": entry["threads_per_instruction"],
            "warp_instructions_per_voxel_round": entry.get("warp_instructions_per_voxel_round")}


def committed_fp64(kernel: str, workload: str) -> dict | None:
    """FP64 CUDA-core FLOP per voxel of a kernel from its committed ncu capture
    (profiles/fp64.json), or None."""
    path = ROOT / "profiles" / "fp64.json"
    if not path.exists():
        return None
    return json.loads(path.read_text()).get("kernels", {}).get(f"{workload}:{kernel}")


# ---- clocks ------------------------------------------------------------------------------

class ClockSampler:
    """Samples one GPU's SM clock and throttle reasons through NVML every 2 ms while running
    (nvidia-smi's 100 ms period misses timed regions of a few milliseconds)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, index: int) -> None:
        self.index = index
        self.samples: list[tuple[float, float, int]] = []
        self.stop = threading.Event()
        self.thread = None

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nvml = pynvml
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(self.index)
        except Exception:  # noqa: BLE001 - no NVML: no clock record
            self.nvml = None
            return self
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()
        return self

    def _run(self):
        nv, h = self.nvml, self.handle
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(mx), int(reasons)))
            except Exception:  # noqa: BLE001
                pass
            time.sleep(0.002)

    def __exit__(self, *exc):
        self.stop.set()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "source": "nvml"}
        reasons = sorted({name for _, _, r in self.samples for name, bit in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(x[0] for x in self.samples),
                "sm_max_mhz": max(x[1] for x in self.samples), "reasons": reasons,
                "samples": len(self.samples), "source": "nvml"}


# ---- workloads ---------------------------------------------------------------------------

class DtiWorkload:
    """Config 1: DTI WLLS on the 64x64x40 volume (79,912 voxels, 1 b0 + 30 directions). value:
    the fused fit and maps with the staged signals resident; e2e: the public model call
    DTIModel(fit_method="wls").fit(volume, gtab, mask), raw host volume in, host maps out."""

    name = "dti_wlls_64x64x40"
    kernels = ("fit_dti_maps_kernel",)
    has_fp32 = True
    # Algorithmic bytes per voxel: 31 float32 samples in, 16 float32 maps + 1 byte out
    # (the 8-byte floor per voxel is host-prepared input too).
    bytes_per_voxel = 4 * 31 + 8 + 16 * 4 + 1

    def __init__(self, seed: int) -> None:
        from larmor_b200.dwi.dti import dti_design
        from larmor_b200.synthetic import dti_volume

        w = self.w = dti_volume(seed=seed)
        self.mask = w.mask
        self.config = {"workload": self.name, "grid": [64, 64, 40], "voxels": w.n_voxels,
                       "measurements": 31, "fit": "wls", "l2": "flushed (256 MiB write) before each step",
                       "e2e_api": "DTIModel(fit_method='wls').fit(volume, gtab, mask)"}
        self.design = dti_design(w.gtab)
        self.signals, _, self.floor = staged_inputs(w)
        self.v = len(self.signals)

    def subset(self, n: int) -> None:
        self.signals, self.floor = self.signals[:n], self.floor[:n]
        self.v = len(self.signals)
        flat = np.flatnonzero(self.mask)
        keep = np.zeros(self.mask.size, dtype=bool)
        keep[flat[:n]] = True
        self.mask = keep.reshape(self.mask.shape)
        self.config["voxels"] = self.v

    def device_setup(self, torch, dev):
        from larmor_b200 import _core

        self.handle = _core.LogDesign.cached(self.design, np.zeros((0, 7)))
        self.d_signals = torch.from_numpy(self.signals).to(dev)
        self.d_floor = torch.from_numpy(self.floor).to(dev)
        self.d_maps = torch.empty((16, self.v), dtype=torch.float32, device=dev)
        self.d_npd = torch.empty((self.v,), dtype=torch.uint8, device=dev)
        # The model call copies the raw volume and the mask voxels' indices in, the masked maps out.
        self.h2d_bytes = self.w.volume.data.nbytes + 8 * self.v
        self.d2h_bytes = 16 * 4 * self.v + self.v

    def step_device(self, precision=0):
        from larmor_b200 import _core

        _core.fit_dti_maps_device(self.handle, self.d_signals, self.d_floor, True, self.d_maps,
                                  self.d_npd, precision=precision)

    def kernel_bytes(self) -> dict:
        """Algorithmic DRAM bytes of one step, per kernel (all its launches in the step)."""
        return {"fit_dti_maps_kernel": self.bytes_per_voxel * self.v}

    def step_e2e(self):
        from larmor_b200.dwi import DTIModel

        self.e2e_fit = DTIModel(fit_method="wls").fit(self.w.volume, self.w.gtab, self.mask)

    def cpu_sample(self, threads: int, budget_s: float) -> tuple[int, float, str]:
        from oracle import oracle as o

        log_s = np.log(np.where((self.signals > 0) & np.isfinite(self.signals), self.signals,
                                self.floor[:, None]).astype(np.float64))
        o.fit_log_signal(self.design, None, log_s[:256], True, n_threads=threads)  # warm-up
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < budget_s:
            params, _ = o.fit_log_signal(self.design, None, log_s, True, n_threads=threads)
            done += len(log_s)
        self.reference_params = params
        return done, time.perf_counter() - t0, f"whole volume ({self.v} voxels) repeated for ~{budget_s:.0f} s"

    def parity(self) -> dict:
        """FA and MD of every voxel, from the device's fused fit and maps (float32 maps) and from
        the FP64 oracle's parameters of the cpu_baseline run (numpy eigh), and the tensors."""
        self.step_device()
        maps = self.d_maps.cpu().numpy().astype(np.float64)
        fa, md = tensor_fa_md(self.reference_params[:, 1:7])
        fa_err = float(np.abs(maps[6] - fa).max())
        md_err = float(np.abs(maps[7] - md).max())
        dt_rel = float((np.abs(maps[0:6].T - self.reference_params[:, 1:7]).max(axis=1)
                        / np.abs(self.reference_params[:, 1:7]).max(axis=1)).max())
        return {"against": "FP64 oracle (C++ restatement of cpp/src/dwi/log_fit.cpp), numpy eigh for FA/MD",
                "voxels": self.v, "fa_abs_max": fa_err, "md_abs_max": md_err, "dt_rel_max": dt_rel,
                "tolerance": {"fa_abs": 1e-4, "md_abs": 1e-4},
                "within_tolerance": bool(fa_err <= 1e-4 and md_err <= 1e-4)}

    def fp32_parity(self) -> dict:
        """The plain FP32 kernel's FA, MD and tensors against the same FP64 oracle fit."""
        self.step_device(precision=1)
        maps = self.d_maps.cpu().numpy().astype(np.float64)
        fa, md = tensor_fa_md(self.reference_params[:, 1:7])
        ref = self.reference_params[:, 1:7]
        return {"fa_abs_max": float(np.abs(maps[6] - fa).max()), "md_abs_max": float(np.abs(maps[7] - md).max()),
                "dt_rel_max": float((np.abs(maps[0:6].T - ref).max(axis=1) / np.abs(ref).max(axis=1)).max())}


class DtiModelWorkload:
    """Config 1 through the model API: DTIModel(fit_method="wls").fit(volume, gtab, mask) on the
    64x64x40 volume (79,912 mask voxels), from the raw float32 volume to the maps. The device
    stages the inputs: the mask voxels' samples, S0 with its neighbourhood repair, the
    per-voxel floors (lar_stage_dwi); then the fused fit and maps. value: staging + fit with the
    raw volume resident; e2e: the whole model call, host volume in, host maps out."""

    name = "dti_model_wlls_64x64x40"
    kernels = ("stage_gather_kernel", "stage_index_kernel", "stage_repair_kernel", "stage_floor_kernel",
               "fit_dti_maps_kernel")
    has_fp32 = False

    def __init__(self, seed: int) -> None:
        from larmor_b200.synthetic import dti_volume

        self.w = dti_volume(seed=seed)
        self.mask = self.w.mask
        self.v = int(self.mask.sum())
        self.config = {"workload": self.name, "grid": [64, 64, 40], "voxels": self.v, "measurements": 31,
                       "fit": "wls", "api": "DTIModel.fit (model level, raw volume in)",
                       "l2": "flushed (256 MiB write) before each step"}

    def subset(self, n: int) -> None:
        flat = np.flatnonzero(self.mask)
        keep = np.zeros(self.mask.size, dtype=bool)
        keep[flat[:n]] = True
        self.mask = keep.reshape(self.mask.shape)
        self.v = int(self.mask.sum())
        self.config["voxels"] = self.v

    def device_setup(self, torch, dev):
        from larmor_b200 import _core
        from larmor_b200.dwi.dti import dti_design
        from larmor_b200.dwi.inputs import upload_volume

        self.torch = torch
        self.raw = upload_volume(self.w.volume)
        self.flat = torch.from_numpy(np.flatnonzero(self.mask).astype(np.int64)).to(dev)
        self.handle = _core.LogDesign.cached(dti_design(self.w.gtab), np.zeros((0, 7)))
        self.d_maps = torch.empty((16, self.v), dtype=torch.float32, device=dev)
        self.d_npd = torch.empty((self.v,), dtype=torch.uint8, device=dev)
        self.h2d_bytes = self.w.volume.data.nbytes + 8 * self.v
        self.d2h_bytes = 16 * 4 * self.v + self.v

    def step_device(self, precision=0):
        from larmor_b200 import _core
        from larmor_b200.dwi.inputs import stage_dwi

        staged = stage_dwi(self.w.volume, self.w.gtab, self.mask, raw=self.raw, flat=self.flat)
        _core.fit_dti_maps_device(self.handle, staged.signals, staged.floor, True, self.d_maps, self.d_npd)

    def kernel_bytes(self) -> dict:
        """Algorithmic DRAM bytes of one step: the gather reads 31 float32 samples and writes 31
        float32 signals, the raw S0, a state byte, the row maximum and a finite byte per voxel;
        the index map write and the repair read 4 + 8 bytes per voxel; the floors 8 + 8; the fit
        reads the signals and the floor and writes 16 float32 maps and a byte."""
        v = self.v
        return {"stage_gather_kernel": v * (31 * 4 * 2 + 8 + 1 + 8 + 1 + 8), "stage_index_kernel": v * 12,
                "stage_repair_kernel": v * (8 + 1 + 8 + 8), "stage_floor_kernel": v * 24,
                "fit_dti_maps_kernel": v * (4 * 31 + 8 + 16 * 4 + 1)}

    def step_e2e(self):
        from larmor_b200.dwi import DTIModel

        DTIModel(fit_method="wls").fit(self.w.volume, self.w.gtab, self.mask)

    def cpu_sample(self, threads: int, budget_s: float) -> tuple[int, float, str]:
        from larmor_b200.dwi.dti import dti_design
        from oracle import oracle as o
        from oracle import staging

        design = dti_design(self.w.gtab)
        vol = self.w.volume
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < budget_s:
            st = staging.stage(vol.data, vol.slope, vol.intercept, self.w.gtab.b0_mask, self.mask)
            sig = st["signals"].astype(np.float64)
            log_s = np.log(np.where((sig > 0) & np.isfinite(sig), sig, st["floor"][:, None]))
            o.fit_log_signal(design, None, log_s, True, n_threads=threads)
            done += self.v
        return done, time.perf_counter() - t0, (f"whole volume ({self.v} voxels): the oracle's staging (numpy) and "
                                                f"FP64 fit, repeated for ~{budget_s:.0f} s")


class DkiWorkload:
    """Config 2: constrained DKI WLLS on the 96x96x60 volume (199,768 voxels, 6 b0 + 2 x 64)."""

    name = "dki_wlls_96x96x60"
    kernels = ("fit_log_warp_kernel", "constrained_fit_kernel", "dki_maps_kernel")
    has_fp32 = True
    # 134 float32 samples + S0 and floor (double) in; 36 float32 maps + npd + broke out.
    bytes_per_voxel = 4 * 134 + 16 + 36 * 4 + 2

    def __init__(self, seed: int) -> None:
        from larmor_b200.dwi.dki import dki_constraints, dki_design
        from larmor_b200.synthetic import dki_volume

        w = dki_volume(seed=2 + 10 * (seed - 1))
        self.design = dki_design(w.gtab)
        self.g = dki_constraints(w.gtab)
        self.signals, self.s0, self.floor = staged_inputs(w)
        self.is_b0 = w.gtab.b0_mask.astype(np.uint8)
        self.v = len(self.signals)
        self.config = {"workload": self.name, "grid": [96, 96, 60], "voxels": self.v, "measurements": 134,
                       "fit": "wls, constrained (768 constraints)", "l2": "flushed (256 MiB write) before each step"}

    def subset(self, n: int) -> None:
        self.signals, self.s0, self.floor = self.signals[:n], self.s0[:n], self.floor[:n]
        self.v = len(self.signals)
        self.config["voxels"] = self.v

    def device_setup(self, torch, dev):
        from larmor_b200 import _core

        self.torch = torch
        self.handle = _core.LogDesign.cached(self.design, self.g)
        up = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        self.d_signals, self.d_s0, self.d_floor, self.d_b0 = up(self.signals), up(self.s0), up(self.floor), up(self.is_b0)
        self.d_maps = torch.empty((36, self.v), dtype=torch.float32, device=dev)
        self.d_npd = torch.empty((self.v,), dtype=torch.uint8, device=dev)
        self.d_broke = torch.empty((self.v,), dtype=torch.uint8, device=dev)
        self.d_params = torch.empty((self.v, 22), dtype=torch.float64, device=dev)
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
        self.h_signals, self.h_s0, self.h_floor = pin(self.signals), pin(self.s0), pin(self.floor)
        self.h_maps = torch.empty((36, self.v), dtype=torch.float32).pin_memory()
        self.h_npd = torch.empty((self.v,), dtype=torch.uint8).pin_memory()
        self.h2d_bytes = self.signals.nbytes + self.s0.nbytes + self.floor.nbytes
        self.d2h_bytes = 36 * 4 * self.v + self.v

    def step_device(self, precision=0):
        from larmor_b200 import _core, _lib

        _lib.check(_lib.lib().lar_fit_dki_maps(
            self.handle.handle, _lib.ptr(self.d_signals), _lib.ptr(self.d_s0), _lib.ptr(self.d_floor),
            _lib.ptr(self.d_b0), self.v, 1, 20, 1e-6, precision, _lib.ptr(self.d_maps), _lib.ptr(self.d_npd),
            _lib.ptr(self.d_broke), _lib.ptr(self.d_params), _core._stream(self.torch)))

    def kernel_bytes(self) -> dict:
        """Algorithmic DRAM bytes of one step, per kernel: the IRLS fit reads the float32
        signals, S0 and floor and writes the parameters and broke flags; the constrained re-fit
        reads the same inputs and the listed parameters of each violator and writes its
        parameters; the maps read the parameters and write 36 float32 maps and npd."""
        self.torch.cuda.synchronize()
        n_viol = self.handle.violators()
        inputs = 4 * 134 + 16
        return {"fit_log_warp_kernel": self.v * (inputs + 22 * 8 + 1),
                "constrained_fit_kernel": n_viol * (inputs + 2 * 22 * 8),
                "dki_maps_kernel": self.v * (22 * 8 + 36 * 4 + 1)}

    def step_e2e(self):
        self.d_signals.copy_(self.h_signals, non_blocking=True)
        self.d_s0.copy_(self.h_s0, non_blocking=True)
        self.d_floor.copy_(self.h_floor, non_blocking=True)
        self.step_device()
        self.h_maps.copy_(self.d_maps, non_blocking=True)
        self.h_npd.copy_(self.d_npd, non_blocking=True)

    def cpu_sample(self, threads: int, budget_s: float) -> tuple[int, float, str]:
        from oracle import oracle as o

        n = min(self.v, 16384)
        s = self.signals[:n].astype(np.float64)
        is_b0 = self.is_b0.astype(bool)
        s0 = self.s0[:n]
        own = s[:, is_b0].mean(axis=1)
        rep = ~np.isclose(s0, own, rtol=1e-9, atol=0.0)
        s[np.ix_(rep, is_b0)] = s0[rep, None]
        s[:, ~is_b0] = np.minimum(s[:, ~is_b0], s0[:, None])
        bad = ~(np.isfinite(s) & (s > 0))
        s[bad] = np.broadcast_to(self.floor[:n, None], s.shape)[bad]
        log_s = np.log(s)
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < budget_s:
            o.fit_log_signal(self.design, self.g, log_s, True, n_threads=threads)
            done += n
        return done, time.perf_counter() - t0, f"first {n} voxels of the volume, repeated for ~{budget_s:.0f} s (fit only)"


class _SdWorkloadBase:
    """The config-3 volume (110x110x70, 500,040 voxels, 10 b0 + 3 x 90) for the SD fits."""

    def _volume(self, seed: int):
        from larmor_b200.synthetic import mfod_volume

        w = mfod_volume(seed=3 + 10 * (seed - 1))
        self.gtab = w.gtab
        signals, self.s0, _ = staged_inputs(w)
        self.signals = signals.astype(np.float64)
        self.v = len(self.signals)

    def subset(self, n: int) -> None:
        self.signals, self.s0 = self.signals[:n], self.s0[:n]
        if hasattr(self, "norm"):
            self.norm = self.norm[:n]
        self.v = len(self.signals)
        self.config["voxels"] = self.v


class MfodWorkload(_SdWorkloadBase):
    """Config 3: three-tissue mFOD (SDModel, method mFOD): WM L2NNLS FOD on 300 directions
    (44 in the loop) + GM + CSF, up to 50 rounds, on S0-normalised signals. value: the fit with
    the signals resident; e2e: the drop-in call _core.fit_multi_tissue with host numpy arrays
    (float64 signals in, new FOD and fraction arrays out)."""

    name = "mfod_3tissue_110x110x70"
    kernels = ("correlate_kernel", "ridge_nnls_half_kernel<3>", "ridge_nnls_kernel<1,2>", "lr_fractions_kernel",
               "ridge_nnls_first_kernel<1,10>", "ridge_nnls_kernel<8,10>", "hr_fractions_kernel")
    has_fp32 = True
    fraction_tol = 1e-7
    # The plain FP32 fit takes seconds per step: a few timed steps bound the run.
    fp32_steps = 2
    fp32_what = ("lar_fit_multi_tissue_plain_fp32: one warp per voxel runs all its rounds in FP32 with the "
                 "textbook Lawson-Hanson steps (the direct GPU port of the reference's per-voxel loop)")
    # 280 double samples in, 300 double amplitudes + 3 fractions out.
    bytes_per_voxel = 8 * 280 + 8 * 303

    def __init__(self, seed: int) -> None:
        from larmor_b200.synthetic import mfod_model_responses

        from larmor_b200.sd.kernel import Kernel
        from larmor_b200.sd.model import compute_shell_weights, low_resolution_dirs
        from larmor_b200.sd.sphere import DIRS_300

        self._volume(seed)
        self.norm = np.ascontiguousarray(np.minimum(self.signals / self.s0[:, None], 1.0))
        rfs = mfod_model_responses()
        weights = compute_shell_weights(self.gtab.bvals, 1.0)
        b, g = self.gtab.bvals, self.gtab.bvecs
        self.hr = Kernel(rfs, b, g, dirs=DIRS_300, weights=weights)
        self.lr = Kernel(rfs, b, g, dirs=low_resolution_dirs(rfs, len(b)), weights=weights)
        self.config = {"workload": self.name, "grid": [110, 110, 70], "voxels": self.v, "measurements": 280,
                       "tissues": "WM (lmax 8 output, 300 directions) + GM + CSF", "max_rounds": 50,
                       "fraction_tol": 1e-7, "l2": "inputs (1.1 GB) larger than L2",
                       "e2e_api": "_core.fit_multi_tissue(numpy float64 signals) -> numpy FODs, fractions"}

    def sd_solver(self):
        from larmor_b200.sd.solvers import L2NNLS

        return L2NNLS()

    def device_setup(self, torch, dev):
        from larmor_b200.sd.solvers import Stage, _deconv_kernel

        self.torch = torch
        self.k_lr, self.k_hr = _deconv_kernel(self.lr), _deconv_kernel(self.hr)
        self.hr_solver = self.sd_solver()._prepare(self.hr, self.gtab.bvals, Stage.HIGH_RES)
        self.lr_solver = self.sd_solver()._prepare(self.lr, self.gtab.bvals, Stage.LOW_RES)
        self.d_signals = torch.from_numpy(self.norm).to(dev)
        self.d_fods = torch.empty((self.v, self.k_hr.ca), dtype=torch.float64, device=dev)
        self.d_fr = torch.empty((self.v, 3), dtype=torch.float64, device=dev)
        self.h2d_bytes = self.norm.nbytes
        self.d2h_bytes = self.v * (self.k_hr.ca + 3) * 8
        if type(self) is MfodWorkload:
            # The plain single-precision fit's inputs and outputs.
            self.d_signals32 = self.d_signals.float()
            self.d_fods32 = torch.empty((self.v, self.k_hr.ca), dtype=torch.float32, device=dev)
            self.d_fr32 = torch.empty((self.v, 3), dtype=torch.float32, device=dev)
            self.d_rounds32 = torch.empty((self.v,), dtype=torch.int32, device=dev)
            self.d_status32 = torch.empty((self.v,), dtype=torch.uint8, device=dev)

    def step_device(self, precision=0):
        from larmor_b200 import _core

        if precision == 1:
            _core.fit_multi_tissue_plain_fp32_device(self.d_signals32, self.lr.weights, self.k_lr, self.lr_solver,
                                                     self.k_hr, self.hr_solver, 50, 1e-7, 1e-2, self.d_fods32,
                                                     self.d_fr32, self.d_rounds32, self.d_status32)
            return
        _core.fit_multi_tissue_device(self.d_signals, self.lr.weights, self.k_lr, self.lr_solver, self.k_hr,
                                      self.hr_solver, 50, 1e-7, 1e-2, self.d_fods, self.d_fr)

    def kernel_bytes(self) -> dict:
        """Algorithmic DRAM bytes of one step, per kernel. A voxel-round of the low-resolution
        loop correlates the 280 signals (read) into 44 correlations (written), whose NNLS reads
        them and writes 44 amplitudes, whose fractions read those and the signals and write 3
        fractions; the high-resolution pass does the same with 300 directions once per voxel."""
        from larmor_b200 import _core

        torch = self.torch
        rounds = torch.zeros((self.v,), dtype=torch.int32, device=self.d_signals.device)
        _core.fit_multi_tissue_device(self.d_signals, self.lr.weights, self.k_lr, self.lr_solver, self.k_hr,
                                      self.hr_solver, 50, 1e-7, 1e-2, self.d_fods, self.d_fr, rounds=rounds)
        self.d_rounds = rounds
        vr = int(rounds.sum().item())
        m, c_lr, c_hr = 280, self.k_lr.ca, self.k_hr.ca
        # The low-resolution NNLS runs two voxels per warp and the high-resolution one a first
        # pass with a 32-column factor; the full-factor kernels refit only the few voxels handed
        # back (counted with the first kernels').
        return {"correlate_kernel": vr * 8 * (m + c_lr) + self.v * 8 * (m + c_hr),
                "ridge_nnls_half_kernel<3>": vr * 8 * 2 * c_lr,
                "ridge_nnls_kernel<1,2>": 0,
                "lr_fractions_kernel": vr * 8 * (c_lr + m + 3),
                "ridge_nnls_first_kernel<1,10>": self.v * 8 * 2 * c_hr,
                "ridge_nnls_kernel<8,10>": 0,
                "hr_fractions_kernel": self.v * 8 * (c_hr + m + 3)}

    def step_e2e(self):
        from larmor_b200 import _core

        self.e2e_out = _core.fit_multi_tissue(self.norm, self.lr.weights, self.k_lr, self.lr_solver, self.k_hr,
                                              self.hr_solver, 50, self.fraction_tol, 1e-2, n_threads=1)

    def cpu_sample(self, threads: int, budget_s: float) -> tuple[int, float, str]:
        from oracle import oracle as o

        self.sample = idx = strided(self.v, 2048)
        signals = np.ascontiguousarray(self.norm[idx])
        lr = dict(k_aniso=self.lr.k_aniso, k_iso=self.lr.k_iso, w_k_iso=self.lr.w_k_iso, w_k_aniso=self.lr.w_k_aniso)
        hr = dict(k_aniso=self.hr.k_aniso, k_iso=self.hr.k_iso, w_k_iso=self.hr.w_k_iso, w_k_aniso=self.hr.w_k_aniso,
                  blocks=[(b.start, b.stop) for b in self.hr.aniso_blocks])
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < budget_s:
            out = o.fit_multi_tissue(signals, self.lr.weights, lr, hr, n_threads=threads, rounds=True)
            done += len(idx)
        self.reference_out = out
        return done, time.perf_counter() - t0, (f"{len(idx)} voxels spread evenly over the volume, repeated for "
                                                f"~{budget_s:.0f} s")

    def fp32_parity(self) -> dict:
        """The plain FP32 fit against the same FP64 oracle fit of the cpu_baseline sample."""
        fods, fr, rounds = self.reference_out
        self.step_device(precision=1)
        idx = self.torch.from_numpy(self.sample).to(self.d_fods32.device)
        got = self.d_fods32[idx].double().cpu().numpy()
        got_fr = self.d_fr32[idx].double().cpu().numpy()
        got_rounds = self.d_rounds32[idx].cpu().numpy()
        status = self.d_status32[idx].cpu().numpy()
        scale = np.maximum(np.abs(fods).max(axis=1), 1e-300)
        rel = np.abs(got - fods).max(axis=1) / scale
        return {"voxels": int(len(self.sample)), "fod_rel_max": float(rel.max()),
                "fod_rel_median": float(np.median(rel)), "fod_rel_p99": float(np.percentile(rel, 99)),
                "fractions_abs_max": float(np.abs(got_fr - fr).max()),
                "identical_active_sets": float(((got > 0) == (fods > 0)).all(axis=1).mean()),
                "identical_round_counts": float((got_rounds == rounds).mean()),
                "status_nonzero": float((status != 0).mean())}

    def parity(self) -> dict:
        """The device fit of the whole volume against the FP64 oracle on the cpu_baseline sample:
        the FOD amplitudes' largest error relative to the voxel's largest amplitude, the
        fractions' largest absolute error, and how many voxels have the oracle's final active
        set (the zero pattern of the 300 amplitudes) and round count."""
        fods, fr, rounds = self.reference_out
        idx = self.torch.from_numpy(self.sample).to(self.d_fods.device)
        got = self.d_fods[idx].cpu().numpy()
        got_fr = self.d_fr[idx].cpu().numpy()
        got_rounds = self.d_rounds[idx].cpu().numpy()
        scale = np.maximum(np.abs(fods).max(axis=1), 1e-300)
        rel = float((np.abs(got - fods).max(axis=1) / scale).max())
        fr_err = float(np.abs(got_fr - fr).max())
        same_set = float(((got > 0) == (fods > 0)).all(axis=1).mean())
        same_rounds = float((got_rounds == rounds).mean())
        e2e_fods, e2e_fr = self.e2e_out
        e2e_same = bool(np.array_equal(e2e_fods[self.sample], got) and np.array_equal(e2e_fr[self.sample], got_fr))
        return {"against": "FP64 oracle (C++ restatement of cpp/src/sd/{nnls,fractions,multi_tissue}.cpp)",
                "voxels": int(len(self.sample)), "sample": "spread evenly over the volume",
                "fods": "the 300 high-resolution amplitudes",
                "fod_rel_max": rel, "fractions_abs_max": fr_err,
                "identical_active_sets": same_set, "identical_round_counts": same_rounds,
                "e2e_equals_device_fit": e2e_same,
                "tolerance": {"fod_rel": 1e-4, "fractions_abs": 1e-4, "identical_active_sets": 1.0},
                "within_tolerance": bool(rel <= 1e-4 and fr_err <= 1e-4 and same_set == 1.0)}


class MsmtWorkload(_SdWorkloadBase):
    """Config 3 through MSMT-CSD: LSI with 47 unknowns (WM lmax 8 + GM + CSF) and 302
    constraints (300 directions + 2) per voxel."""

    name = "msmt_csd_lsi_110x110x70"
    kernels = ("lsi_kernel",)
    has_fp32 = True
    fp32_steps = 1
    fp32_what = ("lar_fit_lsi_plain_fp32: one warp per voxel runs the LSI steps in FP32, the Cholesky factor of the "
                 "active constraints formed anew for every fit, no QR fallback")
    bytes_per_voxel = 8 * 280 + 8 * 47 + 1

    def __init__(self, seed: int) -> None:
        self._volume(seed)
        self.config = {"workload": self.name, "grid": [110, 110, 70], "voxels": self.v, "measurements": 280,
                       "unknowns": 47, "constraints": 302, "l2": "inputs (1.1 GB) larger than L2"}

    def device_setup(self, torch, dev):
        from larmor_b200.sd.msmt import prepare_msmt
        from larmor_b200.sd.sphere import DIRS_300
        from larmor_b200.synthetic import mfod_responses

        self.torch = torch
        self.design = prepare_msmt(mfod_responses(), [8, 0, 0], self.gtab.bvals, self.gtab.bvecs, DIRS_300)
        self.d_signals = torch.from_numpy(self.signals).to(dev)
        self.d_x = torch.empty((self.v, 47), dtype=torch.float64, device=dev)
        self.d_conv = torch.empty((self.v,), dtype=torch.uint8, device=dev)
        self.h_signals = torch.from_numpy(self.signals).pin_memory()
        self.h_x = torch.empty((self.v, 47), dtype=torch.float64).pin_memory()
        self.h_conv = torch.empty((self.v,), dtype=torch.uint8).pin_memory()
        self.h2d_bytes = self.signals.nbytes
        self.d2h_bytes = self.v * (47 * 8 + 1)
        self.d_signals32 = self.d_signals.float()
        self.d_x32 = torch.empty((self.v, 47), dtype=torch.float32, device=dev)
        self.d_status32 = torch.empty((self.v,), dtype=torch.uint8, device=dev)

    def step_device(self, precision=0):
        from larmor_b200 import _core

        if precision == 1:
            _core.fit_lsi_plain_fp32_device(self.design, self.d_signals32, self.d_x32, self.d_status32)
            return
        _core.fit_lsi_device(self.design, self.d_signals, self.d_x, self.d_conv)

    def kernel_bytes(self) -> dict:
        """Algorithmic DRAM bytes of one step: 280 signals in, 47 coefficients and a flag out."""
        return {"lsi_kernel": self.bytes_per_voxel * self.v}

    def step_e2e(self):
        self.d_signals.copy_(self.h_signals, non_blocking=True)
        self.step_device()
        self.h_x.copy_(self.d_x, non_blocking=True)
        self.h_conv.copy_(self.d_conv, non_blocking=True)

    def cpu_sample(self, threads: int, budget_s: float) -> tuple[int, float, str]:
        from larmor_b200.sd.msmt import constraint_matrix, forward_matrix, NORM_REG
        from larmor_b200.sd.sphere import DIRS_300
        from larmor_b200.synthetic import mfod_responses
        from oracle import oracle as o

        f = forward_matrix(mfod_responses(), [8, 0, 0], self.gtab.bvals, self.gtab.bvecs)
        g = constraint_matrix([8, 0, 0], DIRS_300)
        ridge = float(np.sqrt(NORM_REG * np.max(np.sum(f**2, axis=0))))
        n = min(self.v, 8192)
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < budget_s:
            out = o.fit_lsi(f, g, ridge, self.signals[:n], n_threads=threads)
            done += n
        self.reference_out = out
        return done, time.perf_counter() - t0, f"first {n} voxels of the volume, repeated for ~{budget_s:.0f} s"

    def _against_oracle(self, x) -> dict:
        ref, ref_conv = self.reference_out
        got = x[:len(ref)].double().cpu().numpy()
        scale = np.maximum(np.abs(ref).max(axis=1), 1e-300)
        rel = np.abs(got - ref).max(axis=1) / scale
        return {"voxels": int(len(ref)), "x_rel_max": float(rel.max()), "x_rel_median": float(np.median(rel)),
                "x_rel_p99": float(np.percentile(rel, 99))}

    def parity(self) -> dict:
        """The device fit against the FP64 oracle on the cpu_baseline sample: each voxel's largest
        coefficient error relative to its largest coefficient."""
        out = self._against_oracle(self.d_x)
        out.update({"against": "FP64 oracle (C++ restatement of cpp/src/sd/lsi.cpp)", "sample": "first voxels",
                    "converged_identical": float((self.d_conv[:out["voxels"]].cpu().numpy().astype(bool)
                                                  == self.reference_out[1]).mean()),
                    "tolerance": {"x_rel": 1e-4}})
        out["within_tolerance"] = bool(out["x_rel_max"] <= 1e-4)
        return out

    def fp32_parity(self) -> dict:
        """The plain FP32 fit against the same FP64 oracle fit."""
        self.step_device(precision=1)
        out = self._against_oracle(self.d_x32)
        out["status_nonzero"] = float((self.d_status32[:out["voxels"]].cpu().numpy() != 0).mean())
        return out


def _job_kernel_bytes(job) -> dict:
    """Algorithmic DRAM bytes of one job of a batch, per kernel (as the single workloads count
    them); the DKI violator count and the mFOD rounds come from the job's last fit."""
    v, n = job.voxels, job.signals.shape[1]
    if job.kind == "dti":
        return {"fit_dti_maps_kernel": v * (4 * n + 8 + 16 * 4 + 1)}
    if job.kind == "dki":
        viol = int(job.out["broke"].sum().item())  # the voxels whose fit broke a constraint
        return {"fit_log_warp_kernel": v * (4 * n + 16 + 22 * 8 + 1),
                "constrained_fit_kernel": viol * (4 * n + 16 + 2 * 22 * 8),
                "dki_maps_kernel": v * (22 * 8 + 36 * 4 + 1)}
    vr = int(job.out["rounds"].sum().item())
    c_lr, c_hr = job.handles["k_lr"].ca, job.handles["k_hr"].ca
    return {"correlate_kernel": vr * 8 * (n + c_lr) + v * 8 * (n + c_hr),
            "ridge_nnls_half_kernel<3>": vr * 8 * 2 * c_lr,
            "ridge_nnls_kernel<1,2>": 0,
            "lr_fractions_kernel": vr * 8 * (c_lr + n + 3),
            "ridge_nnls_first_kernel<1,10>": v * 8 * 2 * c_hr,
            "ridge_nnls_kernel<8,10>": 0,
            "hr_fractions_kernel": v * 8 * (c_hr + n + 3)}


# The kernels of the per-family work queues and the single-volume kernels whose per-voxel work
# they do (the same algorithmic bytes).
QUEUE_KERNELS = {"batch_dti_kernel": "fit_dti_maps_kernel", "batch_log_warp_kernel": "fit_log_warp_kernel",
                 "batch_refit_kernel": "constrained_fit_kernel", "batch_dki_maps_kernel": "dki_maps_kernel",
                 "batch_plan_kernel": None, "batch_correlate_kernel": "correlate_kernel",
                 "batch_half_kernel<3>": "ridge_nnls_half_kernel<3>", "batch_redo_kernel<1,2>": "ridge_nnls_kernel<1,2>",
                 "batch_lr_fractions_kernel": "lr_fractions_kernel",
                 "batch_first_kernel<1,10>": "ridge_nnls_first_kernel<1,10>",
                 "batch_redo_kernel<8,10>": "ridge_nnls_kernel<8,10>",
                 "batch_hr_fractions_kernel": "hr_fractions_kernel"}


class BatchWorkload:
    """Config 4: 64 seeded volumes of uneven size (10k-400k voxels), gradient table (1-3 shells
    of 30-90 directions) and model (DTI/DKI/mFOD 40/20/40), all fitted by one replay of one
    CUDA graph: each model family's stages are single launches over all of its volumes, taking
    (volume, voxel-block) tickets from one device queue; the three families run side by side."""

    name = "batch_uneven_64_volumes"
    kernels = tuple(QUEUE_KERNELS)
    has_fp32 = False

    def __init__(self, seed: int) -> None:
        from larmor_b200.batch import generate_jobs

        self.jobs = generate_jobs(seed=4 + 10 * (seed - 1))
        self.v = sum(j.voxels for j in self.jobs)
        kinds = {k: sum(1 for j in self.jobs if j.kind == k) for k in ("dti", "dki", "mfod")}
        self.config = {"workload": self.name, "volumes": len(self.jobs), "voxels": self.v, "jobs": kinds,
                       "voxels_per_volume": [min(j.voxels for j in self.jobs), max(j.voxels for j in self.jobs)],
                       "launch": "one CUDA graph replay per step: one work queue per model family "
                                 "(3 parallel branches)",
                       "l2": "inputs (4.8 GB) larger than L2"}

    def subset(self, n: int) -> None:
        self.jobs = self.jobs[:max(1, n)]
        self.v = sum(j.voxels for j in self.jobs)
        self.config["volumes"], self.config["voxels"] = len(self.jobs), self.v

    def device_setup(self, torch, dev):
        from larmor_b200.batch import Batch

        self.torch = torch
        self.batch = Batch(self.jobs, tune=True)
        self.config["launch_settings"] = self.batch.launch_settings
        self.batch.capture()
        self.h_in = [tuple(torch.from_numpy(np.ascontiguousarray(t.cpu().numpy())).pin_memory() for t in j.d_in)
                     for j in self.jobs]
        self.h_out = [{k: torch.empty(t.shape, dtype=t.dtype).pin_memory() for k, t in j.out.items()}
                      for j in self.jobs]
        self.h2d_bytes = sum(t.numel() * t.element_size() for ts in self.h_in for t in ts)
        self.d2h_bytes = sum(t.numel() * t.element_size() for o in self.h_out for t in o.values())

    def step_device(self, precision=0):
        self.batch.run()

    def step_eager(self):
        """The same work launched kernel by kernel (for per-kernel event timing)."""
        self.batch.run_eager()

    def graph_launches(self) -> int:
        return self.batch.graph_kernels

    def step_e2e(self):
        for j, hin in zip(self.jobs, self.h_in):
            for d, h in zip(j.d_in, hin):
                d.copy_(h, non_blocking=True)
        self.batch.run()
        for j, hout in zip(self.jobs, self.h_out):
            for k, t in j.out.items():
                hout[k].copy_(t, non_blocking=True)

    def kernel_bytes(self) -> dict:
        self.torch.cuda.synchronize()
        single: dict = {}
        for j in self.jobs:
            for k, b in _job_kernel_bytes(j).items():
                single[k] = single.get(k, 0) + b
        return {k: single.get(v, 0) if v else 0 for k, v in QUEUE_KERNELS.items()}

    def cpu_sample(self, threads: int, budget_s: float) -> tuple[int, float, str]:
        from larmor_b200.dwi.dki import dki_constraints, dki_design
        from larmor_b200.dwi.dti import dti_design
        from larmor_b200.sd.kernel import Kernel
        from larmor_b200.sd.model import compute_shell_weights, low_resolution_dirs
        from larmor_b200.sd.sphere import DIRS_300
        from oracle import oracle as o

        calls = []
        for j in self.jobs:
            n = min(j.voxels, 128)
            if j.kind in ("dti", "dki"):
                log_s = np.log(np.maximum(j.signals[:n].astype(np.float64), j.floor[:n, None]))
                x = dti_design(j.gtab) if j.kind == "dti" else dki_design(j.gtab)
                g = None if j.kind == "dti" else dki_constraints(j.gtab)
                calls.append((n, lambda x=x, g=g, s=log_s: o.fit_log_signal(x, g, s, True, n_threads=threads)))
            else:
                b, g = j.gtab.bvals, j.gtab.bvecs
                w = compute_shell_weights(b, 1.0)
                hr = Kernel(j.responses, b, g, dirs=DIRS_300, weights=w)
                lr = Kernel(j.responses, b, g, dirs=low_resolution_dirs(j.responses, len(b)), weights=w)
                lrd = dict(k_aniso=lr.k_aniso, k_iso=lr.k_iso, w_k_iso=lr.w_k_iso, w_k_aniso=lr.w_k_aniso)
                hrd = dict(k_aniso=hr.k_aniso, k_iso=hr.k_iso, w_k_iso=hr.w_k_iso, w_k_aniso=hr.w_k_aniso,
                           blocks=[(bb.start, bb.stop) for bb in hr.aniso_blocks])
                sig = np.ascontiguousarray(j.signals[:n])
                calls.append((n, lambda s=sig, lw=lr.weights, a=lrd, h=hrd: o.fit_multi_tissue(
                    s, lw, a, h, n_threads=threads)))
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < budget_s:
            for n, call in calls:
                call()
                done += n
        return done, time.perf_counter() - t0, (f"the first 128 voxels of each of the {len(self.jobs)} volumes "
                                                f"(fits only), repeated for ~{budget_s:.0f} s")


class CsdWorkload(_SdWorkloadBase):
    """Single-shell CSD (CSDModel's solve, src/larmor/sd/csd.py) of the config-3 volume's highest
    shell: b = 3000, 90 directions, 500,040 voxels, lmax 8 (45 coefficients), 300 constraint
    directions, the default solver (up to 50 constrained solves per voxel), with the synthetic
    white matter response of the volume's fibres. The signals are the shell's samples clamped at
    0, as the model passes them."""

    name = "csd_lmax8_b3000_110x110x70"
    kernels = ("csd_kernel",)
    has_fp32 = False

    def __init__(self, seed: int) -> None:
        from larmor_b200.sd.csd_solver import CSDSolver, csd_problem, csd_shell
        from larmor_b200.synthetic import mfod_responses

        self._volume(seed)
        bval = csd_shell(self.gtab)
        on_shell = self.gtab.shell_index == int(np.argmin(np.abs(self.gtab.shells - bval)))
        self.problem = csd_problem(self.gtab.bvecs[on_shell], mfod_responses()[0].shell_coefficients(bval), 8,
                                   CSDSolver())
        self.shell = np.ascontiguousarray(np.maximum(self.signals[:, on_shell], 0.0))
        self.config = {"workload": self.name, "grid": [110, 110, 70], "voxels": self.v, "shell": bval,
                       "measurements": int(on_shell.sum()), "coefficients": 45, "constraints": 300,
                       "max_iter": 50, "l2": "flushed (256 MiB write) before each step"}

    def subset(self, n: int) -> None:
        super().subset(n)
        self.shell = self.shell[:n]

    def device_setup(self, torch, dev):
        from larmor_b200 import _core

        self.torch = torch
        p = self.problem
        self.handle = _core.CsdProblem.cached(p.initial, p.forward, p.constraint, p.norm_weight, p.threshold,
                                              p.max_iter)
        self.d_shell = torch.from_numpy(self.shell).to(dev)
        self.h_shell = torch.from_numpy(self.shell).pin_memory()
        self.h_fods = torch.empty((self.v, 45), dtype=torch.float64).pin_memory()
        self.h_conv = torch.empty((self.v,), dtype=torch.uint8).pin_memory()
        self.h2d_bytes = self.shell.nbytes
        self.d2h_bytes = self.v * (45 * 8 + 1)

    def step_device(self, precision=0):
        from larmor_b200 import _core

        self.d_fods, self.d_conv = _core.fit_csd_device(self.handle, self.d_shell)

    def kernel_bytes(self) -> dict:
        """Algorithmic DRAM bytes of one step: 90 signals in, 45 coefficients and a flag out."""
        return {"csd_kernel": self.v * (8 * self.shell.shape[1] + 8 * 45 + 1)}

    def step_e2e(self):
        self.d_shell.copy_(self.h_shell, non_blocking=True)
        self.step_device()
        self.h_fods.copy_(self.d_fods, non_blocking=True)
        self.h_conv.copy_(self.d_conv, non_blocking=True)

    def cpu_sample(self, threads: int, budget_s: float) -> tuple[int, float, str]:
        from oracle import oracle as o

        p = self.problem
        n = min(self.v, 4096)
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < budget_s:
            o.fit_csd(self.shell[:n], p.initial, p.forward, p.constraint, p.norm_weight, p.threshold, p.max_iter,
                      n_threads=threads)
            done += n
        return done, time.perf_counter() - t0, f"first {n} voxels of the shell, repeated for ~{budget_s:.0f} s"


class DrlWorkload(_SdWorkloadBase):
    """Damped Richardson-Lucy (the DRL solver, src/larmor/sd/solvers.py:72-148) single-tissue fit
    of the config-3 volume: 500,040 voxels, their 280 S0-normalised signals, the white matter
    kernel on the 300 FOD directions (the mFOD workload's fibre response), nu calibrated on it,
    up to 200 iterations per voxel."""

    name = "drl_single_tissue_110x110x70"
    kernels = ("drl_kernel", "drl_tc_kernel")
    has_fp32 = False

    def __init__(self, seed: int) -> None:
        from larmor_b200.sd.kernel import Kernel
        from larmor_b200.sd.rf import AnisotropicRF
        from larmor_b200.sd.sphere import DIRS_300

        self._volume(seed)
        self.norm = np.ascontiguousarray(np.minimum(self.signals / self.s0[:, None], 1.0))
        self.kernel = Kernel([AnisotropicRF([1.7e-3, 0.2e-3, 0.2e-3], 0.0)], self.gtab.bvals, self.gtab.bvecs,
                             dirs=DIRS_300)
        self.config = {"workload": self.name, "grid": [110, 110, 70], "voxels": self.v, "measurements": 280,
                       "directions": 300, "max_iter": 200, "l2": "inputs (1.1 GB) larger than L2",
                       "precision": DRL_PRECISION}

    def device_setup(self, torch, dev):
        from larmor_b200.sd.solvers import DRL, Stage

        self.torch = torch
        self.solver = DRL(precision=DRL_PRECISION)._prepare(self.kernel, self.gtab.bvals, Stage.SINGLE)
        self.d_signals = torch.from_numpy(self.norm).to(dev)
        self.h_signals = torch.from_numpy(self.norm).pin_memory()
        self.h_fods = torch.empty((self.v, 300), dtype=torch.float64).pin_memory()
        self.h2d_bytes = self.norm.nbytes
        self.d2h_bytes = self.v * 300 * 8

    def step_device(self, precision=0):
        from larmor_b200 import _core

        self.d_fods = _core._fit_single_tissue_on_device(self.d_signals, self.solver)

    def kernel_bytes(self) -> dict:
        """Algorithmic DRAM bytes of one step: 280 signals in, 300 amplitudes out per voxel."""
        return {"drl_kernel": self.v * 8 * (280 + 300), "drl_tc_kernel": self.v * 8 * (280 + 300)}

    flops_basis = "2 c^2 FLOP per voxel-iteration (the prediction F K^T K), 200 iterations per voxel (the cap)"

    def kernel_flops(self) -> dict:
        """FLOP of the product of one step at the iteration cap: 2 x 300^2 per voxel-iteration."""
        return {"drl_kernel": self.v * 200 * 2 * 300 ** 2, "drl_tc_kernel": self.v * 200 * 2 * 300 ** 2}

    def kernel_tensor_flops(self) -> dict:
        """The tensor FLOP the tensor-core mode issues at the iteration cap: three TF32 products
        over three 128-direction tiles (384) and 304 padded directions per voxel-iteration."""
        return {"drl_tc_kernel": self.v * 200 * 3 * 2 * 384 * 304}

    def step_e2e(self):
        self.d_signals.copy_(self.h_signals, non_blocking=True)
        self.step_device()
        self.h_fods.copy_(self.d_fods, non_blocking=True)

    def cpu_sample(self, threads: int, budget_s: float) -> tuple[int, float, str]:
        from larmor_b200.sd.solvers import _rl_products, calibrate_drl_nu
        from oracle import oracle as o

        k_t, k_t_k = _rl_products(self.kernel.w_k_aniso)
        nu = getattr(self, "_nu", None)
        if nu is None:
            nu = self._nu = calibrate_drl_nu(self.kernel, self.gtab.bvals) if hasattr(self, "solver") else 1e-3
        n = min(self.v, 512)
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < budget_s:
            self.reference_out = o.drl(self.norm[:n], k_t, k_t_k, nu, 200, 1.0 / 300, n_threads=threads)
            done += n
        return done, time.perf_counter() - t0, f"first {n} voxels of the volume, repeated for ~{budget_s:.0f} s"

    def parity(self) -> dict:
        """The device FODs of the cpu_baseline sample against the FP64 oracle's."""
        if not hasattr(self, "solver"):
            return None
        self.step_device()
        ref = self.reference_out
        got = self.d_fods[:len(ref)].cpu().numpy()
        ok = ~np.isnan(ref).any(axis=1)
        rel = np.abs(got[ok] - ref[ok]).max(axis=1) / np.abs(ref[ok]).max(axis=1)
        tol = 1e-4 if DRL_PRECISION != "fp64" else 1e-9
        return {"against": "FP64 oracle (restatement of cpp/src/sd/drl.cpp)", "voxels": int(ok.sum()),
                "precision": DRL_PRECISION, "fod_rel_max": float(rel.max()), "fod_rel_median": float(np.median(rel)),
                "tolerance": {"fod_rel": tol}, "within_tolerance": bool(rel.max() <= tol)}


class GrlWorkload(MfodWorkload):
    """Three-tissue GRL (SDModel, method GRL: the DRL solver at both resolutions,
    src/larmor/sd/method.py) of the config-3 volume: WM + GM + CSF, inner shells weighted 0.2,
    up to 50 rounds of a low-resolution dRL FOD (44 directions, 199 iterations from 1e-6) and
    the fractions until none moves by 1e-3, then the 300-direction FOD (599 iterations) and the
    final fractions, on S0-normalised signals."""

    name = "grl_3tissue_110x110x70"
    kernels = ("drl_kernel_resident", "drl_kernel", "drl_tc_kernel", "lr_fractions_kernel", "hr_fractions_kernel")
    fraction_tol = 1e-3
    has_fp32 = False

    def __init__(self, seed: int) -> None:
        from larmor_b200.synthetic import mfod_model_responses

        from larmor_b200.sd.kernel import Kernel
        from larmor_b200.sd.model import compute_shell_weights, low_resolution_dirs
        from larmor_b200.sd.sphere import DIRS_300

        self._volume(seed)
        self.norm = np.ascontiguousarray(np.minimum(self.signals / self.s0[:, None], 1.0))
        rfs = mfod_model_responses()
        weights = compute_shell_weights(self.gtab.bvals, 0.2)
        b, g = self.gtab.bvals, self.gtab.bvecs
        self.hr = Kernel(rfs, b, g, dirs=DIRS_300, weights=weights)
        self.lr = Kernel(rfs, b, g, dirs=low_resolution_dirs(rfs, len(b)), weights=weights)
        self.config = {"workload": self.name, "grid": [110, 110, 70], "voxels": self.v, "measurements": 280,
                       "tissues": "WM (300 directions) + GM + CSF", "solver": "DRL (200 / 600 iterations)",
                       "max_rounds": 50, "fraction_tol": self.fraction_tol, "l2": "inputs (1.1 GB) larger than L2",
                       "precision": DRL_PRECISION + (" (the 300-direction final solve; the 44-direction rounds FP64)"
                                                     if DRL_PRECISION != "fp64" else "")}

    def sd_solver(self):
        from larmor_b200.sd.solvers import DRL

        return DRL(precision=DRL_PRECISION)

    def step_device(self, precision=0):
        from larmor_b200 import _core

        _core.fit_multi_tissue_device(self.d_signals, self.lr.weights, self.k_lr, self.lr_solver, self.k_hr,
                                      self.hr_solver, 50, self.fraction_tol, 1e-2, self.d_fods, self.d_fr)

    def kernel_bytes(self) -> dict:
        """Algorithmic DRAM bytes of one step, per kernel. A voxel-round of the low-resolution
        loop reads the 280 signals and writes 44 amplitudes, whose fractions read those and the
        signals and write 3 fractions; the high-resolution pass does the same with 300
        directions once per voxel. dRL's iterations stay on the chip: K^T K comes from shared
        memory (resident at 44 directions) or L2 (staged at 300)."""
        from larmor_b200 import _core

        rounds = self.torch.zeros((self.v,), dtype=self.torch.int32, device=self.d_signals.device)
        _core.fit_multi_tissue_device(self.d_signals, self.lr.weights, self.k_lr, self.lr_solver, self.k_hr,
                                      self.hr_solver, 50, self.fraction_tol, 1e-2, self.d_fods, self.d_fr,
                                      rounds=rounds)
        vr = self._voxel_rounds = int(rounds.sum().item())
        m, c_lr, c_hr = 280, self.k_lr.ca, self.k_hr.ca
        return {"drl_kernel_resident": vr * 8 * (m + c_lr), "drl_kernel": self.v * 8 * (m + c_hr),
                "drl_tc_kernel": self.v * 8 * (m + c_hr),
                "lr_fractions_kernel": vr * 8 * (c_lr + m + 3),
                "hr_fractions_kernel": self.v * 8 * (c_hr + m + 3)}

    flops_basis = ("2 c^2 FLOP per voxel-iteration (the prediction F K^T K) at the iteration caps: 599 per "
                   "voxel at 300 directions, 199 per voxel-round at 44")

    def kernel_flops(self) -> dict:
        """FP64 FLOP of one step at the iteration caps (the voxel-rounds from kernel_bytes)."""
        return {"drl_kernel": self.v * 599 * 2 * self.k_hr.ca ** 2, "drl_tc_kernel": self.v * 599 * 2 * self.k_hr.ca ** 2,
                "drl_kernel_resident": self._voxel_rounds * 199 * 2 * self.k_lr.ca ** 2}

    def kernel_tensor_flops(self) -> dict:
        """The tensor FLOP of the tensor-core final solve at its iteration cap (599): three TF32
        products over the padded 384 x 304 tiles per voxel-iteration."""
        return {"drl_tc_kernel": self.v * 599 * 3 * 2 * 384 * 304}

    def parity(self) -> dict:
        """The device fit of the cpu_baseline sample's voxels against the FP64 oracle's GRL."""
        ref, ref_fr = self.reference_out
        n = len(ref)
        got = self.d_fods[:n].cpu().numpy()
        got_fr = self.d_fr[:n].cpu().numpy()
        rel = np.abs(got - ref).max(axis=1) / np.abs(ref).max(axis=1)
        tol = 1e-4 if DRL_PRECISION != "fp64" else 1e-9
        fr_err = float(np.abs(got_fr - ref_fr).max())
        return {"against": "FP64 oracle (restatement of cpp/src/sd/{drl,multi_tissue,fractions}.cpp)", "voxels": n,
                "precision": DRL_PRECISION, "fod_rel_max": float(rel.max()), "fractions_abs_max": fr_err,
                "tolerance": {"fod_rel": tol, "fractions_abs": 1e-4},
                "within_tolerance": bool(rel.max() <= tol and fr_err <= 1e-4)}

    def cpu_sample(self, threads: int, budget_s: float) -> tuple[int, float, str]:
        from larmor_b200.sd.solvers import _rl_products
        from oracle import oracle as o

        if not hasattr(self, "_nus"):
            # nu of each kernel as calibrate_drl_nu sets it, by the oracle's dRL.
            b = self.gtab.bvals
            signal = np.full((1, len(b)), np.exp(-max(b) * 0.7e-3))
            self._nus = tuple(0.2 * float(np.max(o.drl(signal, *_rl_products(k.k), 0.0, 200, 1.0 / k.k.shape[1])))
                              for k in (self.lr, self.hr))
        n = min(self.v, 4 * threads)
        lr = dict(k_aniso=self.lr.k_aniso, k_iso=self.lr.k_iso, w_k_iso=self.lr.w_k_iso, w_k_aniso=self.lr.w_k_aniso)
        hr = dict(k_aniso=self.hr.k_aniso, k_iso=self.hr.k_iso, w_k_iso=self.hr.w_k_iso, w_k_aniso=self.hr.w_k_aniso,
                  blocks=[(b.start, b.stop) for b in self.hr.aniso_blocks])
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < budget_s:
            self.reference_out = o.fit_multi_tissue(
                self.norm[:n], self.lr.weights, lr, hr, max_rounds=50, fraction_tol=self.fraction_tol, final_tol=1e-2,
                n_threads=threads, lr_drl={"nu": self._nus[0], "n_iter": 199, "init": 1e-6},
                hr_drl={"nu": self._nus[1], "n_iter": 599, "init": 1e-6})
            done += n
        return done, time.perf_counter() - t0, f"first {n} voxels of the volume, repeated for ~{budget_s:.0f} s"


class PeaksWorkload:
    """FOD peaks (find_peaks, src/larmor/sd/peaks.py) of lmax-8 FODs on the config-3 mask
    (110x110x70, 500,040 voxels): the amplitudes of each FOD on the 642-vertex icosphere, then
    the climbs from their local maxima, merged into at most 3 peaks above 0.1 of the largest.
    The FODs are seeded synthetic SH series of 1-3 fibres (Dirichlet(2) fractions, random
    directions, the lmax-8 fibre profile exp(-0.02 l(l+1))) plus N(0, 0.02) noise on every
    coefficient."""

    name = "peaks_lmax8_110x110x70"
    kernels = ("project_sh_kernel", "peak_count_kernel", "scan_blocks_kernel", "scan_sums_kernel", "peak_fill_kernel",
               "climb_pool_kernel", "peak_merge_kernel")
    has_fp32 = False
    unit = "voxel peak searches/s"

    def __init__(self, seed: int) -> None:
        from larmor_b200.sd.sh import build_basis_matrix, get_sh_indices
        from larmor_b200.sd.sphere import get_theta_phi
        from larmor_b200.synthetic import ellipsoid_mask

        mask = ellipsoid_mask((110, 110, 70), 1.0435)
        self.v = int(mask.sum())
        rng = np.random.default_rng(7 + 10 * (seed - 1))
        ls, _ = get_sh_indices(8)
        profile = np.exp(-0.02 * ls * (ls + 1))
        n_fib = rng.integers(1, 4, size=self.v)
        fr = rng.dirichlet([2.0, 2.0, 2.0], size=self.v) * (np.arange(3)[None] < n_fib[:, None])
        fr /= fr.sum(axis=1, keepdims=True)
        coeffs = 0.02 * rng.normal(size=(self.v, 45))
        for f in range(3):
            d = rng.normal(size=(self.v, 3))
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            theta, phi = get_theta_phi(d)
            coeffs += fr[:, f:f + 1] * build_basis_matrix(theta, phi, 8) * profile
        self.coeffs = np.ascontiguousarray(coeffs)
        self.config = {"workload": self.name, "grid": [110, 110, 70], "voxels": self.v, "lmax": 8,
                       "sphere": "642-vertex icosphere", "num_peaks": 3, "relative_threshold": 0.1,
                       "l2": "amplitudes (2.6 GB) larger than L2"}

    def subset(self, n: int) -> None:
        self.coeffs = self.coeffs[:n]
        self.v = len(self.coeffs)
        self.config["voxels"] = self.v

    def device_setup(self, torch, dev):
        from larmor_b200 import _core
        from larmor_b200.sd.peaks import _amplitude_projector, _build_icosphere

        self.torch = torch
        vertices, neighbours = _build_icosphere()
        self.sphere = _core.PeakSphere.cached(vertices, neighbours)
        self.projector = _amplitude_projector(8, False)
        self.d_coeffs = torch.from_numpy(self.coeffs).to(dev)
        self.h_coeffs = torch.from_numpy(self.coeffs).pin_memory()
        self.h_dirs = torch.empty((self.v, 3, 3), dtype=torch.float64).pin_memory()
        self.h_amps = torch.empty((self.v, 3), dtype=torch.float64).pin_memory()
        self.h2d_bytes = self.coeffs.nbytes
        self.d2h_bytes = self.v * 12 * 8

    def step_device(self, precision=0):
        from larmor_b200 import _core

        on_sphere = _core.project_sh_device(self.projector, self.d_coeffs, exact_integral=False)
        self.d_dirs, self.d_amps = _core.find_peaks_device(self.sphere, self.d_coeffs, 8, False, on_sphere, 3, 0.1,
                                                           0.0)

    def climbs(self) -> int:
        """The climbs of one step: the local maxima with a positive amplitude of every voxel's
        amplitudes on the icosphere (counted with torch, in chunks)."""
        from larmor_b200 import _core
        from larmor_b200.sd.peaks import _build_icosphere

        torch = self.torch
        _, neighbours = _build_icosphere()
        nb = torch.from_numpy(neighbours).to(self.d_coeffs.device)
        total = 0
        for start in range(0, self.v, 16384):
            amp = _core.project_sh_device(self.projector, self.d_coeffs[start:start + 16384], exact_integral=False)
            is_max = (amp > 0) & (amp[:, nb] <= amp[:, :, None]).all(dim=2)
            total += int(is_max.sum().item())
        return total

    def kernel_bytes(self) -> dict:
        """Algorithmic DRAM bytes of one step: the projection reads 45 coefficients and writes
        642 amplitudes; the count and the fill read the amplitudes (the fill writes an 8-byte
        start per climb); the pool reads a start and writes a 32-byte result per climb, and reads
        each voxel's 45 coefficients (shared by its climbs);
        the merge reads the results and writes 12 outputs."""
        c = self.climbs()
        return {"project_sh_kernel": self.v * 8 * (45 + 642), "peak_count_kernel": self.v * (8 * 642 + 4),
                "scan_blocks_kernel": self.v * 12, "scan_sums_kernel": 0,
                "peak_fill_kernel": self.v * 8 * 642 + 8 * c,
                "climb_pool_kernel": self.v * 8 * 45 + c * (8 + 32), "peak_merge_kernel": c * 32 + self.v * (12 * 8 + 12)}

    def step_e2e(self):
        self.d_coeffs.copy_(self.h_coeffs, non_blocking=True)
        self.step_device()
        self.h_dirs.copy_(self.d_dirs, non_blocking=True)
        self.h_amps.copy_(self.d_amps, non_blocking=True)

    def cpu_sample(self, threads: int, budget_s: float) -> tuple[int, float, str]:
        from larmor_b200.sd.peaks import _build_icosphere, _get_amplitudes
        from oracle import oracle as o

        vertices, neighbours = _build_icosphere()
        n = min(self.v, 8192)
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < budget_s:
            on = np.ascontiguousarray(_get_amplitudes(self.coeffs[:n], 8, False))
            o.peaks_chunk(self.coeffs[:n], 8, on, vertices, neighbours, 3, 0.1, 0.0, n_threads=threads)
            done += n
        return done, time.perf_counter() - t0, (f"first {n} voxels (numpy amplitudes + the oracle's search), "
                                                f"repeated for ~{budget_s:.0f} s")


WORKLOADS = {"dti": DtiWorkload, "dki": DkiWorkload, "mfod": MfodWorkload, "msmt": MsmtWorkload,
             "batch": BatchWorkload, "peaks": PeaksWorkload, "dti_model": DtiModelWorkload, "csd": CsdWorkload,
             "drl": DrlWorkload, "grl": GrlWorkload}



# ---- runs --------------------------------------------------------------------------------

def _serve_jobs(seed: int, count: int, wl=None):
    """Fit requests drawn from the config-3 distribution: contiguous runs of voxels of the
    110x110x70 three-tissue volume (S0-normalised), their lengths log-uniform in [4096, 65536]."""
    from larmor_b200.batch import MfodJob
    from larmor_b200.synthetic import mfod_model_responses

    wl = MfodWorkload(seed=1) if wl is None else wl
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(count):
        n = int(round(np.exp(rng.uniform(np.log(4096), np.log(65536)))))
        start = int(rng.integers(0, wl.v - n))
        jobs.append(MfodJob(wl.gtab, np.ascontiguousarray(wl.norm[start:start + n]), mfod_model_responses()))
    return jobs


def run_serving(args, source=None) -> dict:
    """Config 5: Poisson arrivals of mFOD fit requests at rates swept up to saturation through
    the continuous-batching server, against the plain per-request fit (one request at a time).
    Latency is arrival to result on the host (wall clock), the quantity a client sees."""
    import torch

    from larmor_b200 import _core
    from larmor_b200.serve import FitServer

    jobs = _serve_jobs(5, args.serve_requests, source)
    voxels = sum(j.voxels for j in jobs)
    # Warm-up: the largest request on every slot at once, so that each slot's handles and
    # scratch are built and sized before the timed arrivals (growing scratch later would free
    # and allocate device memory, which waits for the whole GPU).
    server = FitServer(budget_bytes=80 << 30, slots=args.serve_slots)
    largest = max(jobs, key=lambda j: j.voxels)
    for f in [server.submit(largest) for _ in range(args.serve_slots)]:
        f.result()
    # Plain per-request fits: one request at a time, back to back.
    t0 = time.perf_counter()
    for j in jobs:
        server.submit(j).result()
    plain_s = time.perf_counter() - t0
    plain_rate = len(jobs) / plain_s
    rng = np.random.default_rng(55)
    sweep = {}
    _core.kernel_timing(True)
    launches0 = _core.launch_count()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        for factor in args.serve_load:
            lam = factor * plain_rate
            gaps = rng.exponential(1.0 / lam, len(jobs))
            first = len(server.completed)
            t_start = time.perf_counter()
            futures = []
            for j, gap in zip(jobs, gaps):
                time.sleep(gap)
                futures.append(server.submit(j))
            for f in futures:
                f.result()
            t_end = time.perf_counter()
            lat = sorted(1e3 * (r.finished - r.arrival) for r in server.completed[first:])
            sweep[f"{factor:g}x"] = {"arrival_rate_per_s": lam, "p50_ms": float(np.percentile(lat, 50)),
                                     "p99_ms": float(np.percentile(lat, 99)),
                                     "throughput_voxels_per_s": voxels / (t_end - t_start)}
    launches = _core.launch_count() - launches0
    kernel_ms = {k: _core.kernel_time(k) for k in MfodWorkload.kernels}
    _core.kernel_timing(False)
    peak_running = server.peak_running
    server.close()
    top_load = f"{args.serve_load[-1]:g}x"
    best = max(v["throughput_voxels_per_s"] for v in sweep.values())
    top = max(kernel_ms, key=lambda k: kernel_ms[k][0])
    return {
        "metric": METRIC, "value": best, "unit": "voxel fits/s", "n_gpus": 1, "steps": len(args.serve_load),
        "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "serve_mfod_poisson", "requests_per_rate": len(jobs), "voxels_per_rate": voxels,
                   "request_voxels": "log-uniform 4096-65536 (config-3 volume)", "slots": args.serve_slots,
                   "hbm_budget_gb": 80, "rates": "multiples of the plain per-request rate",
                   "timing": "host wall clock, arrival to result"},
        "serving": sweep,
        "plain_per_request": {"value": voxels / plain_s, "unit": "voxel fits/s", "requests_per_s": plain_rate},
        "saturation": {"load": top_load, "peak_concurrent_requests": peak_running},
        "e2e": {"value": best, "unit": "voxel fits/s", "h2d_bytes_per_step": sum(j.signals.nbytes for j in jobs),
                "d2h_bytes_per_step": sum(j.voxels * 8 * 308 for j in jobs)},
        "roofline": None, "dominant_kernel": top,
        "kernel_share": {k: round(t / max(sum(x for x, _ in kernel_ms.values()), 1e-30), 4)
                         for k, (t, _) in kernel_ms.items()},
        "cpu_baseline": None, "gpu_launches": launches, "clocks": clocks.summary(),
    }


def run_reference(args, wl) -> dict:
    threads = os.cpu_count() or 1
    per_step = []
    sample = ""
    for i in range(args.warmup + args.steps):
        done, secs, sample = wl.cpu_sample(threads, args.reference_budget)
        if i >= args.warmup:
            per_step.append((done, secs))
    voxels = sum(d for d, _ in per_step)
    secs = sum(s for _, s in per_step)
    value = voxels / secs
    return {
        "metric": METRIC, "value": value, "unit": getattr(wl, "unit", "voxel fits/s"), "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * secs / len(per_step), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": wl.config,
        "cpu_baseline": {"value": value, "unit": getattr(wl, "unit", "voxel fits/s"), "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": getattr(wl, "unit", "voxel fits/s"), "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def measure(wl, args, world: int, rank: int, dist, dev) -> dict:
    """The bench line of one workload: K device-resident steps (value), the plain FP32 variant
    where the workload has one, K end-to-end steps through the public call (e2e), the dominant
    kernel's roofline, and on rank 0 the FP64 oracle on a bounded sample of the same workload
    (cpu_baseline) with the device results' error against it (parity). Every rank takes the
    same collective steps."""
    import torch

    from larmor_b200 import _core

    flush = torch.empty(256 * 2**20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(step, k):
        """Total event time (ms) of k steps, each preceded by an L2 flush outside the events."""
        total = 0.0
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        for i in range(k):
            flush.fill_(i & 0xFF)
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        for a, b in ev:
            total += a.elapsed_time(b)
        return total

    def max_over_ranks(x: float) -> float:
        from larmor_b200.sharding import max_over_ranks as slowest

        return slowest(x, device=dev)

    # Warm-up, then the timed device-resident steps.
    for _ in range(args.warmup):
        wl.step_device()
    barrier()
    gpu_index = dev.index if dev.index is not None else 0
    visible = os.environ.get("CUDA_VISIBLE_DEVICES")
    smi_index = int(visible.split(",")[gpu_index]) if visible and visible.split(",")[gpu_index].isdigit() else gpu_index

    _core.kernel_timing(True)
    launches0 = _core.launch_count()
    with ClockSampler(smi_index) as clocks:
        dev_ms = timed(wl.step_device, args.steps)
    barrier()
    launches = _core.launch_count() - launches0
    kernel_ms = {name: _core.kernel_time(name) for name in wl.kernels}
    _core.kernel_timing(False)
    if hasattr(wl, "graph_launches"):
        # Graph replays launch the library's kernels without a host call: count the recorded
        # kernels, and time each kernel in the same work launched eagerly.
        launches = wl.graph_launches() * args.steps
        _core.kernel_timing(True)
        for _ in range(args.steps):
            wl.step_eager()
        torch.cuda.synchronize()
        kernel_ms = {name: _core.kernel_time(name) for name in wl.kernels}
        _core.kernel_timing(False)
    dev_ms = max_over_ranks(dev_ms)

    # The plain FP32 kernel, for comparison.
    fp32_ms = None
    fp32_steps = max(1, min(args.steps, getattr(wl, "fp32_steps", args.steps)))
    if wl.has_fp32:
        for _ in range(min(args.warmup, fp32_steps)):
            wl.step_device(precision=1)
        barrier()
        fp32_ms = max_over_ranks(timed(lambda: wl.step_device(precision=1), fp32_steps))

    # End to end through host buffers.
    e2e_steps = max(1, min(args.steps, getattr(wl, "e2e_steps", args.steps)))
    for _ in range(min(args.warmup, 3)):
        wl.step_e2e()
    barrier()
    e2e_ms = max_over_ranks(timed(wl.step_e2e, e2e_steps))

    voxels_all = wl.v * world
    value = voxels_all * args.steps / (dev_ms / 1e3)
    pk, pk_kind = peaks()
    # The dominant kernel: the most device time in the timed region (CUDA events on its stream).
    step_bytes = wl.kernel_bytes()
    top = max(kernel_ms, key=lambda k: kernel_ms[k][0])
    top_ms, top_launches = kernel_ms[top]
    avg_launch_s = top_ms / max(top_launches, 1) / 1e3
    bytes_per_launch = step_bytes[top] * args.steps / max(top_launches, 1)
    achieved_gbs = bytes_per_launch / avg_launch_s / 1e9 if avg_launch_s > 0 else 0.0
    traffic = committed_traffic(top, wl.name, bytes_per_launch)
    total_kernel_ms = max(sum(t for t, _ in kernel_ms.values()), 1e-30)

    cpu, parity, fp32_parity = None, None, None
    if rank == 0:
        threads = os.cpu_count() or 1
        done, secs, sample = wl.cpu_sample(threads, args.cpu_budget)
        cpu = {"value": done / secs, "unit": getattr(wl, "unit", "voxel fits/s"), "cores": threads, "kind": "port",
               "sample": sample}
        if hasattr(wl, "parity"):
            parity = wl.parity()
        if fp32_ms is not None and hasattr(wl, "fp32_parity"):
            fp32_parity = wl.fp32_parity()

    line = {
        "metric": METRIC, "value": value, "unit": getattr(wl, "unit", "voxel fits/s"), "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": wl.config,
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved_gbs / pk["hbm_gbs"], "traffic": traffic,
                     "kernel": top, "peak_source": pk_kind,
                     "algorithmic_bytes_per_launch": bytes_per_launch,
                     "avg_launch_ms": avg_launch_s * 1e3, "launches": top_launches,
                     "kernel_share": {k: round(t / total_kernel_ms, 4) for k, (t, _) in kernel_ms.items()}},
        "cpu_baseline": cpu,
        "e2e": {"value": voxels_all * e2e_steps / (e2e_ms / 1e3), "unit": getattr(wl, "unit", "voxel fits/s"),
                "h2d_bytes_per_step": wl.h2d_bytes, "d2h_bytes_per_step": wl.d2h_bytes, "steps": e2e_steps},
        "plain_fp32": None if fp32_ms is None else {
            "value": voxels_all * fp32_steps / (fp32_ms / 1e3), "unit": "voxel fits/s",
            "ms_per_step": fp32_ms / fp32_steps, "steps": fp32_steps, "parity": fp32_parity,
            "what": getattr(wl, "fp32_what", "the same kernels in FP32 (precision=LAR_FP32)")},
        "parity": parity,
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    if hasattr(wl, "kernel_flops"):
        # Tensor-core kernels: FP64 ones against the nominal FP64 tensor rate, the TF32 one
        # against the TF32 rate; the HBM bytes stay beside it.
        flops = wl.kernel_flops().get(top)
        if flops is not None and top == "drl_tc_kernel":
            hw = wl.kernel_tensor_flops()[top] * args.steps / max(top_launches, 1)
            line["roofline"].update(tf32_tensor_roofline(hw, flops * args.steps / max(top_launches, 1), avg_launch_s, pk))
            line["roofline"]["flops_basis"] = wl.flops_basis + "; tensor FLOP: 3 x 2 x 384 x 304 per voxel-iteration"
        elif flops is not None:
            line["roofline"].update(fp64_tensor_roofline(flops * args.steps / max(top_launches, 1), avg_launch_s))
            line["roofline"]["flops_basis"] = wl.flops_basis
    issue = committed_issue(top, wl.name, bytes_per_launch)
    if issue is not None and avg_launch_s > 0:
        # The issue roofline of an instruction-bound kernel: warp instructions per second
        # against the SMs' issue slots (4 schedulers x 1 warp instruction per cycle each).
        sm_mhz = line["clocks"].get("sm_mhz") or line["clocks"].get("sm_max_mhz") or 1965.0
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        peak = sms * 4 * sm_mhz * 1e6
        achieved = issue["warp_instructions"] / avg_launch_s
        line["issue_roofline"] = {
            "kernel": top, "unit": "warp instructions/s", "achieved": achieved, "peak": peak, "frac": achieved / peak,
            "peak_basis": f"{sms} SMs x 4 schedulers x 1 warp instruction per cycle at the median SM clock {sm_mhz} MHz",
            "warp_instructions_per_launch": issue["warp_instructions"],
            "warp_instructions_per_voxel_round": issue["warp_instructions_per_voxel_round"],
            "threads_per_instruction": issue["threads_per_instruction"],
            "source": "profiles/issue.json (ncu smsp__inst_executed.sum per algorithmic byte, scaled to this launch)"}
    fp64 = committed_fp64(top, wl.name)
    if fp64 is not None and avg_launch_s > 0:
        # The FP64 roofline of a CUDA-core FP64 kernel: its FLOP (counted per voxel by ncu)
        # against the FP64 pipe's rate, 32 FP64 FMA per SM per cycle (the pipe's active
        # fraction in the capture matches this rate: 38.6% busy at 7.5 TFLOP/s).
        sm_mhz = line["clocks"].get("sm_mhz") or line["clocks"].get("sm_max_mhz") or 1965.0
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        peak = sms * 32 * 2 * sm_mhz * 1e6 / 1e12
        achieved = fp64["fp64_flop_per_voxel"] * (voxels_all / world) * args.steps / max(top_launches, 1) \
            / avg_launch_s / 1e12
        line["fp64_roofline"] = {
            "kernel": top, "unit": "TFLOP/s", "achieved": achieved, "peak": peak, "frac": achieved / peak,
            "peak_basis": f"{sms} SMs x 32 FP64 FMA x 2 per cycle at the median SM clock {sm_mhz} MHz",
            "fp64_flop_per_voxel": fp64["fp64_flop_per_voxel"],
            "source": "profiles/fp64.json (ncu FP64 instruction counts of the same kernel and volume)"}
    if hasattr(wl, "extra"):
        def timed_host(step):
            for _ in range(args.warmup):
                step()
            barrier()
            return max_over_ranks(timed(step, args.steps)) / args.steps

        line.update(wl.extra(timed_host))
    del flush
    return line


def main() -> int:
    global REFERENCE_ARM, DRL_PRECISION
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="mfod", choices=sorted(WORKLOADS) + ["serve"])
    ap.add_argument("--impl", default="larmor_b200", choices=["larmor_b200", "reference"])
    ap.add_argument("--reference-budget", type=float, default=3.0,
                    help="seconds of CPU work per reference step")
    ap.add_argument("--cpu-budget", type=float, default=10.0,
                    help="seconds of CPU baseline work on rank 0")
    ap.add_argument("--voxels", type=int, default=0,
                    help="fit only the first N voxels of the volume (small cases for ncu)")
    ap.add_argument("--serve-requests", type=int, default=24, help="requests per arrival rate (serve)")
    ap.add_argument("--serve-slots", type=int, default=6, help="requests on the GPU at once (serve)")
    ap.add_argument("--serve-load", type=float, nargs="+", default=[0.5, 1.0, 2.0, 4.0],
                    help="arrival rates as multiples of the plain per-request rate (serve)")
    ap.add_argument("--drl-precision", default="fp64", choices=["fp64", "tf32x3"],
                    help="dRL arithmetic of the drl and grl workloads")
    ap.add_argument("--no-extras", action="store_true",
                    help="the mfod line without its DTI and serving sub-objects")
    ap.add_argument("--profile", action="store_true",
                    help="warm-up and K device-resident steps only, timed per step on stdout (for ncu); "
                         "prints no bench line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    DRL_PRECISION = args.drl_precision

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        REFERENCE_ARM = True
        if rank != 0:
            return 0
        if args.workload == "serve":
            wl = MfodWorkload(seed=1)
            line = run_reference(args, wl)
            line["config"] = {"workload": "serve_mfod_poisson", "reference": "the mFOD fit of config-3 voxels"}
        else:
            wl = WORKLOADS[args.workload](seed=1)
            line = run_reference(args, wl)
        print(json.dumps(line))
        return 0

    if args.workload == "serve":
        if rank != 0:
            return 0
        print(json.dumps(run_serving(args)))
        return 0

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local if world > 1 else torch.cuda.current_device())
    torch.cuda.set_device(dev)

    wl = WORKLOADS[args.workload](seed=1 + rank)
    if args.voxels:
        wl.subset(args.voxels)
    wl.device_setup(torch, dev)
    if args.profile:
        from larmor_b200 import _core

        for i in range(args.warmup + args.steps):
            last = i == args.warmup + args.steps - 1
            _core.kernel_timing(last)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            wl.step_device()
            torch.cuda.synchronize()
            print(f"{wl.name} voxels {wl.v} step {i} {1e3 * (time.perf_counter() - t0):.3f} ms")
        times = {k: _core.kernel_time(k) for k in wl.kernels}
        _core.kernel_timing(False)
        print("kernels (ms, launches) of the last step:",
              ", ".join(f"{k} {t:.2f} ({n})" for k, (t, n) in times.items() if n))
        return 0

    line = measure(wl, args, world, rank, dist, dev)
    if args.workload == "mfod" and not args.no_extras and not args.voxels:
        # The metric names DTI and serving beside mFOD: config 1 measured the same way, and a
        # short serving sweep (rank 0 only; it has no collective) of requests cut from the same
        # volume.
        source = argparse.Namespace(v=wl.v, gtab=wl.gtab, norm=wl.norm)
        del wl
        dti = DtiWorkload(seed=1 + rank)
        dti.device_setup(torch, dev)
        sub = argparse.Namespace(**vars(args))
        sub.cpu_budget = min(args.cpu_budget, 5.0)
        line["dti"] = measure(dti, sub, world, rank, dist, dev)
        for key in ("metric", "n_gpus", "higher_is_better", "scaling", "vs_baseline", "data"):
            line["dti"].pop(key, None)
        del dti
        if rank == 0:
            srv = argparse.Namespace(**vars(args))
            srv.serve_requests, srv.serve_load = 16, [1.0, 2.0]
            serve = run_serving(srv, source)
            line["serve"] = {k: serve[k] for k in ("value", "unit", "config", "serving", "plain_per_request",
                                                   "saturation", "dominant_kernel", "gpu_launches", "clocks")}
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
