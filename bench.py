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


def committed_traffic(kernel: str, workload: str) -> float | None:
    """Per-launch DRAM bytes of a kernel from the committed ncu summary, if any."""
    path = ROOT / "profiles" / "traffic.json"
    if not path.exists():
        return None
    table = json.loads(path.read_text())
    entry = table.get(f"{workload}:{kernel}")
    return None if entry is None else float(entry["bytes_per_launch"])


# ---- clocks ------------------------------------------------------------------------------

class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons of one GPU while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int) -> None:
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[3:7]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---- workloads ---------------------------------------------------------------------------

class DtiWorkload:
    """Config 1: DTI WLLS on the 64x64x40 volume (79,912 voxels, 1 b0 + 30 directions)."""

    name = "dti_wlls_64x64x40"
    kernel = "fit_dti_maps_kernel"
    # Algorithmic bytes per voxel: 31 float32 samples in, 16 float32 maps + 1 byte out
    # (the 8-byte floor per voxel is host-prepared input too).
    bytes_per_voxel = 4 * 31 + 8 + 16 * 4 + 1

    def __init__(self, seed: int) -> None:
        from larmor_b200.dwi.dti import dti_design
        from larmor_b200.dwi.inputs import estimate_s0, masked_signals, sample_floors
        from larmor_b200.synthetic import dti_volume

        w = dti_volume(seed=seed)
        self.config = {"workload": self.name, "grid": [64, 64, 40], "voxels": w.n_voxels,
                       "measurements": 31, "fit": "wls", "l2": "flushed (256 MiB write) before each step"}
        self.design = dti_design(w.gtab)
        s0 = estimate_s0(w.volume, w.gtab, w.mask)[w.mask]
        self.signals = masked_signals(w.volume, np.nonzero(w.mask))
        self.floor = sample_floors(s0, None, len(self.signals))
        self.v = len(self.signals)

    def device_setup(self, torch, dev):
        from larmor_b200 import _core

        self.handle = _core.LogDesign.cached(self.design, np.zeros((0, 7)))
        self.d_signals = torch.from_numpy(self.signals).to(dev)
        self.d_floor = torch.from_numpy(self.floor).to(dev)
        self.d_maps = torch.empty((16, self.v), dtype=torch.float32, device=dev)
        self.d_npd = torch.empty((self.v,), dtype=torch.uint8, device=dev)
        self.h_signals = torch.from_numpy(self.signals).pin_memory()
        self.h_floor = torch.from_numpy(self.floor).pin_memory()
        self.h_maps = torch.empty((16, self.v), dtype=torch.float32).pin_memory()
        self.h_npd = torch.empty((self.v,), dtype=torch.uint8).pin_memory()
        self.h2d_bytes = self.signals.nbytes + self.floor.nbytes
        self.d2h_bytes = 16 * 4 * self.v + self.v

    def step_device(self, precision=0):
        from larmor_b200 import _core

        _core.fit_dti_maps_device(self.handle, self.d_signals, self.d_floor, True, self.d_maps,
                                  self.d_npd, precision=precision)

    def step_e2e(self):
        from larmor_b200 import _core

        self.d_signals.copy_(self.h_signals, non_blocking=True)
        self.d_floor.copy_(self.h_floor, non_blocking=True)
        _core.fit_dti_maps_device(self.handle, self.d_signals, self.d_floor, True, self.d_maps, self.d_npd)
        self.h_maps.copy_(self.d_maps, non_blocking=True)
        self.h_npd.copy_(self.d_npd, non_blocking=True)

    def cpu_sample(self, threads: int, budget_s: float) -> tuple[int, float, str]:
        from oracle import oracle as o

        log_s = np.log(np.where((self.signals > 0) & np.isfinite(self.signals), self.signals,
                                self.floor[:, None]).astype(np.float64))
        o.fit_log_signal(self.design, None, log_s[:256], True, n_threads=threads)  # warm-up
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < budget_s:
            o.fit_log_signal(self.design, None, log_s, True, n_threads=threads)
            done += len(log_s)
        return done, time.perf_counter() - t0, f"whole volume ({self.v} voxels) repeated for ~{budget_s:.0f} s"


WORKLOADS = {"dti": DtiWorkload}


# ---- runs --------------------------------------------------------------------------------

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
        "metric": METRIC, "value": value, "unit": "voxel fits/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * secs / len(per_step), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": wl.config,
        "cpu_baseline": {"value": value, "unit": "voxel fits/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "voxel fits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="dti", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="larmor_b200", choices=["larmor_b200", "reference"])
    ap.add_argument("--reference-budget", type=float, default=3.0,
                    help="seconds of CPU work per reference step")
    ap.add_argument("--cpu-budget", type=float, default=10.0,
                    help="seconds of CPU baseline work on rank 0")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        wl = WORKLOADS[args.workload](seed=1)
        print(json.dumps(run_reference(args, wl)))
        return 0

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local if world > 1 else torch.cuda.current_device())
    torch.cuda.set_device(dev)

    wl = WORKLOADS[args.workload](seed=1 + rank)
    wl.device_setup(torch, dev)
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
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # Warm-up, then the timed device-resident steps.
    for _ in range(args.warmup):
        wl.step_device()
    barrier()
    gpu_index = dev.index if dev.index is not None else 0
    visible = os.environ.get("CUDA_VISIBLE_DEVICES")
    smi_index = int(visible.split(",")[gpu_index]) if visible and visible.split(",")[gpu_index].isdigit() else gpu_index
    with ClockSampler(smi_index) as clocks:
        dev_ms = timed(wl.step_device, args.steps)
    barrier()
    dev_ms = max_over_ranks(dev_ms)

    # The plain FP32 kernel, for comparison.
    for _ in range(args.warmup):
        wl.step_device(precision=1)
    barrier()
    fp32_ms = max_over_ranks(timed(lambda: wl.step_device(precision=1), args.steps))

    # End to end through host buffers.
    for _ in range(args.warmup):
        wl.step_e2e()
    barrier()
    e2e_ms = max_over_ranks(timed(wl.step_e2e, args.steps))

    voxels_all = wl.v * world
    value = voxels_all * args.steps / (dev_ms / 1e3)
    avg_launch_s = dev_ms / args.steps / 1e3
    pk, pk_kind = peaks()
    achieved_gbs = wl.bytes_per_voxel * wl.v / avg_launch_s / 1e9
    traffic = committed_traffic(wl.kernel, wl.name)

    cpu = None
    if rank == 0:
        threads = os.cpu_count() or 1
        done, secs, sample = wl.cpu_sample(threads, args.cpu_budget)
        cpu = {"value": done / secs, "unit": "voxel fits/s", "cores": threads, "kind": "port",
               "sample": sample}

    line = {
        "metric": METRIC, "value": value, "unit": "voxel fits/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": wl.config,
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved_gbs / pk["hbm_gbs"], "traffic": traffic,
                     "kernel": wl.kernel, "peak_source": pk_kind,
                     "algorithmic_bytes_per_voxel": wl.bytes_per_voxel},
        "cpu_baseline": cpu,
        "e2e": {"value": voxels_all * args.steps / (e2e_ms / 1e3), "unit": "voxel fits/s",
                "h2d_bytes_per_step": wl.h2d_bytes, "d2h_bytes_per_step": wl.d2h_bytes},
        "plain_fp32": {"value": voxels_all * args.steps / (fp32_ms / 1e3), "unit": "voxel fits/s",
                       "ms_per_step": fp32_ms / args.steps},
        "gpu_launches": args.steps,
        "clocks": clocks.summary(),
    }
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
