"""Builds the CUDA library liblarmor_b200.so in-tree for sm_100a (B200).

    python -m larmor_b200.build

nvcc cross-compiles without a GPU. The library links the CUDA runtime statically, so it loads
next to any PyTorch build; its C ABI is declared in include/larmor_b200.h.
"""

from __future__ import annotations

import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
LIB = PACKAGE / "liblarmor_b200.so"
SOURCES = ["capi.cu", "log_fit.cu", "log_fit_warp.cu", "constrained_fit.cu", "dki_metrics.cu", "noalloc.cu", "lsi.cu", "multi_tissue.cu", "sh_project.cu", "peaks.cu", "staging.cu", "csd.cu", "drl.cu", "plain_fp32.cu", "drl_tc.cu", "batch.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3", "-shared",
    "-I", str(ROOT / "include"),
]


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build larmor_b200")
    return found


def stale() -> bool:
    if not LIB.exists():
        return True
    mtime = LIB.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp"))
    deps.append(ROOT / "include" / "larmor_b200.h")
    return any(p.stat().st_mtime > mtime for p in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compiles every CUDA source into liblarmor_b200.so (one nvcc per source, in parallel, then
    one link); returns its path."""
    if not force and not stale():
        return LIB
    import os
    import tempfile
    from concurrent.futures import ThreadPoolExecutor

    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    with tempfile.TemporaryDirectory(prefix="larmor_b200_build_") as tmp:
        objects = [str(Path(tmp) / (Path(src).stem + ".o")) for src in SOURCES]

        def compile_one(job):
            src, obj = job
            cmd = [nvcc(), *compile_flags, "-c", str(CSRC / src), "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            return subprocess.run(cmd, capture_output=True, text=True)

        with ThreadPoolExecutor(max(1, min(len(SOURCES), os.cpu_count() or 1))) as pool:
            results = list(pool.map(compile_one, zip(SOURCES, objects)))
        for src, r in zip(SOURCES, results):
            if verbose or r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode:
                raise subprocess.CalledProcessError(r.returncode, f"nvcc -c {src}")
        link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objects, "-o", str(LIB)]
        subprocess.run(link, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
