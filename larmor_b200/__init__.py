"""larmor_b200: Larmor's voxelwise fitting hot path (DTI/DKI least squares, MSMT-CSD and mFOD
NNLS/LSI) as sm_100a CUDA kernels behind a C ABI, with the reference's Python API.

The CUDA library is liblarmor_b200.so beside this file (build: python -m larmor_b200.build);
its C ABI is include/larmor_b200.h. There is no CPU fallback.
"""

from larmor_b200.types import GradientTable, Volume

__all__ = ["GradientTable", "Volume"]
__version__ = "0.1.0"
