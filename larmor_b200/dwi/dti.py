"""Diffusion tensor imaging (DTI) on the GPU, with the API of src/larmor/dwi/dti.py.

`DTIModel(fit_method=...).fit(volume, gtab, mask)` returns the same `DTIFit` maps as the
reference. The raw volume goes to the device once; the staging kernels there scale the mask
voxels' samples, estimate S0 and the per-voxel sample floor (stage_dwi); one fused sm_100a
kernel then floors and logs the samples, fits
the tensor (OLS, or WLS iterated to a predicted-log change of 1e-6 or 20 reweightings), and
writes the 16 maps of compute_dti_metrics (src/larmor/dwi/dti.py:170-235).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from larmor_b200 import _core, _lib
from larmor_b200._log import LarmorLogger
from larmor_b200._threads import n_threads
from larmor_b200.dwi.inputs import as_mask, check_dwi, stage_dwi
from larmor_b200.dwi.mask import unmask_maps
from larmor_b200.types import GradientTable, Volume

FIT_METHODS = ("ols", "wls")
# Reweighting stops once no predicted log signal changes by more than this
# (src/larmor/dwi/fitting.py:9-12).
LOG_SIGNAL_TOL = 1e-6
MAX_REWEIGHTINGS = 20
PRECISIONS = {"fp64": _lib.LAR_FP64, "fp32": _lib.LAR_FP32}


@dataclass(frozen=True)
class DTIFit:
    """Result of a DTI fit, as float32 maps on the image grid (zero outside the mask); see
    the reference's DTIFit (src/larmor/dwi/dti.py:27-57) for the meaning of each map."""

    dt: np.ndarray
    fa: np.ndarray
    md: np.ndarray
    ad: np.ndarray
    rd: np.ndarray
    pe: np.ndarray
    eigen_vals: np.ndarray
    npd: np.ndarray


def dti_design(gtab: GradientTable) -> np.ndarray:
    """The design [1, -b_matrix] (N, 7) of the log signal (src/larmor/dwi/dti.py:148-154)."""
    design = np.column_stack([np.ones(len(gtab.bvals)), -gtab.b_matrix])
    if np.linalg.matrix_rank(design) < design.shape[1]:
        raise ValueError(
            "The b-values and b-vectors cannot determine a tensor: DTI needs at least two "
            "distinct b-values and six non-coplanar directions."
        )
    return design


class DTIModel:
    """Diffusion tensor imaging (DTI): one diffusion tensor per voxel.

    Args:
        fit_method: "ols" (default) or "wls".
        precision: "fp64" (default; the reference's double precision) or "fp32" (the plain
            single-precision kernel, kept for comparison).
    """

    def __init__(self, *, fit_method: str = "ols", precision: str = "fp64") -> None:
        if fit_method not in FIT_METHODS:
            raise ValueError(
                f"Unknown DTI fit method {fit_method!r}: use one of {', '.join(FIT_METHODS)}."
            )
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {', '.join(PRECISIONS)}, got {precision!r}")
        self.fit_method = fit_method
        self.precision = precision

    def fit(self, volume: Volume, gtab: GradientTable, mask=None, *, n_jobs: int = -1) -> DTIFit:
        """Fits the tensor in every voxel of the mask; see the reference's DTIModel.fit
        (src/larmor/dwi/dti.py:92-167). A mask is required: the automatic brain mask is outside
        this package."""
        n_threads(n_jobs)
        check_dwi(volume, gtab)
        if mask is None:
            raise ValueError("DTIModel.fit needs a mask on the volume's grid.")
        mask = as_mask(volume, mask)
        design = dti_design(gtab)
        staged = stage_dwi(volume, gtab, mask)
        maps, npd = fit_dti_device(design, staged.signals, staged.floor, self.fit_method == "wls",
                                   PRECISIONS[self.precision])
        # The maps go back on the grid on the device; one copy of the grid leaves it.
        grid = unmask_maps(maps, DTI_MAP_ROWS, staged.flat, mask.shape, flags=npd)
        n_npd = int(grid["flags"].sum())
        if n_npd:
            LarmorLogger.warning(
                "%d of %d fitted voxels have a tensor that is not positive definite.", n_npd, int(mask.sum()))
        return DTIFit(npd=grid["flags"], **{name: grid[name] for name, _, _ in DTI_MAP_ROWS})


# The rows of the fused fit's (16, v) maps that make up each DTIFit map.
DTI_MAP_ROWS = [("dt", 0, 6), ("fa", 6, 1), ("md", 7, 1), ("ad", 8, 1), ("rd", 9, 1), ("pe", 10, 3),
                ("eigen_vals", 13, 3)]


def fit_dti_signals(design: np.ndarray, signals: np.ndarray, floor: np.ndarray, weighted: bool,
                    precision: int = _lib.LAR_FP64) -> tuple[np.ndarray, np.ndarray]:
    """Fits float32 signals (v, N) (a host array or a device tensor) with per-voxel floors (v,)
    on the device; returns maps (16, v) and npd (v,) on the host."""
    maps, npd = fit_dti_device(design, signals, floor, weighted, precision)
    return _core._to_host(maps), _core._to_host(npd).astype(bool)


def fit_dti_device(design: np.ndarray, signals, floor, weighted: bool, precision: int = _lib.LAR_FP64):
    """fit_dti_signals with the maps (16, v) float32 and npd (v,) uint8 left on the device."""
    torch = _core._torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    handle = _core.LogDesign.cached(design, np.zeros((0, design.shape[1])))
    v = len(signals)
    maps = torch.empty((16, v), dtype=torch.float32, device=dev)
    npd = torch.empty((v,), dtype=torch.uint8, device=dev)
    if v:
        s = _core._on_device(torch, np.ascontiguousarray(signals, dtype=np.float32), dev) \
            if isinstance(signals, np.ndarray) else signals.contiguous()
        f = _core._on_device(torch, np.ascontiguousarray(floor, dtype=np.float64), dev) \
            if isinstance(floor, np.ndarray) else floor.contiguous()
        _core.fit_dti_maps_device(handle, s, f, weighted, maps, npd, max_iter=MAX_REWEIGHTINGS,
                                  tol=LOG_SIGNAL_TOL, precision=precision)
    return maps, npd
