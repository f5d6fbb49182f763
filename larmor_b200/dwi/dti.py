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
from larmor_b200.dwi.mask import unmask
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
        maps, npd = fit_dti_signals(design, staged.signals, staged.floor, self.fit_method == "wls",
                                    PRECISIONS[self.precision])
        if npd.any():
            LarmorLogger.warning(
                "%d of %d fitted voxels have a tensor that is not positive definite.",
                int(npd.sum()), len(npd))
        return DTIFit(
            dt=unmask(maps[0:6].T, mask),
            fa=unmask(maps[6], mask),
            md=unmask(maps[7], mask),
            ad=unmask(maps[8], mask),
            rd=unmask(maps[9], mask),
            pe=unmask(maps[10:13].T, mask),
            eigen_vals=unmask(maps[13:16].T, mask),
            npd=unmask(npd, mask, fill_value=False, dtype=bool),
        )


def fit_dti_signals(design: np.ndarray, signals: np.ndarray, floor: np.ndarray, weighted: bool,
                    precision: int = _lib.LAR_FP64) -> tuple[np.ndarray, np.ndarray]:
    """Fits float32 signals (v, N) (a host array or a device tensor) with per-voxel floors (v,)
    on the device; returns maps (16, v) and npd (v,)."""
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
    return maps.cpu().numpy(), npd.cpu().numpy().astype(bool)
