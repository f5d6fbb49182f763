"""Diffusion kurtosis imaging (DKI) on the GPU, with the API of src/larmor/dwi/dki.py.

`DKIModel(fit_method=..., constrained=...).fit(volume, gtab, mask)` returns the reference's
`DKIFit` maps. The host estimates S0 and the sample floor and gathers the masked float32
signals; on the device one kernel caps and floors the samples and runs the 22-parameter
(I)RLS fit (a warp per voxel), a second re-fits the voxels that break a constraint (least
distance by NNLS, FP64), and a third computes the DTI and kurtosis maps.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from larmor_b200 import _core, _lib
from larmor_b200._log import LarmorLogger
from larmor_b200._threads import n_threads
from larmor_b200.dwi.dti import LOG_SIGNAL_TOL, MAX_REWEIGHTINGS, PRECISIONS
from larmor_b200.dwi.inputs import (
    as_mask,
    check_dwi,
    stage_dwi,
)
from larmor_b200.dwi.mask import unmask_maps
from larmor_b200.types import GradientTable, Volume

FIT_METHODS = ("ols", "wls")
# The 15 unique elements of the kurtosis tensor (0 = x), in the order of DKIFit.kt, and the
# number of distinct permutations of each (src/larmor/dwi/dki.py:30-48).
KT_INDICES = (
    (0, 0, 0, 0), (1, 1, 1, 1), (2, 2, 2, 2), (0, 0, 0, 1), (0, 0, 0, 2), (1, 1, 1, 0),
    (1, 1, 1, 2), (2, 2, 2, 0), (2, 2, 2, 1), (0, 0, 1, 1), (0, 0, 2, 2), (1, 1, 2, 2),
    (0, 0, 1, 2), (1, 1, 0, 2), (2, 2, 0, 1),
)
KT_MULTIPLICITY = (1, 1, 1, 4, 4, 4, 4, 4, 4, 6, 6, 6, 12, 12, 12)
# Constant C of the bound K(n) <= C / (b_max D(n)), and the constraint directions.
KURTOSIS_BOUND_C = 3.0
N_CONSTRAINT_DIRS = 256


@dataclass(frozen=True)
class DKIFit:
    """Result of a DKI fit as float32 maps on the grid (zero outside the fitted mask); the
    fields are the reference's DKIFit (src/larmor/dwi/dki.py:64-113)."""

    dt: np.ndarray
    kt: np.ndarray
    s0: np.ndarray
    fa: np.ndarray
    md: np.ndarray
    ad: np.ndarray
    rd: np.ndarray
    pe: np.ndarray
    eigen_vals: np.ndarray
    npd: np.ndarray
    mk: np.ndarray
    ak: np.ndarray
    rk: np.ndarray
    ka: np.ndarray


def _kt_rows(dirs: np.ndarray) -> np.ndarray:
    return np.stack([m * dirs[:, i] * dirs[:, j] * dirs[:, k] * dirs[:, q]
                     for (i, j, k, q), m in zip(KT_INDICES, KT_MULTIPLICITY)], axis=1)


def dki_design(gtab: GradientTable) -> np.ndarray:
    """The design (N, 22): log S0, the six D elements, the fifteen of MD^2 W
    (src/larmor/dwi/dki.py:345-380)."""
    if gtab.count_shells() < 2:
        raise ValueError(
            "DKI needs at least two non-zero b-value shells; the gradient table has "
            f"{gtab.count_shells()}."
        )
    b2 = gtab.bvals**2 / 6
    g = gtab.bvecs
    kt_columns = [m * b2 * g[:, i] * g[:, j] * g[:, k] * g[:, q]
                  for (i, j, k, q), m in zip(KT_INDICES, KT_MULTIPLICITY)]
    design = np.column_stack([np.ones(len(b2)), -gtab.b_matrix, *kt_columns])
    norms = np.linalg.norm(design, axis=0)
    if np.linalg.matrix_rank(design / np.where(norms > 0, norms, 1.0)) < design.shape[1]:
        raise ValueError(
            "The b-values and b-vectors cannot determine the diffusion and kurtosis tensors: "
            "DKI needs a b0 or a third shell, and enough non-collinear directions."
        )
    return design


def fibonacci_half_sphere(n: int) -> np.ndarray:
    """n unit vectors (n, 3) spread over the half sphere z > 0 (src/larmor/dwi/dki.py:414-420)."""
    i = np.arange(n) + 0.5
    z = 1 - i / n
    phi = np.pi * (3 - np.sqrt(5)) * i
    r = np.sqrt(1 - z**2)
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


def dki_constraints(gtab: GradientTable) -> np.ndarray:
    """G (768, 22) of D(n) >= 0, MD^2 W(n) >= 0 and the kurtosis upper bound on 256 directions
    (src/larmor/dwi/dki.py:383-411)."""
    dirs = fibonacci_half_sphere(N_CONSTRAINT_DIRS)
    x, y, z = dirs.T
    d_rows = np.stack([x * x, 2 * x * y, 2 * x * z, y * y, 2 * y * z, z * z], axis=1)
    v_rows = _kt_rows(dirs)
    zero_1 = np.zeros((len(dirs), 1))
    bound = KURTOSIS_BOUND_C / float(gtab.bvals.max())
    return np.vstack([
        np.hstack([zero_1, d_rows, np.zeros_like(v_rows)]),
        np.hstack([zero_1, np.zeros_like(d_rows), v_rows]),
        np.hstack([zero_1, bound * d_rows, -v_rows]),
    ])


class DKIModel:
    """Diffusion kurtosis imaging: a diffusion and a kurtosis tensor per voxel.

    Args:
        fit_method: "ols" or "wls" (default).
        constrained: Whether D(n) >= 0, K(n) >= 0 and K(n) <= 3 / (b_max D(n)) are imposed on
            256 directions (default True).
        precision: "fp64" (default) or "fp32" for the unconstrained fit; the constrained re-fit
            and the maps are FP64.
    """

    def __init__(self, *, fit_method: str = "wls", constrained: bool = True,
                 precision: str = "fp64") -> None:
        if fit_method not in FIT_METHODS:
            raise ValueError(
                f"Unknown DKI fit method {fit_method!r}: use one of {', '.join(FIT_METHODS)}."
            )
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {', '.join(PRECISIONS)}, got {precision!r}")
        self.fit_method = fit_method
        self.constrained = constrained
        self.precision = precision

    def fit(self, volume: Volume, gtab: GradientTable, mask=None, *, n_jobs: int = -1) -> DKIFit:
        """Fits both tensors in every voxel of the mask; see the reference's DKIModel.fit
        (src/larmor/dwi/dki.py:153-282). A mask is required."""
        n_threads(n_jobs)
        check_dwi(volume, gtab)
        design = dki_design(gtab)
        if mask is None:
            raise ValueError("DKIModel.fit needs a mask on the volume's grid.")
        mask = as_mask(volume, mask)
        fitted = mask.copy()
        is_b0 = gtab.b0_mask
        # The raw volume goes to the device once; S0, the float32 signals and the floors are
        # staged there (stage_dwi). Without b0s every voxel is fitted and floored from the
        # largest finite signal.
        staged = stage_dwi(volume, gtab, mask)
        signals, s0, floor = staged.signals, staged.s0, staged.floor
        if s0 is not None:
            torch = _core._torch()
            usable = (torch.isfinite(s0) & (s0 > 0)).cpu().numpy()
            if not usable.all():
                LarmorLogger.warning(
                    "%d mask voxels have no usable S0 (no plausible b0 in them or near them); "
                    "they are not fitted and come out as 0.", int((~usable).sum()))
                keep = torch.from_numpy(np.flatnonzero(usable)).to(s0.device)
                signals, s0, floor = signals[keep], s0[keep], floor[keep]
            fitted[mask] = usable
        g = dki_constraints(gtab) if self.constrained else np.zeros((0, design.shape[1]))
        maps, npd, broke = fit_dki_device(design, g, signals, s0, floor, is_b0,
                                          self.fit_method == "wls", PRECISIONS[self.precision])
        if self.constrained:
            LarmorLogger.info("%d of %d voxels break a constraint.", int(broke.sum().item()), len(broke))
        # The maps go back on the grid on the device; one copy of the grid leaves it.
        torch = _core._torch()
        flat = staged.flat if fitted is mask or np.array_equal(fitted, mask) else \
            torch.from_numpy(np.flatnonzero(fitted).astype(np.int64)).to(maps.device)
        grid = unmask_maps(maps, DKI_MAP_ROWS, flat, fitted.shape, flags=npd)
        return DKIFit(npd=grid["flags"], **{name: grid[name] for name, _, _ in DKI_MAP_ROWS})


# The rows of the fused fit's (36, v) maps that make up each DKIFit map.
DKI_MAP_ROWS = [("dt", 0, 6), ("fa", 6, 1), ("md", 7, 1), ("ad", 8, 1), ("rd", 9, 1), ("pe", 10, 3),
                ("eigen_vals", 13, 3), ("kt", 16, 15), ("s0", 31, 1), ("mk", 32, 1), ("ak", 33, 1),
                ("rk", 34, 1), ("ka", 35, 1)]


def fit_dki_signals(design, g, signals, s0, floor, is_b0, weighted, precision=_lib.LAR_FP64):
    """Fits float32 signals (v, N) on the device (host arrays, or device tensors for signals, s0
    and floor); returns maps (36, v), npd (v,), broke (v,) on the host."""
    maps, npd, broke = fit_dki_device(design, g, signals, s0, floor, is_b0, weighted, precision)
    return _core._to_host(maps), _core._to_host(npd).astype(bool), _core._to_host(broke).astype(bool)


def fit_dki_device(design, g, signals, s0, floor, is_b0, weighted, precision=_lib.LAR_FP64):
    """fit_dki_signals with the maps (36, v) float32, npd and broke (v,) uint8 on the device."""
    torch = _core._torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    handle = _core.LogDesign.cached(design, g)
    v = len(signals)
    maps = torch.empty((36, v), dtype=torch.float32, device=dev)
    npd = torch.empty((v,), dtype=torch.uint8, device=dev)
    broke = torch.empty((v,), dtype=torch.uint8, device=dev)
    params = torch.empty((v, 22), dtype=torch.float64, device=dev)
    if v:
        def dev_array(a, dtype):
            if a is None or not isinstance(a, np.ndarray):
                return None if a is None else a.contiguous()
            return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).to(dev)

        s = dev_array(signals, np.float32)
        f = dev_array(floor, np.float64)
        b0 = torch.from_numpy(np.ascontiguousarray(is_b0, dtype=np.uint8)).to(dev)
        s0d = dev_array(s0, np.float64)
        _lib.check(_lib.lib().lar_fit_dki_maps(
            handle.handle, _lib.ptr(s), _lib.ptr(s0d), _lib.ptr(f), _lib.ptr(b0), v, int(weighted),
            MAX_REWEIGHTINGS, LOG_SIGNAL_TOL, int(precision), _lib.ptr(maps), _lib.ptr(npd),
            _lib.ptr(broke), _lib.ptr(params), _core._stream(torch)))
    return maps, npd, broke


def dki_maps_device(params, maps, npd) -> None:
    """The 36 DKI maps of device params (v, 22)."""
    torch = _core._torch()
    _lib.check(_lib.lib().lar_dki_maps(_lib.ptr(params), params.shape[0], _lib.ptr(maps),
                                       _lib.ptr(npd), _core._stream(torch)))
