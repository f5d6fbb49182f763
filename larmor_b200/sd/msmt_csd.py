"""Multi-shell multi-tissue CSD (MSMT-CSD) on the GPU, with the API of src/larmor/sd/msmt_csd.py.

`MSMTCSDModel(rfs, lmax=8).fit(volume, gtab, mask)` returns the reference's `SDFit`: one FOD
per anisotropic response (SH coefficients in the chosen basis) and, with several responses,
each tissue's fraction. The LSI problem is prepared once on the host (FP64) and every voxel is
solved by the lsi kernel (a warp per voxel).
"""

from __future__ import annotations

import numpy as np

from larmor_b200 import _core
from larmor_b200._log import LarmorLogger
from larmor_b200._threads import n_threads
from larmor_b200.dwi.inputs import as_mask, check_dwi, stage_dwi
from larmor_b200.dwi.mask import unmask
from larmor_b200.sd.model import SDFit
from larmor_b200.sd.msmt import prepare_msmt
from larmor_b200.sd.rf import ZonalSHRF
from larmor_b200.sd.sh import BASES, convert_sh_basis
from larmor_b200.sd.sphere import DIRS_300
from larmor_b200.types import GradientTable, Volume

FRACTION_SUM_OFFSET = 1e-16
# The relative peak threshold to give FOD peak finding for CSD and MSMT-CSD FODs.
PEAK_RELATIVE_THRESHOLD = 0.1


class MSMTCSDModel:
    """MSMT-CSD with one ZonalSHRF per tissue (anisotropic ones first in the outputs).

    Args:
        rfs: The responses; estimating them from the data is outside this package.
        lmax: Maximum SH degree of the FODs (even, >= 2), lowered to the anisotropic
            responses' lowest lmax.
        basis: SH basis of the returned FODs: "tournier", "leemans" or "descoteaux".
        directions: Unit vectors (n, 3) on which the FOD amplitudes are kept non-negative;
            defaults to the 300 built-in directions.
    """

    def __init__(self, rfs: list[ZonalSHRF], *, lmax: int = 8, basis: str = "tournier",
                 directions: np.ndarray | None = None, progress: bool = False) -> None:
        if lmax < 2 or lmax % 2 != 0:
            raise ValueError(f"lmax must be even and at least 2, got {lmax}")
        if basis not in BASES:
            raise ValueError(f"Invalid basis {basis}, expected one of {', '.join(BASES)}")
        if rfs is None:
            raise ValueError("MSMTCSDModel needs the tissue responses; estimating them is out of scope.")
        if not any(rf.lmax > 0 for rf in rfs):
            raise ValueError("MSMT-CSD needs at least one response with lmax above 0.")
        self.rfs = [rf for rf in rfs if rf.lmax > 0] + [rf for rf in rfs if rf.lmax == 0]
        self.lmax = lmax
        self.basis = basis
        self.directions = DIRS_300 if directions is None else np.asarray(directions)
        self.progress = progress

    def fit(self, volume: Volume, gtab: GradientTable, mask=None, *, n_jobs: int = -1) -> SDFit:
        """Fits the FODs and tissue fractions of every voxel of the mask (every voxel when
        None); see src/larmor/sd/msmt_csd.py:235-326. Voxels whose signal is not finite are NaN."""
        threads = n_threads(n_jobs)
        check_dwi(volume, gtab)
        mask = np.ones(volume.data.shape[:-1], dtype=bool) if mask is None else as_mask(volume, mask)
        rfs = self.rfs
        n_aniso = sum(1 for rf in rfs if rf.lmax > 0)
        lmax = min(self.lmax, *(rf.lmax for rf in rfs[:n_aniso]))
        if lmax < self.lmax:
            LarmorLogger.warning(f"lmax {self.lmax} is above the lmax of an anisotropic response, "
                                 f"lowering to {lmax}")
        lmaxes = [lmax] * n_aniso + [0] * (len(rfs) - n_aniso)
        sizes = [(d + 1) * (d + 2) // 2 for d in lmaxes]
        starts = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(int)
        design = prepare_msmt(rfs, lmaxes, gtab.bvals, gtab.bvecs, self.directions)
        # The raw volume goes to the device once and the mask voxels' signals are staged there.
        staged = stage_dwi(volume, gtab, mask)
        finite = staged.finite.cpu().numpy().astype(bool)
        if not finite.all():
            LarmorLogger.warning(f"{int((~finite).sum())} voxels have a NaN or infinite signal; their "
                                 "FODs and fractions are NaN.")
        torch = _core._torch()
        signals = staged.signals
        if not finite.all():
            signals = signals[torch.from_numpy(np.flatnonzero(finite)).to(signals.device)]
        signals = signals.to(torch.float64).contiguous()
        x = torch.empty((signals.shape[0], design.n), dtype=torch.float64, device=signals.device)
        conv = torch.empty((signals.shape[0],), dtype=torch.uint8, device=signals.device)
        if signals.shape[0]:
            _core.fit_lsi_device(design, signals, x, conv)
        fitted, converged = x.cpu().numpy(), conv.cpu().numpy().astype(bool)
        if not converged.all():
            LarmorLogger.warning(f"The constrained fit of {int((~converged).sum())} voxels stopped at "
                                 "its iteration limit; their FODs may be slightly negative.")
        coefficients = np.full((len(finite), fitted.shape[1]), np.nan)
        coefficients[finite] = fitted
        fods, fractions = fods_and_fractions(coefficients, mask, starts, sizes, n_aniso, self.basis)
        return SDFit(fods=fods, tissue_fractions=fractions, basis=self.basis, lmax=lmax,
                     peak_relative_threshold=PEAK_RELATIVE_THRESHOLD)


def fods_and_fractions(coefficients, mask, starts, sizes, n_aniso, basis):
    """FODs on the grid in `basis` and the fractions c00 sqrt(4 pi), normalised
    (src/larmor/sd/msmt_csd.py:329-363)."""
    fods = [unmask(convert_sh_basis(coefficients[:, s:s + n], "tournier", basis), mask)
            for s, n in zip(starts[:n_aniso], sizes[:n_aniso])]
    fractions = None
    if len(starts) > 1:
        shares = np.maximum(coefficients[:, starts] * np.sqrt(4 * np.pi), 0.0)
        total = shares.sum(axis=1, keepdims=True) + FRACTION_SUM_OFFSET
        fractions = unmask(shares / total, mask)
    return fods, fractions
