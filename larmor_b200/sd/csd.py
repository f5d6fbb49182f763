"""Single-shell constrained spherical deconvolution (CSD) on the GPU, with the API of
src/larmor/sd/csd.py.

`CSDModel(response, solver=..., lmax=..., basis=...).fit(volume, gtab, mask)` fits the shell with
the highest b-value, as the reference does. The raw volume is staged on the device (stage_dwi).
The shell's samples of the voxels whose shell samples are all finite are clamped at 0 there, and
solved there (lar_fit_csd). Only the FOD coefficients come back. Estimating the response from the
data (the reference's estimate_csd_rf) is outside this package: pass a ZonalSHRF.
"""

from __future__ import annotations

import numpy as np

from larmor_b200 import _core
from larmor_b200._log import LarmorLogger
from larmor_b200._threads import n_threads
from larmor_b200.dwi.inputs import as_mask, check_dwi, stage_dwi
from larmor_b200.dwi.mask import unmask
from larmor_b200.sd.csd_solver import CSDSolver, csd_problem, csd_shell, warn_unconverged
from larmor_b200.sd.model import SDFit
from larmor_b200.sd.rf import ZonalSHRF
from larmor_b200.sd.sh import BASES, convert_sh_basis
from larmor_b200.types import GradientTable, Volume


class CSDModel:
    """Constrained spherical deconvolution of one shell (src/larmor/sd/csd.py:CSDModel).

    Args:
        response: The white matter response, with a row for the shell to fit.
        solver: The CSD settings. Defaults to CSDSolver's defaults.
        lmax: Maximum degree of the FOD's SH coefficients. Defaults to 8.
        basis: SH basis of the FODs fit returns. Defaults to "tournier".

    Raises:
        ValueError: If the response is not a ZonalSHRF, lmax is odd or below 2, or the basis is
            unknown.
    """

    def __init__(self, response: ZonalSHRF | None = None, *, solver: CSDSolver | None = None, lmax: int = 8,
                 basis: str = "tournier") -> None:
        if response is not None and not isinstance(response, ZonalSHRF):
            raise ValueError(f"CSD takes a ZonalSHRF response, got {type(response).__name__}.")
        if lmax < 2 or lmax % 2 != 0:
            raise ValueError(f"lmax must be even and at least 2, got {lmax}")
        if basis not in BASES:
            raise ValueError(f"Invalid basis {basis}, expected one of {', '.join(BASES)}")
        self.response = response
        self.solver = CSDSolver() if solver is None else solver
        self.lmax = lmax
        self.basis = basis

    def fit(self, volume: Volume, gtab: GradientTable, mask=None, *, n_jobs: int = -1) -> SDFit:
        """One FOD per mask voxel as SH coefficients in the model's basis, zero outside the mask,
        NaN where the voxel's samples on the shell are not finite; no tissue fractions
        (src/larmor/sd/csd.py:CSDModel.fit).

        Raises:
            ValueError: If n_jobs is 0 or below -1, the data have no diffusion-weighted shell, or
                the response has no row near its b-value.
            NotImplementedError: Without a response (estimating one is outside this package).
        """
        n_threads(n_jobs)
        check_dwi(volume, gtab)
        mask = np.ones(volume.data.shape[:-1], dtype=bool) if mask is None else as_mask(volume, mask)
        bval = csd_shell(gtab)
        on_shell = gtab.shell_index == int(np.argmin(np.abs(gtab.shells - bval)))
        if self.response is None:
            raise NotImplementedError("larmor_b200's CSDModel needs a response: estimating it from the data is "
                                      "outside this package")
        zonal = self.response.shell_coefficients(bval)
        if gtab.count_shells() > 1:
            LarmorLogger.warning(f"CSD fits one shell: using b = {bval:g} s/mm^2 ({int(on_shell.sum())} volumes) "
                                 "and leaving out the others.")
        problem = csd_problem(gtab.bvecs[on_shell], zonal, self.lmax, self.solver)
        torch = _core._torch()
        staged = stage_dwi(volume, gtab, mask)
        columns = torch.from_numpy(np.flatnonzero(on_shell)).to(staged.signals.device)
        shell = staged.signals.index_select(1, columns)
        finite = torch.isfinite(shell).all(dim=1).cpu().numpy()
        if not finite.all():
            LarmorLogger.warning(f"{int((~finite).sum())} voxels have a NaN or infinite signal; their FODs are NaN.")
            shell = shell[torch.from_numpy(np.flatnonzero(finite)).to(shell.device)]
        signals = shell.clamp(min=0.0).to(torch.float64).contiguous()
        handle = _core.CsdProblem.cached(problem.initial, problem.forward, problem.constraint, problem.norm_weight,
                                         problem.threshold, problem.max_iter)
        fods, converged = _core.fit_csd_device(handle, signals)
        warn_unconverged(int((converged == 0).sum().item()), self.solver.max_iter)
        coeffs = np.full((len(finite), problem.forward.shape[1]), np.nan)
        coeffs[finite] = fods.cpu().numpy()
        if self.basis != "tournier":
            coeffs = convert_sh_basis(coeffs, "tournier", self.basis)
        return SDFit(fods=[unmask(coeffs, mask)], tissue_fractions=None, basis=self.basis, lmax=self.lmax)
