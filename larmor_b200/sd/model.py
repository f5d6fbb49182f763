"""Spherical deconvolution results (src/larmor/sd/model.py:48-81)."""

from __future__ import annotations

import functools
from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class SDFit:
    """FODs (one per anisotropic response, SH coefficients (X, Y, Z, C) in `basis`), tissue
    fractions (X, Y, Z, N) or None for a single-tissue fit, the lmax used, and the relative
    threshold to give peak finding."""

    fods: list[np.ndarray]
    tissue_fractions: np.ndarray | None
    basis: str
    lmax: int
    peak_relative_threshold: float = 0.1


# ---- SDModel ---------------------------------------------------------------------------

from larmor_b200._log import LarmorLogger  # noqa: E402
from larmor_b200._threads import n_threads  # noqa: E402
from larmor_b200.dwi.inputs import as_mask, check_dwi, normalise_signals, stage_dwi  # noqa: E402
from larmor_b200.dwi.mask import unmask  # noqa: E402
from larmor_b200.sd.kernel import Kernel, order_rfs  # noqa: E402
from larmor_b200.sd.rf import IsotropicRF  # noqa: E402
from larmor_b200 import _core  # noqa: E402
from larmor_b200.sd.sh import BASES, build_basis_matrix, fit_sh  # noqa: E402
from larmor_b200.sd.sphere import DIRS_300, get_dirs, get_theta_phi  # noqa: E402
from larmor_b200.dwi.shells import SHELL_TOLERANCE, shell_mask  # noqa: E402,F401
from larmor_b200.sd.peaks import SD_MODEL_PEAK_RELATIVE_THRESHOLD  # noqa: E402


def compute_max_lmax(bvals: np.ndarray, proposed_lmax: int) -> int:
    """The largest even lmax <= proposed whose coefficients the highest shell's directions
    can determine (src/larmor/sd/model.py:443-468)."""
    n_dirs = np.sum(shell_mask(bvals, np.max(bvals)))
    lmax = proposed_lmax
    while lmax > 0:
        if n_dirs >= (lmax + 1) * (lmax + 2) // 2:
            return lmax
        lmax -= 2
    raise ValueError(f"Not enough gradient directions ({n_dirs}) to fit even lmax=2.")


def compute_shell_weights(bvals: np.ndarray, inner_weight: float = 0.2) -> np.ndarray:
    weights = np.full(bvals.shape, inner_weight, dtype=np.float64)
    weights[shell_mask(bvals, np.max(bvals))] = 1.0
    return weights


def low_resolution_dirs(rfs, n_meas: int) -> list[np.ndarray]:
    """Each anisotropic response's coarse directions: the spiral of min(n_meas, its count)
    points without its last, which repeats the first (src/larmor/sd/model.py:394-409)."""
    return [get_dirs(min(n_meas, rf.low_resolution_dirs))[:-1] for rf in rfs if not isinstance(rf, IsotropicRF)]


@functools.lru_cache(maxsize=16)
def sh_projector(lmax: int, basis: str):
    """The device projector of amplitudes on DIRS_300 onto the SH basis of lmax: the
    least-squares fit of fit_sh (pinv of the full-rank basis matrix) times 300 / (4 pi)."""
    from larmor_b200 import _core

    theta, phi = get_theta_phi(np.asarray(DIRS_300, dtype=np.float64))
    matrix = build_basis_matrix(theta, phi, lmax, basis)
    density = len(DIRS_300) / (4.0 * np.pi)
    return _core.ShProjector(np.ascontiguousarray(np.linalg.pinv(matrix) * density))


def to_sh(fods: np.ndarray, lmax: int, basis: str, *, exact_integral: bool = False) -> np.ndarray:
    """Amplitudes on DIRS_300 to SH coefficients, times 300 / (4 pi); with exact_integral c00 is
    the amplitudes' sum / sqrt(4 pi) (src/larmor/sd/model.py:412-440)."""
    density = len(DIRS_300) / (4.0 * np.pi)
    coeffs = fit_sh(fods, DIRS_300, lmax, basis=basis) * density
    if exact_integral:
        coeffs[:, 0] = fods.sum(axis=1) / np.sqrt(4.0 * np.pi)
    return coeffs


class SDModel:
    """Spherical deconvolution with the mFOD method (L2NNLS FODs, one per anisotropic response,
    all shells weighted equally), on the GPU; the reference's SDModel (src/larmor/sd/model.py:84).
    The GRL method takes the DRL solver (damped Richardson-Lucy), single- and multi-tissue."""

    def __init__(self, rfs, *, method="mFOD", solver=None, inner_shell_weight=None, lmax: int = 8,
                 basis: str = "tournier", progress: bool = False) -> None:
        from larmor_b200.sd.method import SDMethod

        if basis not in BASES:
            raise ValueError(f"Invalid basis {basis}, expected one of {', '.join(BASES)}")
        if lmax < 2 or lmax % 2 != 0:
            raise ValueError(f"lmax must be even and at least 2, got {lmax}")
        if inner_shell_weight is not None and not 0 < inner_shell_weight <= 1:
            raise ValueError(f"inner_shell_weight must be in (0, 1], got {inner_shell_weight}")
        self.rfs = order_rfs(rfs)
        self.method = SDMethod(method)
        self.method._check_rfs(self.rfs)
        self.solver = solver
        self.inner_shell_weight = self.method.inner_shell_weight if inner_shell_weight is None else inner_shell_weight
        self.lmax = lmax
        self.basis = basis
        self.num_iso = sum(1 for rf in self.rfs if isinstance(rf, IsotropicRF))
        self.is_multi_tissue = self.num_iso > 0 or len(self.rfs) - self.num_iso > 1
        self.progress = progress

    def fit(self, volume, gtab, mask=None, *, n_jobs: int = -1) -> SDFit:
        """The FODs (SH coefficients in the model's basis) and fractions of every voxel of the
        mask (every voxel when None); see src/larmor/sd/model.py:171-260."""
        from larmor_b200.sd.solvers import DRL, L2NNLS

        solver = self.solver if self.solver is not None else self.method.default_solver()
        if not isinstance(solver, (L2NNLS, DRL)):
            raise NotImplementedError("larmor_b200 runs the L2NNLS and DRL solvers only")
        threads = n_threads(n_jobs)
        check_dwi(volume, gtab)
        lmax = compute_max_lmax(gtab.bvals, self.lmax)
        if lmax < self.lmax:
            LarmorLogger.warning(f"lmax {self.lmax} needs more directions than the highest shell has, "
                                 f"lowering to {lmax}")
        mask = np.ones(volume.data.shape[:-1], dtype=bool) if mask is None else as_mask(volume, mask)
        if not gtab.b0_mask.any():
            raise ValueError(f"No b0 volume: no b-value is at or below {gtab.b0_threshold} s/mm^2.")
        # The raw volume goes to the device once: S0 and the signals normalised by it, capped at 1
        # (diffusion weighting only lowers the signal: a value above S0 is noise), are staged
        # there (stage_dwi, normalise_signals).
        staged = stage_dwi(volume, gtab, mask)
        normalised, finite = normalise_signals(staged.signals, staged.s0)
        finite = finite.cpu().numpy().astype(bool)
        if not finite.all():
            LarmorLogger.warning(f"{int((~finite).sum())} voxels have a NaN or infinite signal or no S0; "
                                 "their FODs and fractions are NaN.")
            keep = _core._torch().from_numpy(np.flatnonzero(finite)).to(normalised.device)
            normalised = normalised[keep]
        amplitudes, fitted_fractions, hr = self._fit_normalised(normalised, gtab, solver, threads)
        n_coeffs = (lmax + 1) * (lmax + 2) // 2
        projector = sh_projector(lmax, self.basis)
        fods = []
        for block in hr.aniso_blocks:
            sh = np.full((len(finite), n_coeffs), np.nan)
            if len(normalised):
                sh[finite] = _core.project_sh_device(projector, amplitudes[:, block], True).cpu().numpy()
            fods.append(unmask(sh, mask))
        fractions = None
        if fitted_fractions is not None:
            fr = np.full((len(finite), fitted_fractions.shape[1]), np.nan)
            fr[finite] = fitted_fractions
            fractions = unmask(fr, mask)
        return SDFit(fods=fods, tissue_fractions=fractions, basis=self.basis, lmax=lmax,
                     peak_relative_threshold=SD_MODEL_PEAK_RELATIVE_THRESHOLD)

    def _prepare(self, solver, bvals, bvecs):
        """The kernels and solvers of the fit (src/larmor/sd/model.py:272-321)."""
        from larmor_b200.sd.solvers import Stage

        if not self.is_multi_tissue:
            kernel = Kernel(self.rfs, bvals, bvecs, dirs=DIRS_300)
            return kernel, None, solver._prepare(kernel, bvals, Stage.SINGLE), None
        weights = compute_shell_weights(bvals, self.inner_shell_weight)
        hr = Kernel(self.rfs, bvals, bvecs, dirs=DIRS_300, weights=weights)
        lr = Kernel(self.rfs, bvals, bvecs, dirs=low_resolution_dirs(self.rfs, len(bvals)), weights=weights)
        return hr, lr, solver._prepare(hr, bvals, Stage.HIGH_RES), solver._prepare(lr, bvals, Stage.LOW_RES)

    def _fit_normalised(self, signals, gtab, solver, threads):
        """The high-resolution amplitudes (on the device) and fractions (host) of the
        S0-normalised signals."""
        from larmor_b200.sd.solvers import fit_multi_tissue_on_device, fit_single_tissue_on_device

        hr, lr, hr_solver, lr_solver = self._prepare(solver, gtab.bvals, gtab.bvecs)
        if lr is None:
            return fit_single_tissue_on_device(signals, hr_solver), None, hr
        fods, fractions = fit_multi_tissue_on_device(signals, lr, hr, lr_solver, hr_solver,
                                                     fraction_tol=self.method._fraction_tolerance)
        return fods, fractions.cpu().numpy(), hr
