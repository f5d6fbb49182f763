"""The solve of single-shell constrained spherical deconvolution (CSD) on the GPU, with the API
of src/larmor/sd/csd_solver.py.

The settings (CSDSolver), the shell choice and the problem's matrices are built on the host as
the reference builds them: the forward model M = basis x the response's rotational harmonics,
the constraint rows (the SH basis on the constraint directions, weighted by
neg_lambda * 50 * c_0 / n_directions), the norm penalty norm_lambda * 2e-4 * (M^T M)_00, and
the linear estimate the iterations start from. The per-voxel solve runs on the device
(_core.fit_csd -> lar_fit_csd).

References:
    Tournier JD, Calamante F, Connelly A. Robust determination of the fibre orientation
    distribution in diffusion MRI: non-negativity constrained super-resolved spherical
    deconvolution. NeuroImage 35 (2007) 1459-1472. The defaults and the weight scaling are
    those of MRtrix3's dwi2fod csd.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from math import isfinite

import numpy as np

from larmor_b200 import _core
from larmor_b200._log import LarmorLogger
from larmor_b200.sd.sh import build_basis_matrix, get_sh_indices
from larmor_b200.sd.sphere import DIRS_300, get_theta_phi
from larmor_b200.types import GradientTable

# Scale of the non-negativity weight: neg_lambda * CONSTRAINT_SCALE * c_0 / n_directions.
CONSTRAINT_SCALE = 50.0
# Scale of the norm penalty: norm_lambda * NORM_SCALE * (M^T M)_00.
NORM_SCALE = 2e-4


@dataclass(frozen=True, kw_only=True)
class CSDSolver:
    """The settings of CSD (src/larmor/sd/csd_solver.py:CSDSolver): the non-negativity and norm
    strengths, the amplitude below which a direction is constrained (in FOD units), the most
    constrained solves per voxel (0 gives the linear estimate), the degree of the linear start,
    and the constraint directions (None: the 300 built-in ones).

    Raises:
        ValueError: If a lambda is negative or not finite, the threshold is not finite, max_iter
            is negative, init_lmax is odd or negative, or the directions are not an (n, 3) array
            of finite, non-zero vectors.
    """

    neg_lambda: float = 1.0
    norm_lambda: float = 1.0
    threshold: float = 0.0
    max_iter: int = 50
    init_lmax: int = 4
    directions: np.ndarray | None = field(default=None, compare=False)

    def __post_init__(self) -> None:
        for name in ("neg_lambda", "norm_lambda"):
            value = getattr(self, name)
            if not isfinite(value) or value < 0:
                raise ValueError(f"{name} must be a finite number >= 0, got {value}")
        if not isfinite(self.threshold):
            raise ValueError(f"threshold must be finite, got {self.threshold}")
        if self.max_iter < 0:
            raise ValueError(f"max_iter must be at least 0, got {self.max_iter}")
        if self.init_lmax < 0 or self.init_lmax % 2:
            raise ValueError(f"init_lmax must be even and >= 0, got {self.init_lmax}")
        if self.directions is not None:
            dirs = np.asarray(self.directions)
            if dirs.ndim != 2 or dirs.shape[1] != 3 or len(dirs) == 0:
                raise ValueError(f"directions must be an (n, 3) array, got shape {dirs.shape}")
            lengths = np.linalg.norm(dirs, axis=1)
            bad = ~(np.isfinite(lengths) & (lengths > 0))
            if bad.any():
                raise ValueError(f"directions must be finite, non-zero vectors; rows {np.flatnonzero(bad)} are not")


def csd_shell(gtab: GradientTable) -> float:
    """The b-value of the shell CSD fits: the highest.

    Raises:
        ValueError: If every volume is a b0.
    """
    shells = gtab.shells
    if len(shells) == 0:
        raise ValueError("CSD needs a diffusion-weighted shell; every volume is a b0.")
    return float(shells[-1])


def rotational_harmonics(zonal: np.ndarray, lmax: int) -> np.ndarray:
    """The convolution factor c_l / sqrt((2l + 1) / 4 pi) of each even degree l <= lmax; 0 for the
    degrees the response lacks."""
    factors = np.zeros(lmax // 2 + 1)
    n = min(len(factors), len(zonal))
    ell = 2 * np.arange(n)
    factors[:n] = zonal[:n] / np.sqrt((2 * ell + 1) / (4 * np.pi))
    return factors


def sh_basis(dirs: np.ndarray, lmax: int) -> np.ndarray:
    """The tournier SH basis up to lmax on unit vectors, (n, C)."""
    theta, phi = get_theta_phi(dirs)
    return build_basis_matrix(theta, phi, lmax, "tournier")


def initial_matrix(bvecs: np.ndarray, zonal: np.ndarray, lmax: int, init_lmax: int) -> np.ndarray:
    """The linear deconvolution the iterations start from, (C0, n_meas): a least-squares SH fit
    of the signal up to the highest degree the measurements, the response and lmax allow, each
    coefficient divided by its convolution factor, the degrees above init_lmax dropped."""
    n_meas = len(bvecs)
    data_lmax = 0
    while (data_lmax + 3) * (data_lmax + 4) // 2 <= n_meas:
        data_lmax += 2
    fit_lmax = min(data_lmax, 2 * (len(zonal) - 1), lmax)
    ell = get_sh_indices(fit_lmax)[0]
    factors = rotational_harmonics(zonal, fit_lmax)[ell // 2]
    keep = ell <= min(fit_lmax, init_lmax)
    return (np.linalg.pinv(sh_basis(bvecs, fit_lmax)) / factors[:, None])[keep]


@dataclass(frozen=True)
class CSDProblem:
    """The matrices and settings of one shell's CSD fit: initial (C0, m), forward (m, C),
    constraint (k, C), the norm weight, the threshold (weighted) and the iteration limit."""

    initial: np.ndarray
    forward: np.ndarray
    constraint: np.ndarray
    norm_weight: float
    threshold: float
    max_iter: int


def csd_problem(bvecs: np.ndarray, zonal: np.ndarray, lmax: int, solver: CSDSolver) -> CSDProblem:
    """Checks a CSD fit of one shell and builds its matrices
    (src/larmor/sd/csd_solver.py:csd_problem).

    Raises:
        ValueError: If the shell has fewer than 6 measurements, the response's l = 0 coefficient
            is not positive or it has no anisotropic degree, or norm_lambda is 0 while the data
            or the response do not determine every coefficient (the solve would be singular).
    """
    if len(bvecs) < 6:
        raise ValueError(f"CSD needs at least 6 measurements on the shell, got {len(bvecs)}.")
    if not zonal[0] > 0 or len(zonal) < 2:
        raise ValueError("The response needs a positive l = 0 coefficient and at least one anisotropic degree "
                         "(l = 2).")
    response_lmax = 2 * (len(zonal) - 1)
    if lmax > response_lmax:
        LarmorLogger.warning(f"The response has degrees up to {response_lmax} only; the FOD's degrees up to "
                             f"{lmax} above it are set by the constraint alone.")
    ell = get_sh_indices(lmax)[0]
    if solver.norm_lambda == 0 and (len(ell) > len(bvecs) or lmax > response_lmax):
        raise ValueError(f"norm_lambda 0 leaves the solve singular: lmax {lmax} has {len(ell)} coefficients for "
                         f"{len(bvecs)} measurements and a response up to degree {response_lmax}; give "
                         "norm_lambda > 0.")
    forward = sh_basis(bvecs, lmax) * rotational_harmonics(zonal, lmax)[ell // 2]
    directions = np.asarray(DIRS_300 if solver.directions is None else solver.directions, dtype=np.float64)
    directions = directions / np.linalg.norm(directions, axis=1, keepdims=True)
    weight = solver.neg_lambda * CONSTRAINT_SCALE * zonal[0] / len(directions)
    constraint = sh_basis(directions, lmax) * weight
    norm_weight = solver.norm_lambda * NORM_SCALE * float(forward[:, 0] @ forward[:, 0])
    return CSDProblem(
        initial=np.ascontiguousarray(initial_matrix(bvecs, zonal, lmax, solver.init_lmax)),
        forward=np.ascontiguousarray(forward),
        constraint=np.ascontiguousarray(constraint),
        norm_weight=norm_weight,
        threshold=solver.threshold * weight,
        max_iter=solver.max_iter,
    )


def solve_csd(signals: np.ndarray, problem: CSDProblem, n_threads: int) -> tuple[np.ndarray, np.ndarray]:
    """The FODs (n, C) of the signals (n, m) in the tournier basis, negative samples fitted as 0,
    and whether each voxel's set of constrained directions repeated (n,)."""
    return _core.fit_csd(np.ascontiguousarray(np.maximum(signals, 0.0), dtype=np.float64), problem.initial,
                         problem.forward, problem.constraint, norm_weight=problem.norm_weight,
                         threshold=problem.threshold, max_iter=problem.max_iter, n_threads=n_threads)


def warn_unconverged(n_unconverged: int, max_iter: int) -> None:
    if n_unconverged:
        LarmorLogger.warning(f"{n_unconverged} voxels did not converge within {max_iter} iterations; their FODs "
                             "are those of the last one.")


def fit_csd(signals: np.ndarray, bvecs: np.ndarray, zonal: np.ndarray, lmax: int, solver: CSDSolver,
            n_threads: int) -> np.ndarray:
    """The FODs (n, C) of many voxels of one shell (src/larmor/sd/csd_solver.py:fit_csd)."""
    problem = csd_problem(bvecs, zonal, lmax, solver)
    fods, converged = solve_csd(signals, problem, n_threads)
    warn_unconverged(int((~converged).sum()), solver.max_iter)
    return fods
