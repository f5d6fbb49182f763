"""MSMT-CSD as a linearly constrained least-squares problem, and its GPU fit.

The unknowns of a voxel are the SH coefficients of every tissue's FOD, concatenated in tissue
order; an isotropic tissue contributes its c00 only. A measurement with b-value b and unit
gradient direction g is modelled as the Funk-Hecke convolution of each FOD with its tissue's
zonal response:

    s(b, g) = sum_t sum_(l, m)  k_l * R_t,l(b) * Y_lm(g) * x_t,lm,    k_l = sqrt(4 pi / (2l + 1)),

where R_t,l(b) is the response's degree-l coefficient on the shell of b (0 past the response's
own lmax) and Y_lm the real tournier basis. A measurement without a direction (a b0) sees only
l = 0. The inequality constraints keep every anisotropic FOD's amplitude non-negative on a set
of directions and every isotropic coefficient non-negative. The matrices follow
src/larmor/sd/msmt.py:20-116 in value; the LSI itself runs on the device (lar_fit_lsi).
"""

from __future__ import annotations

import numpy as np

from larmor_b200 import _core
from larmor_b200.sd.rf import ZonalSHRF
from larmor_b200.sd.sh import build_basis_matrix, get_sh_indices
from larmor_b200.sd.sphere import get_theta_phi

# The LSI's ridge is sqrt(NORM_REG) times the largest column norm of the forward matrix.
NORM_REG = 1e-10


def _unknowns(lmaxes: list[int]) -> tuple[np.ndarray, np.ndarray]:
    """The SH degree and the tissue of every unknown, in the order of the concatenated
    coefficient vector."""
    degree = [get_sh_indices(lmax)[0] for lmax in lmaxes]
    tissue = [np.full(len(d), t) for t, d in enumerate(degree)]
    return np.concatenate(degree), np.concatenate(tissue)


def forward_matrix(rfs: list[ZonalSHRF], lmaxes: list[int], bvals: np.ndarray, bvecs: np.ndarray) -> np.ndarray:
    """The (measurements, unknowns) matrix A of the model above: A[i, j] = Y_j(g_i) k_l R_t,l(b_i)
    for unknown j of degree l in tissue t."""
    degree, tissue = _unknowns(lmaxes)
    directed = np.linalg.norm(bvecs, axis=1) > 0
    theta, phi = get_theta_phi(np.where(directed[:, None], bvecs, np.array([0.0, 0.0, 1.0])))
    # The basis value of every unknown's (l, m) at every measurement; b0s carry only l = 0.
    sh = np.hstack([build_basis_matrix(theta, phi, lmax) for lmax in lmaxes])
    sh[np.ix_(~directed, degree > 0)] = 0.0
    # Each unknown's radial gain R_t,l(b) on each measurement's shell, 0 past the response.
    gain = np.zeros((len(bvals), len(degree)))
    for t, rf in enumerate(rfs):
        columns = np.flatnonzero(tissue == t)
        per_shell = np.stack([rf.shell_coefficients(b) for b in bvals])
        slot = degree[columns] // 2
        known = slot < per_shell.shape[1]
        gain[:, columns[known]] = per_shell[:, slot[known]]
    funk_hecke = np.sqrt(4 * np.pi / (2 * degree + 1))
    return sh * funk_hecke * gain


def constraint_matrix(lmaxes: list[int], dirs: np.ndarray) -> np.ndarray:
    """The rows of G x >= 0: an anisotropic tissue's FOD amplitude on every direction (its SH
    basis there), an isotropic tissue's one coefficient."""
    degree, tissue = _unknowns(lmaxes)
    theta, phi = get_theta_phi(dirs)
    n_rows = sum(1 if lmax == 0 else len(dirs) for lmax in lmaxes)
    g = np.zeros((n_rows, len(degree)))
    row = 0
    for t, lmax in enumerate(lmaxes):
        columns = np.flatnonzero(tissue == t)
        if lmax == 0:
            g[row, columns[0]] = 1.0
            row += 1
        else:
            g[row:row + len(dirs), columns] = build_basis_matrix(theta, phi, lmax)
            row += len(dirs)
    return g


def prepare_msmt(rfs, lmaxes, bvals, bvecs, dirs) -> _core.LsiDesign:
    """The LSI design of an MSMT-CSD fit: the forward and constraint matrices above and the ridge
    sqrt(NORM_REG * largest squared column norm), prepared once on the device.

    Raises:
        ValueError: If the forward matrix has fewer independent columns than unknowns, so that
            the measurements cannot separate the tissues' coefficients.
    """
    forward = forward_matrix(rfs, lmaxes, bvals, bvecs)
    n_unknowns = forward.shape[1]
    rank = int(np.linalg.matrix_rank(forward))
    if rank < n_unknowns:
        raise ValueError(
            f"The gradient table cannot separate {n_unknowns} SH coefficients of {len(rfs)} tissues at lmax "
            f"{max(lmaxes)}: its forward matrix has rank {rank}. Use a table with more b-values or "
            "directions, fewer tissues, or a lower lmax."
        )
    largest = float(np.max(np.sum(forward**2, axis=0)))
    ridge = float(np.sqrt(NORM_REG * largest))
    return _core.LsiDesign(np.ascontiguousarray(forward), np.ascontiguousarray(constraint_matrix(lmaxes, dirs)),
                           ridge)


def fit_msmt(signals: np.ndarray, design: _core.LsiDesign, n_threads: int):
    """The coefficients (v, n) and converged flags (v,) of every voxel (fit_lsi on the GPU)."""
    return _core.fit_lsi(np.ascontiguousarray(signals, dtype=np.float64), design, n_threads=n_threads)
