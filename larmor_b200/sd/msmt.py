"""The constrained least-squares problem of MSMT-CSD (src/larmor/sd/msmt.py) and its GPU fit."""

from __future__ import annotations

import numpy as np

from larmor_b200 import _core
from larmor_b200.sd.rf import ZonalSHRF
from larmor_b200.sd.sh import build_basis_matrix, get_sh_indices
from larmor_b200.sd.sphere import get_theta_phi

# Ridge added to the normal matrix A^T A, relative to its largest diagonal entry.
NORM_REG = 1e-10


def _sh_size(lmax: int) -> int:
    return (lmax + 1) * (lmax + 2) // 2


def forward_matrix(rfs: list[ZonalSHRF], lmaxes: list[int], bvals: np.ndarray, bvecs: np.ndarray) -> np.ndarray:
    """The matrix (n_meas, sum of coefficients) from every tissue's SH coefficients to the
    signal: sqrt(4 pi / (2l + 1)) r_l(b) Y_lm(g) (src/larmor/sd/msmt.py:20-56)."""
    has_direction = np.linalg.norm(bvecs, axis=1) > 0
    theta, phi = get_theta_phi(np.where(has_direction[:, np.newaxis], bvecs, [0, 0, 1]))
    blocks = []
    for rf, tissue_lmax in zip(rfs, lmaxes, strict=True):
        degrees, _ = get_sh_indices(tissue_lmax)
        basis = build_basis_matrix(theta, phi, tissue_lmax)
        basis[np.ix_(~has_direction, degrees > 0)] = 0.0
        response = np.array([rf.shell_coefficients(b) for b in bvals])
        padded = np.zeros((len(bvals), tissue_lmax // 2 + 1))
        n_columns = min(padded.shape[1], response.shape[1])
        padded[:, :n_columns] = response[:, :n_columns]
        scale = np.sqrt(4 * np.pi / (2 * degrees + 1))
        blocks.append(basis * scale * padded[:, degrees // 2])
    return np.hstack(blocks)


def constraint_matrix(lmaxes: list[int], dirs: np.ndarray) -> np.ndarray:
    """G x >= 0: each FOD's amplitude on every direction, each isotropic coefficient
    (src/larmor/sd/msmt.py:59-83)."""
    theta, phi = get_theta_phi(dirs)
    n_columns = sum(_sh_size(t) for t in lmaxes)
    rows, start = [], 0
    for t in lmaxes:
        size = _sh_size(t)
        if t == 0:
            block = np.zeros((1, n_columns))
            block[0, start] = 1.0
        else:
            block = np.zeros((len(dirs), n_columns))
            block[:, start:start + size] = build_basis_matrix(theta, phi, t)
        rows.append(block)
        start += size
    return np.vstack(rows)


def prepare_msmt(rfs, lmaxes, bvals, bvecs, dirs) -> _core.LsiDesign:
    """The prepared LSI problem of an MSMT-CSD fit (src/larmor/sd/msmt.py:86-116)."""
    forward = forward_matrix(rfs, lmaxes, bvals, bvecs)
    rank = int(np.linalg.matrix_rank(forward))
    if rank < forward.shape[1]:
        raise ValueError(
            f"The measurements determine only {rank} of the {forward.shape[1]} SH coefficients of "
            f"{len(rfs)} tissues at lmax {max(lmaxes)}: they need more distinct b-values or "
            "directions, or fewer tissues or a lower lmax."
        )
    constraints = constraint_matrix(lmaxes, dirs)
    ridge = float(np.sqrt(NORM_REG * np.max(np.sum(forward**2, axis=0))))
    return _core.LsiDesign(np.ascontiguousarray(forward), np.ascontiguousarray(constraints), ridge)


def fit_msmt(signals: np.ndarray, design: _core.LsiDesign, n_threads: int):
    """The coefficients (v, n) and converged flags (v,) of every voxel (fit_lsi on the GPU)."""
    return _core.fit_lsi(np.ascontiguousarray(signals, dtype=np.float64), design, n_threads=n_threads)
