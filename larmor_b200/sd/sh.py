"""Real even-degree spherical harmonic bases (src/larmor/sd/sh.py).

The bases ("tournier" as MRtrix, "descoteaux", "leemans" as ExploreDTI/MRIToolkit) and their
coefficient order (by l, then m from -l to l) define the FOD coefficients the models return,
so they follow the reference's definitions exactly.
"""

from __future__ import annotations

import math

import numpy as np
from scipy.special import lpmv

from larmor_b200.sd.sphere import get_theta_phi

BASES = ("tournier", "descoteaux", "leemans")


def get_sh_indices(lmax: int, full: bool = False) -> tuple[np.ndarray, np.ndarray]:
    step = 1 if full else 2
    ls, ms = [], []
    for ell in range(0, lmax + 1, step):
        for m in range(-ell, ell + 1):
            ls.append(ell)
            ms.append(m)
    return np.array(ls), np.array(ms)


def get_sh_coeffs(ell: int, m: int, theta, phi, basis: str = "tournier") -> np.ndarray:
    """Y_lm at the directions, with the Condon-Shortley phase in the Legendre functions."""
    if basis == "leemans":
        return get_sh_coeffs(ell, m, theta, phi - np.pi / 2, "tournier")
    a = abs(m)
    norm = np.sqrt((2 * ell + 1) / (4.0 * np.pi) * (math.factorial(ell - a) / math.factorial(ell + a)))
    val = norm * lpmv(a, ell, np.cos(theta))
    if basis == "tournier":
        if m < 0:
            return np.sqrt(2) * val * np.sin(a * phi)
        if m == 0:
            return val
        return np.sqrt(2) * val * np.cos(m * phi)
    if basis == "descoteaux":
        if m < 0:
            return np.sqrt(2) * (-1) ** a * val * np.cos(a * phi)
        if m == 0:
            return val
        return np.sqrt(2) * val * np.sin(m * phi)
    raise ValueError(f"Unsupported basis {basis}")


def build_basis_matrix(theta, phi, lmax: int, basis: str = "tournier", full: bool = False) -> np.ndarray:
    ls, ms = get_sh_indices(lmax, full)
    out = np.zeros((len(theta), len(ls)))
    for j, (ell, m) in enumerate(zip(ls, ms)):
        out[:, j] = get_sh_coeffs(ell, m, theta, phi, basis)
    return out


def fit_sh(amplitudes, directions, lmax: int, *, basis: str = "tournier", full: bool = False) -> np.ndarray:
    values = np.asarray(amplitudes, dtype=np.float64)
    dirs = np.asarray(directions, dtype=np.float64)
    theta, phi = get_theta_phi(dirs)
    matrix = build_basis_matrix(theta, phi, lmax, basis, full=full)
    flat = values.reshape(-1, values.shape[-1])
    coeffs = np.linalg.lstsq(matrix, flat.T)[0].T
    return coeffs.reshape(*values.shape[:-1], matrix.shape[1])


def sh_layout(num_coeffs: int) -> tuple[int, bool]:
    lmax = (-3 + math.isqrt(8 * num_coeffs + 1)) // 2
    if num_coeffs >= 1 and (lmax + 1) * (lmax + 2) // 2 == num_coeffs and lmax % 2 == 0:
        return lmax, False
    lmax = math.isqrt(num_coeffs) - 1
    if num_coeffs >= 1 and (lmax + 1) ** 2 == num_coeffs:
        return lmax, True
    raise ValueError(f"{num_coeffs} SH coefficients fit no layout: a symmetric FOD has (lmax + 1)(lmax + 2) / 2 "
                     "(1, 6, 15, 28, 45, ...), an asymmetric one (lmax + 1)^2 (4, 9, 16, 25, ...).")


def _perm_sign(lmax: int, full: bool, basis: str):
    _, ms = get_sh_indices(lmax, full)
    idx = np.arange(len(ms))
    a = np.abs(ms)
    sign_of = lambda k: 1 - 2 * (k % 2)  # noqa: E731
    if basis == "tournier":
        return idx, np.ones(len(ms), dtype=np.int8)
    if basis == "descoteaux":
        return idx - 2 * ms, np.where(ms < 0, sign_of(a), 1).astype(np.int8)
    if basis == "leemans":
        odd = a % 2 == 1
        perm = np.where(odd, idx - 2 * ms, idx)
        sign = np.where(odd, np.where(ms < 0, -1, 1) * sign_of((a - 1) // 2), sign_of(a // 2))
        return perm, sign.astype(np.int8)
    raise ValueError(f"Invalid basis {basis}, expected one of {', '.join(BASES)}")


def convert_sh_basis(coeffs: np.ndarray, from_basis: str, to_basis: str) -> np.ndarray:
    for b in (from_basis, to_basis):
        if b not in BASES:
            raise ValueError(f"Invalid basis {b}, expected one of {', '.join(BASES)}")
    lmax, full = sh_layout(coeffs.shape[-1])
    if from_basis == to_basis:
        return np.copy(coeffs)
    p_from, s_from = _perm_sign(lmax, full, from_basis)
    p_to, s_to = _perm_sign(lmax, full, to_basis)
    tournier = coeffs[..., p_from] * s_from[p_from]
    return tournier[..., p_to] * s_to
