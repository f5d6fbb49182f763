"""Seeded synthetic DWI workloads with the shapes and value distributions of the benchmark
configurations (no public dataset is named for them; these generators stand in).

- dti_volume: 64x64x40 float32, ellipsoid mask (79,912 voxels), 1 b0 + 30 unit directions at
  b = 1000 s/mm^2; tensors with l1 ~ U[1.2, 2.0]e-3, l2 = l3 ~ U[0.2, 0.6]e-3 mm^2/s, random
  orientation; S0 = 1000, Rician noise at SNR 20.
- dki_volume: 96x96x60, ellipsoid mask (199,768 voxels), 6 b0 + 64 directions at b = 1000 and
  64 at b = 2000; a stick (fraction U[0.3, 0.7], d = 2e-3) plus a zeppelin (d_par = 2e-3,
  d_perp ~ U[0.4, 0.8]e-3) with random orientation; S0 = 1000, SNR 30.
- mfod_volume: 110x110x70, ellipsoid mask (500,040 voxels), 10 b0 + 90 directions on each of
  b = 1000, 2000, 3000; 1-3 stick-zeppelin fibres (crossing angles U[30, 90] deg, fractions
  Dirichlet(2)) with GM (D = 0.8e-3) and CSF (D = 3e-3) partial volumes; SNR 25.

Rician noise is |S + sigma (n1 + i n2)| with sigma = S0 / SNR, as the reference's
src/larmor/simulation/noise.py:11 adds it.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from larmor_b200.types import GradientTable, Volume


@dataclass
class Workload:
    volume: Volume
    gtab: GradientTable
    mask: np.ndarray
    name: str

    @property
    def n_voxels(self) -> int:
        return int(self.mask.sum())


def ellipsoid_mask(shape: tuple[int, int, int], radius: float) -> np.ndarray:
    """The centred ellipsoid sum(((i - c) / (s / 2))^2) <= radius^2 of a grid."""
    grids = np.meshgrid(*[np.arange(s, dtype=np.float64) for s in shape], indexing="ij")
    total = np.zeros(shape)
    for g, s in zip(grids, shape):
        c = (s - 1) / 2.0
        total += ((g - c) / (s / 2.0)) ** 2
    return total <= radius**2


def unit_directions(rng: np.random.Generator, n: int) -> np.ndarray:
    d = rng.normal(size=(n, 3))
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """n rotation matrices (n, 3, 3): the Q of the QR of a normal 3x3, signs fixed."""
    a = rng.normal(size=(n, 3, 3))
    q, r = np.linalg.qr(a)
    q = q * np.sign(np.diagonal(r, axis1=1, axis2=2))[:, None, :]
    return q


def rician(rng: np.random.Generator, signal: np.ndarray, sigma: float) -> np.ndarray:
    n1 = rng.normal(size=signal.shape)
    n2 = rng.normal(size=signal.shape)
    return np.sqrt((signal + sigma * n1) ** 2 + (sigma * n2) ** 2)


def _fill(shape, mask, inside: np.ndarray) -> np.ndarray:
    data = np.zeros(shape + (inside.shape[1],), dtype=np.float32)
    data[mask] = inside.astype(np.float32)
    return data


def dti_volume(seed: int = 1, shape=(64, 64, 40), radius: float = 0.977, snr: float = 20.0,
               n_dirs: int = 30, s0: float = 1000.0) -> Workload:
    rng = np.random.default_rng(seed)
    mask = ellipsoid_mask(shape, radius)
    v = int(mask.sum())
    dirs = unit_directions(rng, n_dirs)
    bvals = np.concatenate([[0.0], np.full(n_dirs, 1000.0)])
    bvecs = np.vstack([np.zeros((1, 3)), dirs])
    l1 = rng.uniform(1.2e-3, 2.0e-3, v)
    l23 = rng.uniform(0.2e-3, 0.6e-3, v)
    rot = random_rotations(rng, v)
    evals = np.stack([l1, l23, l23], axis=1)
    tensors = np.einsum("vij,vj,vkj->vik", rot, evals, rot)
    adc = np.einsum("ni,vij,nj->vn", bvecs, tensors, bvecs)
    signal = s0 * np.exp(-bvals[None, :] * adc)
    noisy = rician(rng, signal, s0 / snr)
    return Workload(Volume(_fill(shape, mask, noisy), np.eye(4)), GradientTable(bvals, bvecs), mask, "dti")


def _stick_zeppelin(bvals, bvecs, axis, f, d_par, d_perp):
    """Signal (v, N) of a stick (fraction f) plus a zeppelin along unit axis (v, 3)."""
    cos2 = (bvecs @ axis.T).T ** 2  # (v, N)
    stick = np.exp(-bvals[None, :] * d_par * cos2)
    zep = np.exp(-bvals[None, :] * (d_perp[:, None] + (d_par - d_perp[:, None]) * cos2))
    return f[:, None] * stick + (1 - f[:, None]) * zep


def dki_volume(seed: int = 2, shape=(96, 96, 60), radius: float = 0.884, snr: float = 30.0,
               s0: float = 1000.0) -> Workload:
    rng = np.random.default_rng(seed)
    mask = ellipsoid_mask(shape, radius)
    v = int(mask.sum())
    d1, d2 = unit_directions(rng, 64), unit_directions(rng, 64)
    bvals = np.concatenate([np.zeros(6), np.full(64, 1000.0), np.full(64, 2000.0)])
    bvecs = np.vstack([np.zeros((6, 3)), d1, d2])
    axis = unit_directions(rng, v)
    f = rng.uniform(0.3, 0.7, v)
    d_perp = rng.uniform(0.4e-3, 0.8e-3, v)
    signal = s0 * _stick_zeppelin(bvals, bvecs, axis, f, 2.0e-3, d_perp)
    noisy = rician(rng, signal, s0 / snr)
    return Workload(Volume(_fill(shape, mask, noisy), np.eye(4)), GradientTable(bvals, bvecs), mask, "dki")


def mfod_table(rng: np.random.Generator) -> GradientTable:
    """10 b0 + 90 directions on each of b = 1000, 2000, 3000, the sets rotated between shells."""
    base = unit_directions(rng, 90)
    rots = random_rotations(rng, 3)
    bvals = np.concatenate([np.zeros(10)] + [np.full(90, b) for b in (1000.0, 2000.0, 3000.0)])
    bvecs = np.vstack([np.zeros((10, 3))] + [base @ r.T for r in rots])
    return GradientTable(bvals, bvecs)


def mfod_signals(rng: np.random.Generator, gtab: GradientTable, v: int, s0: float = 1000.0,
                 snr: float = 25.0) -> np.ndarray:
    """Signals (v, N) of 1-3 stick-zeppelin fibres plus GM and CSF partial volumes."""
    bvals, bvecs = gtab.bvals, gtab.bvecs
    n_fib = rng.integers(1, 4, v)
    first = unit_directions(rng, v)
    wm = np.zeros((v, len(bvals)))
    fractions = np.zeros((v, 3))
    for k in range(3):
        fractions[:, k] = rng.gamma(2.0, size=v)
    fractions = np.where(np.arange(3)[None, :] < n_fib[:, None], fractions, 0.0)
    fractions /= fractions.sum(axis=1, keepdims=True)
    axis = first
    for k in range(3):
        if k > 0:
            # A new fibre at U[30, 90] degrees from the first, about a random perpendicular.
            perp = np.cross(first, unit_directions(rng, v))
            perp /= np.linalg.norm(perp, axis=1, keepdims=True)
            ang = np.radians(rng.uniform(30.0, 90.0, v))
            axis = np.cos(ang)[:, None] * first + np.sin(ang)[:, None] * perp
        f_ic = np.full(v, 0.6)
        wm += fractions[:, k:k + 1] * _stick_zeppelin(bvals, bvecs, axis, f_ic, 1.7e-3, np.full(v, 0.5e-3))
    pv = rng.dirichlet([6.0, 2.0, 1.0], size=v)  # WM, GM, CSF shares
    gm = np.exp(-bvals * 0.8e-3)[None, :]
    csf = np.exp(-bvals * 3.0e-3)[None, :]
    signal = s0 * (pv[:, :1] * wm + pv[:, 1:2] * gm + pv[:, 2:3] * csf)
    return rician(rng, signal, s0 / snr)


def mfod_volume(seed: int = 3, shape=(110, 110, 70), radius: float = 1.0435) -> Workload:
    rng = np.random.default_rng(seed)
    mask = ellipsoid_mask(shape, radius)
    gtab = mfod_table(rng)
    signals = mfod_signals(rng, gtab, int(mask.sum()))
    return Workload(Volume(_fill(shape, mask, signals), np.eye(4)), gtab, mask, "mfod")


def mfod_responses(s0: float = 1000.0):
    """ZonalSHRF responses (WM, GM, CSF) of the mFOD generator's tissues on its shells: the WM
    profile of one stick-zeppelin fibre projected on the zonal SH by Gauss-Legendre quadrature,
    as the reference's tests build a tensor response (tests/sd/test_msmt.py:41-58)."""
    from larmor_b200.sd.rf import ZonalSHRF
    from larmor_b200.sd.sh import build_basis_matrix

    shells = np.array([0.0, 1000.0, 2000.0, 3000.0])
    nodes, weights = np.polynomial.legendre.leggauss(64)
    theta = np.arccos(nodes)
    zonal = build_basis_matrix(theta, np.zeros_like(theta), 8)[:, [0, 3, 10, 21, 36]]
    rows = []
    for b in shells:
        cos2 = nodes**2
        stick = np.exp(-b * 1.7e-3 * cos2)
        zep = np.exp(-b * (0.5e-3 + (1.7e-3 - 0.5e-3) * cos2))
        profile = s0 * (0.6 * stick + 0.4 * zep)
        rows.append(2 * np.pi * (weights * profile) @ zonal)
    wm = ZonalSHRF(bvals=shells, coefficients=np.array(rows))
    gm = ZonalSHRF(bvals=shells, coefficients=np.sqrt(4 * np.pi) * (s0 * np.exp(-shells * 0.8e-3))[:, None])
    csf = ZonalSHRF(bvals=shells, coefficients=np.sqrt(4 * np.pi) * (s0 * np.exp(-shells * 3e-3))[:, None])
    return [wm, gm, csf]


def mfod_model_responses():
    """The SDModel responses of the mFOD workload: the WM tensor of the single fibre
    (AnisotropicRF), GM and CSF isotropic."""
    from larmor_b200.sd.rf import AnisotropicRF, IsotropicRF

    return [AnisotropicRF([1.7e-3, 0.2e-3, 0.2e-3], 0.0), IsotropicRF(0.8e-3), IsotropicRF(3e-3)]
