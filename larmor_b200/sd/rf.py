"""Response functions: the signal model of each tissue (src/larmor/sd/rf.py).

IsotropicRF, AnisotropicRF (a tensor with an isotropic kurtosis term) and ZonalSHRF (zonal SH
coefficients per shell, MRtrix's response format) give the columns of the deconvolution
kernels and forward matrices. Their formulas are the reference's, so the kernels agree.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import ClassVar

import numpy as np
from scipy.special import eval_legendre

# SHELL_TOLERANCE: a b-value belongs to a response's shell within this distance.
from larmor_b200.dwi.shells import SHELL_TOLERANCE
from larmor_b200.sd.sphere import get_theta_phi


@dataclass
class ResponseFunction:
    # Spiral points of an anisotropic response in the coarse loop of a multi-tissue fit.
    low_resolution_dirs: ClassVar[int] = 45

    def signal(self, bvals: np.ndarray, bvecs: np.ndarray, dirs: np.ndarray) -> np.ndarray:
        raise NotImplementedError


@dataclass
class IsotropicRF(ResponseFunction):
    """exp(-b D), one column."""

    diffusivity: float

    def signal(self, bvals, bvecs, dirs):
        return np.exp(-bvals * self.diffusivity)[:, np.newaxis]


@dataclass
class AnisotropicRF(ResponseFunction):
    """exp(-b g^T D g + b^2 MD^2 K / 6) + offset with D's first eigenvector along each direction."""

    eigen_vals: np.ndarray | list[float]
    mean_kurtosis: float
    signal_offset: float = field(default=0.0, kw_only=True)

    def signal(self, bvals, bvecs, dirs):
        l1, l2, l3 = self.eigen_vals
        a = np.diag([l2, l3, l1])
        theta, phi = get_theta_phi(dirs)
        ct, st, cp, sp = np.cos(theta), np.sin(theta), np.cos(phi), np.sin(phi)
        zeros = np.zeros_like(theta)
        r = np.stack([
            np.stack([cp * ct, -sp, cp * st], axis=-1),
            np.stack([sp * ct, cp, sp * st], axis=-1),
            np.stack([-st, zeros, ct], axis=-1),
        ], axis=-2)
        d_rot = r @ a @ np.swapaxes(r, -1, -2)
        gdg = np.einsum("mi, nij, mj -> mn", bvecs, d_rot, bvecs)
        md2 = np.mean(self.eigen_vals) ** 2
        b = bvals[:, np.newaxis]
        return np.exp(-b * gdg + (1 / 6) * (b**2) * md2 * self.mean_kurtosis) + self.signal_offset


@dataclass(kw_only=True)
class ZonalSHRF(ResponseFunction):
    """A response by its zonal SH coefficients (l = 0, 2, ...) on each shell (n_shells, n_l)."""

    bvals: np.ndarray
    coefficients: np.ndarray

    def __post_init__(self) -> None:
        self.bvals = np.atleast_1d(np.asarray(self.bvals, dtype=np.float64))
        self.coefficients = np.atleast_2d(np.asarray(self.coefficients, dtype=np.float64))
        if self.bvals.ndim != 1 or self.coefficients.shape[0] != len(self.bvals):
            raise ValueError(
                f"Expected one row of coefficients per b-value, got {len(self.bvals)} b-values "
                f"and coefficients of shape {self.coefficients.shape}."
            )
        if not np.isfinite(self.coefficients).all():
            raise ValueError("The response coefficients must be finite numbers.")

    @property
    def lmax(self) -> int:
        return 2 * (int(self.coefficients.shape[1]) - 1)

    def shell_coefficients(self, bval: float) -> np.ndarray:
        distances = np.abs(self.bvals - bval)
        nearest = int(np.argmin(distances))
        if distances[nearest] >= SHELL_TOLERANCE:
            shells = ", ".join(f"{b:g}" for b in self.bvals)
            raise ValueError(f"The response has no shell near b = {bval:g} s/mm^2; its shells are {shells}.")
        return self.coefficients[nearest]

    def signal(self, bvals, bvecs, dirs):
        cosines = np.clip(bvecs @ dirs.T, -1.0, 1.0)
        degrees = np.arange(0, self.lmax + 1, 2)
        per_meas = np.array([self.shell_coefficients(b) for b in bvals])
        weights = per_meas * np.sqrt((2 * degrees + 1) / (4 * np.pi))
        s = np.zeros(cosines.shape)
        for column, degree in enumerate(degrees):
            s += weights[:, column, np.newaxis] * eval_legendre(degree, cosines)
        return s
