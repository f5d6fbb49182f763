"""Spherical deconvolution methods (src/larmor/sd/method.py)."""

from __future__ import annotations

from enum import StrEnum

from larmor_b200.sd.rf import IsotropicRF
from larmor_b200.sd.solvers import DRL, FRACTION_TOL, L2NNLS


class SDMethod(StrEnum):
    GRL = "GRL"
    MFOD = "mFOD"

    @classmethod
    def _missing_(cls, value):
        if isinstance(value, str):
            for member in cls:
                if member.value.lower() == value.lower():
                    return member
        raise ValueError(f"Unknown method {value!r}; valid methods are {', '.join(m.value for m in cls)}.")

    def default_solver(self):
        return L2NNLS() if self is SDMethod.MFOD else DRL()

    @property
    def inner_shell_weight(self) -> float:
        return 0.2 if self is SDMethod.GRL else 1.0

    @property
    def _fraction_tolerance(self) -> float:
        return FRACTION_TOL if self is SDMethod.GRL else 1e-7

    def _check_rfs(self, rfs) -> None:
        n_aniso = sum(1 for rf in rfs if not isinstance(rf, IsotropicRF))
        if self is SDMethod.GRL and n_aniso != 1:
            raise ValueError(f"{self} takes exactly one anisotropic response function, got {n_aniso}.")
        if self is SDMethod.MFOD and n_aniso < 1:
            raise ValueError(f"{self} takes at least one anisotropic response function.")
