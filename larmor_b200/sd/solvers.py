"""The FOD solvers (L2NNLS, dRL) and the multi-tissue fit (src/larmor/sd/solvers.py), on the GPU."""

from __future__ import annotations

from dataclasses import dataclass
from enum import Enum, auto
from math import isfinite

import numpy as np

from larmor_b200 import _core
from larmor_b200.sd.kernel import Kernel

# Maximum number of rounds of the multi-tissue loop.
MAX_ROUNDS = 50
# Default change in every fraction below which a voxel leaves the loop.
FRACTION_TOL = 1e-3
# In the final fraction fit, a tissue worth less than about this share of the signal gets 0.
FINAL_FRACTION_TOL_X = 1e-2


class Stage(Enum):
    SINGLE = auto()
    LOW_RES = auto()
    HIGH_RES = auto()


@dataclass(frozen=True, kw_only=True)
class L2NNLS:
    """NNLS with a ridge penalty reg (0 = plain NNLS), the mFOD method's solver; the loop's
    low-resolution solves use reg 0 (src/larmor/sd/solvers.py:151-210)."""

    reg: float = 0.1
    tol_x: float = 1e-6

    def __post_init__(self) -> None:
        if not isfinite(self.reg) or self.reg < 0:
            raise ValueError(f"reg must be a finite number >= 0, got {self.reg}")
        if not self.tol_x > 0:
            raise ValueError(f"tol_x must be positive, got {self.tol_x}")

    def _prepare(self, kernel: Kernel, bvals: np.ndarray, stage: Stage) -> _core.FodSolver:
        reg = 0.0 if stage is Stage.LOW_RES else self.reg
        return _core.FodSolver.l2nnls(np.ascontiguousarray(kernel.w_k_aniso), reg, self.tol_x)


# The near-zero start of a multi-tissue dRL solve (src/larmor/sd/solvers.py:21).
MULTI_TISSUE_DRL_INIT = 1e-6


def _rl_products(k: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """K^T and K^T K, the matrices of a Richardson-Lucy solve."""
    return np.ascontiguousarray(k.T), np.ascontiguousarray(k.T @ k)


def calibrate_drl_nu(kernel: Kernel, bvals: np.ndarray, target_adc: float = 0.7e-3, scale: float = 0.2,
                     n_iter: int = 200) -> float:
    """dRL's damping threshold nu for a kernel (src/larmor/sd/solvers.py:37-69): scale times the
    largest FOD amplitude an undamped deconvolution with the whole kernel gives for a purely
    isotropic tissue, exp(-b_max target_adc) on every measurement (run on the device)."""
    signal = np.full((1, len(bvals)), np.exp(-max(bvals) * target_adc))
    k_t, k_t_k = _rl_products(kernel.k)
    solver = _core.FodSolver.drl(k_t, k_t_k, nu=0.0, n_iter=n_iter, init=1.0 / kernel.k.shape[1])
    fake_fod = _core.fit_single_tissue(signal, solver, n_threads=1)
    return float(scale * np.max(fake_fod))


@dataclass(frozen=True, kw_only=True)
class DRL:
    """Damped Richardson-Lucy deconvolution, an FOD solver (src/larmor/sd/solvers.py:72-148):
    the FOD stays non-negative, and the updates of amplitudes below nu (nu_scale times the
    largest amplitude an undamped fit gives for an isotropic tissue of diffusivity target_adc) are
    damped. num_iter caps a single-tissue fit's iterations and hr_num_iter the final solve of a
    multi-tissue one. Both run on the device: a multi-tissue (GRL) fit solves each round's
    low-resolution FODs and the final high-resolution one by dRL, from MULTI_TISSUE_DRL_INIT,
    with one iteration fewer than asked. precision "fp64" keeps the reference's arithmetic;
    "tf32x3" runs the solves of 65 to 320 directions on the tensor cores (FodSolver.set_precision).

    Raises:
        ValueError: If an iteration count is below 1, target_adc or nu_scale is not a positive
            number, or precision is unknown.
    """

    num_iter: int = 200
    hr_num_iter: int = 600
    target_adc: float = 0.7e-3
    nu_scale: float = 0.2
    precision: str = "fp64"

    def __post_init__(self) -> None:
        if self.num_iter < 1 or self.hr_num_iter < 1:
            raise ValueError(f"num_iter and hr_num_iter must be at least 1, got {self.num_iter} and "
                             f"{self.hr_num_iter}")
        for name in ("target_adc", "nu_scale"):
            value = getattr(self, name)
            if not (np.isfinite(value) and value > 0):
                raise ValueError(f"{name} must be a positive number, got {value}")
        if self.precision not in ("fp64", "tf32x3"):
            raise ValueError(f"precision must be 'fp64' or 'tf32x3', got {self.precision!r}")

    def _solver(self, k_t, k_t_k, nu, n_iter, init) -> _core.FodSolver:
        solver = _core.FodSolver.drl(k_t, k_t_k, nu=nu, n_iter=n_iter, init=init)
        if self.precision != "fp64" and 64 < k_t.shape[0] <= 320:
            solver.set_precision(self.precision)
        return solver

    def _prepare(self, kernel: Kernel, bvals: np.ndarray, stage: Stage) -> _core.FodSolver:
        nu = calibrate_drl_nu(kernel, bvals, self.target_adc, self.nu_scale)
        k_t, k_t_k = _rl_products(kernel.w_k_aniso)
        if stage is Stage.SINGLE:
            return self._solver(k_t, k_t_k, nu, self.num_iter, 1.0 / kernel.w_k_aniso.shape[1])
        # A multi-tissue solve counts its near-zero start as the first iteration
        # (src/larmor/sd/solvers.py:144-148).
        n_iter = self.num_iter if stage is Stage.LOW_RES else self.hr_num_iter
        return self._solver(k_t, k_t_k, nu, n_iter - 1, MULTI_TISSUE_DRL_INIT)


# The FOD solvers SDModel takes (src/larmor/sd/solvers.py:296, without the elastic net, which
# this package does not include).
type SDSolver = DRL | L2NNLS


def _deconv_kernel(kernel: Kernel) -> _core.DeconvKernel:
    return _core.DeconvKernel(
        np.ascontiguousarray(kernel.k_aniso),
        None if kernel.k_iso is None else np.ascontiguousarray(kernel.k_iso),
        None if kernel.w_k_iso is None else np.ascontiguousarray(kernel.w_k_iso),
        [(b.start, b.stop) for b in kernel.aniso_blocks],
    )


def fit_single_tissue(signals, solver, n_threads):
    return _core.fit_single_tissue(np.ascontiguousarray(signals, dtype=np.float64), solver, n_threads=n_threads)


def fit_single_tissue_on_device(signals, solver):
    """fit_single_tissue with the FODs left on the device (a torch tensor); signals a host array
    or a float64 device tensor."""
    if isinstance(signals, np.ndarray):
        signals = _core._array(np.ascontiguousarray(signals, dtype=np.float64), "signals", 2)
    return _core._fit_single_tissue_on_device(signals, solver)


def fit_multi_tissue_on_device(signals, lr_kernel: Kernel, hr_kernel: Kernel, lr_solver, hr_solver,
                               fraction_tol: float = FRACTION_TOL):
    """fit_multi_tissue with the amplitudes and fractions left on the device (torch tensors);
    signals a host array or a float64 device tensor."""
    if isinstance(signals, np.ndarray):
        signals = np.ascontiguousarray(signals, dtype=np.float64)
    return _core._fit_multi_tissue_on_device(
        signals, np.ascontiguousarray(lr_kernel.weights, dtype=np.float64),
        _deconv_kernel(lr_kernel), lr_solver, _deconv_kernel(hr_kernel), hr_solver, MAX_ROUNDS, fraction_tol,
        FINAL_FRACTION_TOL_X)


def fit_multi_tissue(signals, lr_kernel: Kernel, hr_kernel: Kernel, lr_solver, hr_solver, n_threads: int = 1,
                     fraction_tol: float = FRACTION_TOL):
    """The high-resolution FOD amplitudes (n, ca_hr) and the fractions (n, n_rfs)
    (src/larmor/sd/solvers.py:329-373)."""
    return _core.fit_multi_tissue(
        np.ascontiguousarray(signals, dtype=np.float64),
        np.ascontiguousarray(lr_kernel.weights, dtype=np.float64),
        _deconv_kernel(lr_kernel), lr_solver, _deconv_kernel(hr_kernel), hr_solver,
        max_outer=MAX_ROUNDS, fraction_tol=fraction_tol, final_tol_x=FINAL_FRACTION_TOL_X, n_threads=n_threads)
