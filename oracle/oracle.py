"""ORACLE — test infrastructure only.

ctypes bindings of the FP64 CPU restatement in fits.cpp (liblarmor_oracle.so). Only the tests,
the smoke check and bench.py's CPU-baseline leg import this module; the product path
(larmor_b200) never does.

Each function mirrors the reference call it restates:
    fit_log_signal     larmor._core.fit_log_signal   cpp/src/python/dwi.cpp:42
    lsi_design         larmor._core.LsiDesign        cpp/src/sd/lsi.cpp:75
    fit_lsi            larmor._core.fit_lsi          cpp/src/python/sd.cpp:370
    nnls               larmor._core.lsqnonneg        cpp/src/sd/nnls.cpp:332
    ridge_nnls         FodSolver.l2nnls + fit_single_tissue  cpp/src/sd/solver.cpp:422
    fit_multi_tissue   larmor._core.fit_multi_tissue cpp/src/python/sd.cpp:310
    sh_derivatives     larmor._core.sh_derivatives   cpp/src/python/sh.cpp:69
    climb              larmor._core.climb            cpp/src/python/sh.cpp:84
    peaks_chunk        larmor._core.peaks_chunk      cpp/src/python/sh.cpp:112
    fit_csd            larmor._core.fit_csd          cpp/src/python/sd.cpp:171
    drl                FodSolver.drl + fit_single_tissue  cpp/src/sd/solver.cpp:9, drl.cpp:39
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liblarmor_oracle.so"

_i64 = ctypes.c_int64
_dbl = ctypes.c_double
_ptr = ctypes.c_void_p

_lib: ctypes.CDLL | None = None


def build() -> Path:
    """Builds liblarmor_oracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        _lib.oracle_last_error.restype = ctypes.c_char_p
        _lib.oracle_median.restype = _dbl
        _lib.oracle_median.argtypes = [_ptr, _i64]
    return _lib


def _p(a: np.ndarray | None) -> ctypes.c_void_p:
    return ctypes.c_void_p(None if a is None else a.ctypes.data)


def _check(code: int) -> None:
    if code != 0:
        raise ValueError(lib().oracle_last_error().decode())


def _c64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def default_threads() -> int:
    return os.cpu_count() or 1


def fit_log_signal(x, g, log_s, weighted, max_iter=20, tol=1e-6, n_threads=1, iterations=False):
    """Parameters (v, p), broke (v,) [, IRLS iterations (v,)] of every row of log_s (v, n)."""
    x, log_s = _c64(x), _c64(log_s)
    n, p = x.shape
    g = np.zeros((0, p)) if g is None else _c64(g)
    v = log_s.shape[0]
    params = np.empty((v, p))
    broke = np.zeros(v, np.uint8)
    iters = np.zeros(v, np.int32)
    _check(lib().oracle_fit_log_signal(
        _p(x), _i64(n), _i64(p), _p(g), _i64(g.shape[0]), _p(log_s), _i64(v), int(bool(weighted)),
        _i64(max_iter), _dbl(tol), int(n_threads), _p(params), _p(broke), _p(iters)))
    if iterations:
        return params, broke.astype(bool), iters
    return params, broke.astype(bool)


def log_design(x):
    """Column scales (p,) and the pseudo-inverse (p, n) of the scaled design."""
    x = _c64(x)
    n, p = x.shape
    scales, pinv = np.empty(p), np.empty((p, n))
    _check(lib().oracle_log_design(_p(x), _i64(n), _i64(p), _p(scales), _p(pinv)))
    return scales, pinv


def lsi_design(a, g, ridge):
    """The prepared LSI problem: dict of q_t, back, e, gram, abs_sums."""
    a, g = _c64(a), _c64(g)
    m, n = a.shape
    k = g.shape[0]
    out = dict(q_t=np.empty((n, m)), back=np.empty((n, n)), e=np.empty((k, n)),
               gram=np.empty((k, k)), abs_sums=np.empty(k))
    _check(lib().oracle_lsi_design(_p(a), _i64(m), _i64(n), _p(g), _i64(k), _dbl(ridge),
                                   *(_p(out[key]) for key in ("q_t", "back", "e", "gram", "abs_sums"))))
    return out


def fit_lsi(a, g, ridge, signals, only_qr=False, n_threads=1, details=False):
    """Solutions (v, n) and converged (v,) [, status, outer steps, active (v, k)]."""
    a, g, signals = _c64(a), _c64(g), _c64(signals)
    m, n = a.shape
    k = g.shape[0]
    v = signals.shape[0]
    x = np.empty((v, n))
    conv = np.zeros(v, np.uint8)
    status = np.zeros(v, np.int32)
    outer = np.zeros(v, np.int32)
    active = np.zeros((v, k), np.uint8) if details else None
    _check(lib().oracle_fit_lsi(_p(a), _i64(m), _i64(n), _p(g), _i64(k), _dbl(ridge), _p(signals),
                                _i64(v), int(bool(only_qr)), int(n_threads), _p(x), _p(conv),
                                _p(status), _p(outer), _p(active)))
    if details:
        return x, conv.astype(bool), status, outer, active.astype(bool)
    return x, conv.astype(bool)


def nnls(c, d, tol=None, max_inner=None):
    """x (cols,) and converged of min ||c x - d||, x >= 0."""
    c, d = _c64(c), _c64(d)
    rows, cols = c.shape
    x = np.empty(cols)
    conv = np.zeros(1, np.uint8)
    _check(lib().oracle_nnls(_p(c), _i64(rows), _i64(cols), _p(d), _dbl(-1.0 if tol is None else tol),
                             _i64(-1 if max_inner is None else max_inner), _p(x), _p(conv)))
    return x, bool(conv[0])


def ridge_nnls(k, ridge, tol_x, signals, n_threads=1):
    """FODs (v, c) of min ||k f - s||^2 + ridge^2 ||f||^2, f >= 0, per row of signals."""
    k, signals = _c64(k), _c64(signals)
    m, c = k.shape
    v = signals.shape[0]
    out = np.empty((v, c))
    _check(lib().oracle_ridge_nnls(_p(k), _i64(m), _i64(c), _dbl(ridge), _dbl(tol_x), _p(signals),
                                   _i64(v), int(n_threads), _p(out)))
    return out


def fit_multi_tissue(signals, weights, lr, hr, lr_ridge=0.0, hr_ridge=0.1, tol_x=1e-6,
                     max_rounds=50, fraction_tol=1e-7, final_tol=1e-2, n_threads=1, rounds=False,
                     lr_drl=None, hr_drl=None):
    """HR FODs (v, ca_hr) and fractions (v, n_blocks + ci) of the multi-tissue fit.

    lr and hr are dicts with k_aniso (m, ca), k_iso (m, ci), w_k_iso, w_k_aniso and, for hr,
    blocks [(start, stop), ...]. lr_drl / hr_drl, dicts of nu, n_iter and init, make that
    stage's FOD solve damped Richardson-Lucy on w_k_aniso (GRL) instead of the ridge NNLS.
    """
    signals, weights = _c64(signals), _c64(weights)
    v, m = signals.shape
    la, ha = (_c64(lr["k_aniso"]), _c64(hr["k_aniso"]))
    ci = lr["k_iso"].shape[1]
    blocks = np.ascontiguousarray(np.array(hr["blocks"], dtype=np.int64).reshape(-1))
    nb = len(hr["blocks"])
    fods = np.empty((v, ha.shape[1]))
    fr = np.empty((v, nb + ci))
    rd = np.zeros(v, np.int32)
    keep = [_c64(lr[key]) for key in ("k_iso", "w_k_iso", "w_k_aniso")] + \
           [_c64(hr[key]) for key in ("k_iso", "w_k_iso", "w_k_aniso")]

    def drl_args(settings, w_aniso):
        if settings is None:
            return [None, None, _dbl(0.0), _i64(0), _dbl(0.0)]
        k_t, gram = _c64(w_aniso.T), _c64(w_aniso.T @ w_aniso)
        keep.extend([k_t, gram])
        return [_p(k_t), _p(gram), _dbl(settings["nu"]), _i64(settings["n_iter"]), _dbl(settings["init"])]

    extra = drl_args(lr_drl, keep[2]) + drl_args(hr_drl, keep[5])
    _check(lib().oracle_fit_multi_tissue(
        _p(signals), _i64(v), _i64(m), _p(weights),
        _p(la), _i64(la.shape[1]), _p(keep[0]), _p(keep[1]), _p(keep[2]), _dbl(lr_ridge), _dbl(tol_x),
        _p(ha), _i64(ha.shape[1]), _p(keep[3]), _p(keep[4]), _p(keep[5]), _dbl(hr_ridge), _dbl(tol_x),
        _i64(ci), _p(blocks), _i64(nb), _i64(max_rounds), _dbl(fraction_tol), _dbl(final_tol),
        int(n_threads), _p(fods), _p(fr), _p(rd), *extra))
    if rounds:
        return fods, fr, rd
    return fods, fr


def median(values) -> float:
    values = _c64(values)
    return float(lib().oracle_median(_p(values), _i64(len(values))))


# ---- FOD peaks (peaks.cpp) ---------------------------------------------------------------


def sh_derivatives(sh, lmax, theta, phi, full=False) -> tuple[float, ...]:
    """larmor._core.sh_derivatives (cpp/src/python/sh.cpp:69-82)."""
    sh = _c64(sh)
    out = np.empty(6)
    lib().oracle_sh_derivatives(_p(sh), _i64(lmax), int(full), _dbl(theta), _dbl(phi), _p(out))
    return tuple(float(x) for x in out)


def climb(sh, lmax, start, max_iters=50, tol=1e-4, max_step=0.2, full=False):
    """larmor._core.climb (cpp/src/python/sh.cpp:84-108): (direction (3,), amplitude), NaN when
    the climb does not stop within max_iters."""
    sh = _c64(sh)
    start = _c64(start)
    d = np.empty(3)
    a = np.empty(1)
    lib().oracle_climb(_p(sh), _i64(lmax), int(full), _p(start), _i64(max_iters), _dbl(tol), _dbl(max_step),
                       _p(d), _p(a))
    return d, float(a[0])


def peaks_chunk(coeffs, lmax, on_sphere, vertices, neighbours, n_peaks, relative_threshold, threshold,
                n_threads=1, full=False):
    """larmor._core.peaks_chunk (cpp/src/python/sh.cpp:112-176): directions (n, n_peaks, 3) and
    amplitudes (n, n_peaks). The arguments are assumed valid."""
    coeffs = _c64(coeffs)
    on_sphere = _c64(on_sphere)
    vertices = _c64(vertices)
    neighbours = np.ascontiguousarray(neighbours, dtype=np.int64)
    n = coeffs.shape[0]
    dirs = np.empty((n, n_peaks, 3))
    amps = np.empty((n, n_peaks))
    lib().oracle_peaks_chunk(_p(coeffs), _i64(n), _i64(coeffs.shape[1]), _i64(lmax), int(full), _p(on_sphere),
                             _p(vertices), _p(neighbours), _i64(len(vertices)), _i64(n_peaks),
                             _dbl(relative_threshold), _dbl(threshold), _i64(n_threads), _p(dirs), _p(amps))
    return dirs, amps


# ---- single-shell CSD (csd.cpp) ------------------------------------------------------------


def fit_csd(signals, initial, forward, constraint, norm_weight, threshold, max_iter, n_threads=1):
    """larmor._core.fit_csd (cpp/src/python/sd.cpp:171-209): FODs (n, c) and converged (n,).
    The arguments are assumed valid."""
    signals, initial, forward, constraint = (_c64(a) for a in (signals, initial, forward, constraint))
    n, c = signals.shape[0], forward.shape[1]
    fods = np.empty((n, c))
    conv = np.empty(n, dtype=np.uint8)
    lib().oracle_fit_csd(_p(signals), _i64(n), _i64(signals.shape[1]), _p(initial), _i64(initial.shape[0]),
                         _p(forward), _i64(c), _p(constraint), _i64(constraint.shape[0]), _dbl(norm_weight),
                         _dbl(threshold), _i64(max_iter), _i64(n_threads), _p(fods), _p(conv))
    return fods, conv.astype(bool)


# ---- damped Richardson-Lucy (drl.cpp) ----------------------------------------------------


def drl(signals, k_t, k_t_k, nu, n_iter, init, n_threads=1):
    """FodSolver.drl(k_t, k_t_k, nu, n_iter, init) + fit_single_tissue (cpp/src/sd/solver.cpp:9-12,
    cpp/src/sd/drl.cpp:39-100): the FODs (v, c). The arguments are assumed valid."""
    signals, k_t, k_t_k = _c64(signals), _c64(k_t), _c64(k_t_k)
    v, c = signals.shape[0], k_t.shape[0]
    fods = np.empty((v, c))
    lib().oracle_drl(_p(signals), _i64(v), _i64(signals.shape[1]), _p(k_t), _p(k_t_k), _i64(c), _dbl(nu),
                     _i64(n_iter), _dbl(init), _i64(n_threads), _p(fods))
    return fods
