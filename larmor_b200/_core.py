"""Drop-in replacement of Larmor's compiled module `larmor._core` for the fitting hot path.

The functions here keep the names, arguments, return values and errors of the reference's
bindings (src/larmor/_core.pyi; cpp/src/python/dwi.cpp, cpp/src/python/sd.cpp): inputs are
C-contiguous float64 numpy arrays on the host (another dtype is a TypeError, a non-contiguous
array a ValueError), outputs are new numpy arrays. Underneath, each call copies its inputs to
the current CUDA device, runs the sm_100a kernels of liblarmor_b200.so through its C ABI, and
copies the results back. `n_threads` is accepted and checked for compatibility; the GPU
decides its own parallelism, and the per-voxel results do not depend on it.

Prepared designs are cached on the device by the content of their matrices, so a model that
fits many chunks of one volume uploads its design once.

There is no CPU fallback: without a CUDA device or the built library, every fit raises.
"""

from __future__ import annotations

import ctypes
import hashlib
from collections import OrderedDict

import numpy as np

from larmor_b200 import _lib

_CACHE_SIZE = 32


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError(
            "larmor_b200 runs on a CUDA device (B200, sm_100a); none is available and there "
            "is no CPU fallback"
        )
    return torch


def _stream(torch) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _array(a, name: str, ndim: int, dtype=np.float64) -> np.ndarray:
    """Checks a bound array as the reference's bindings do (.noconvert(), require_contiguous)."""
    if not isinstance(a, np.ndarray) or a.dtype != dtype:
        got = type(a).__name__ if not isinstance(a, np.ndarray) else str(a.dtype)
        raise TypeError(f"{name} must be a {np.dtype(dtype)} numpy array, got {got}")
    if a.ndim != ndim:
        raise ValueError(f"{name} must have {ndim} dimensions, got shape {a.shape}")
    if not a.flags.c_contiguous:
        raise ValueError(f"{name} must be C-contiguous")
    return a


def _require_threads(n_threads: int) -> None:
    if n_threads < 1:
        raise ValueError("n_threads must be at least 1")


def _digest(*arrays: np.ndarray, extra: bytes = b"") -> bytes:
    h = hashlib.blake2b(digest_size=20)
    for a in arrays:
        h.update(str(a.shape).encode())
        h.update(np.ascontiguousarray(a).tobytes())
    h.update(extra)
    return h.digest()


class _HandleCache:
    """A small LRU of prepared device designs keyed by the digest of their matrices."""

    def __init__(self, size: int) -> None:
        self.size = size
        self.entries: OrderedDict[bytes, object] = OrderedDict()

    def get(self, key: bytes, make):
        if key in self.entries:
            self.entries.move_to_end(key)
            return self.entries[key]
        value = make()
        self.entries[key] = value
        if len(self.entries) > self.size:
            self.entries.popitem(last=False)
        return value


_designs = _HandleCache(_CACHE_SIZE)


class LogDesign:
    """A log-signal design x (n, p) with constraints g (m, p), prepared on the device.

    Replaces make_log_signal_design (cpp/src/dwi/log_fit.cpp:220): unit-norm columns, the
    pseudo-inverse and the column-scaled constraints, computed once in FP64 and kept in device
    memory in FP64 and FP32.
    """

    def __init__(self, x: np.ndarray, g: np.ndarray) -> None:
        self.n, self.p = x.shape
        self.m = g.shape[0]
        self._handle = ctypes.c_void_p()
        lib = _lib.lib()
        _lib.check(lib.lar_log_design_create(
            _lib.ptr(x), self.n, self.p, _lib.ptr(g if g.size else None), self.m,
            ctypes.byref(self._handle)))

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._handle

    def __del__(self) -> None:
        handle = getattr(self, "_handle", None)
        if handle is not None and handle.value:
            try:
                _lib.lib().lar_log_design_destroy(handle)
            except Exception:  # interpreter shutdown
                pass

    @classmethod
    def cached(cls, x: np.ndarray, g: np.ndarray) -> LogDesign:
        x = np.ascontiguousarray(x, dtype=np.float64)
        g = np.ascontiguousarray(g, dtype=np.float64).reshape(-1, x.shape[1])
        return _designs.get(_digest(x, g, extra=b"log"), lambda: cls(x, g))


def fit_log_signal(x, g, log_s, weighted, max_iter, tol, n_threads):
    """Fits each row of log_s (v, n) by least squares on the design x (n, p).

    With weighted=True the fit is weighted by the predicted signal, iterated until no predicted
    log signal changes by more than tol or for max_iter weighted fits. A voxel whose solution
    has g @ p < 0 in some row of g (m, p) is fitted again subject to g @ p >= 0; m = 0 means no
    constraints.

    Returns the parameters (v, p) and whether each voxel broke a constraint (v,).

    Raises:
        TypeError: If an array is not float64.
        ValueError: If an array is not C-contiguous, the shapes do not match, max_iter is
            negative or n_threads is 0.
    """
    x = _array(x, "x", 2)
    g = _array(g, "g", 2)
    log_s = _array(log_s, "log_s", 2)
    n, p = x.shape
    if n < p or g.shape[1] != p or log_s.shape[1] != n:
        raise ValueError(
            f"x must be (n, p) with n >= p, g (m, p) and log_s (v, n): got x {x.shape}, "
            f"g {g.shape}, log_s {log_s.shape}"
        )
    if max_iter < 0:
        raise ValueError("max_iter must be at least 0")
    _require_threads(n_threads)
    torch = _torch()
    design = LogDesign.cached(x, g)
    v = log_s.shape[0]
    dev = torch.device("cuda", torch.cuda.current_device())
    params = torch.empty((v, p), dtype=torch.float64, device=dev)
    broke = torch.empty((v,), dtype=torch.uint8, device=dev)
    if v:
        ls = torch.from_numpy(log_s).to(dev)
        fit_log_signal_device(design, ls, bool(weighted), int(max_iter), float(tol), params, broke)
    return params.cpu().numpy(), broke.cpu().numpy().astype(bool)


def fit_log_signal_device(design: LogDesign, log_s, weighted: bool, max_iter: int, tol: float,
                          params, broke, iterations=None, precision: int = _lib.LAR_FP64) -> None:
    """The device-resident form of fit_log_signal: torch CUDA tensors in and out."""
    torch = _torch()
    _lib.check(_lib.lib().lar_fit_log_signal(
        design.handle, _lib.ptr(log_s), log_s.shape[0], int(weighted), int(max_iter), float(tol),
        int(precision), _lib.ptr(params), _lib.ptr(broke), _lib.ptr(iterations), _stream(torch)))


def fit_dti_maps_device(design: LogDesign, signals, floor, weighted: bool, maps, npd,
                        params=None, max_iter: int = 20, tol: float = 1e-6,
                        precision: int = _lib.LAR_FP64) -> None:
    """Floors, logs and fits float32 signals (v, n) and writes the 16 DTI maps (16, v)."""
    torch = _torch()
    _lib.check(_lib.lib().lar_fit_dti_maps(
        design.handle, _lib.ptr(signals), _lib.ptr(floor), signals.shape[0], int(weighted),
        int(max_iter), float(tol), int(precision), _lib.ptr(maps), _lib.ptr(npd), _lib.ptr(params),
        _stream(torch)))


class LsiDesign:
    """A least-squares problem with inequality constraints, prepared once for many voxels.

    Prepares min ||a x - s||^2 + ridge^2 ||x||^2 subject to g x >= 0, a (m, n), g (k, n), as
    cpp/src/sd/lsi.cpp:75-125 does (in FP64 on the host), and keeps it on the device.

    Raises:
        TypeError: If a or g is not a float64 numpy array.
        ValueError: If the shapes do not match, ridge is negative, or [a; ridge I] does not
            have full column rank.
    """

    def __init__(self, a, g, ridge) -> None:
        a = _array(a, "a", 2)
        g = _array(g, "g", 2)
        if g.shape[1] != a.shape[1]:
            raise ValueError(f"the constraints have {g.shape[1]} columns but the design has {a.shape[1]}")
        if not ridge >= 0.0:
            raise ValueError("the ridge must be at least 0")
        self.m, self.n = a.shape
        self.k = g.shape[0]
        self._handle = ctypes.c_void_p()
        _lib.check(_lib.lib().lar_lsi_design_create(_lib.ptr(a), self.m, self.n, _lib.ptr(g), self.k,
                                                    float(ridge), ctypes.byref(self._handle)))

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._handle

    def matrices(self) -> dict:
        """The prepared matrices q_t (n, m), back (n, n), e (k, n), gram (k, k), abs_sums (k,)."""
        out = dict(q_t=np.empty((self.n, self.m)), back=np.empty((self.n, self.n)),
                   e=np.empty((self.k, self.n)), gram=np.empty((self.k, self.k)), abs_sums=np.empty(self.k))
        _lib.check(_lib.lib().lar_lsi_design_matrices(
            self._handle, *(_lib.ptr(out[key]) for key in ("q_t", "back", "e", "gram", "abs_sums"))))
        return out

    def __del__(self) -> None:
        handle = getattr(self, "_handle", None)
        if handle is not None and handle.value:
            try:
                _lib.lib().lar_lsi_design_destroy(handle)
            except Exception:
                pass


def fit_lsi(signals, design: LsiDesign, n_threads):
    """Solves the constrained least-squares problem of every row of signals (v, m).

    Returns the solutions (v, n) and whether each voxel's NNLS converged (v,).

    Raises:
        TypeError: If signals is not a float64 numpy array.
        ValueError: If signals is not C-contiguous, does not have the design's number of
            measurements, or n_threads is 0.
    """
    signals = _array(signals, "signals", 2)
    if signals.shape[1] != design.m:
        raise ValueError(f"signals {signals.shape} do not have the design's {design.m} measurements")
    _require_threads(n_threads)
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    v = signals.shape[0]
    x = torch.empty((v, design.n), dtype=torch.float64, device=dev)
    conv = torch.empty((v,), dtype=torch.uint8, device=dev)
    if v:
        s = torch.from_numpy(signals).to(dev)
        fit_lsi_device(design, s, x, conv)
    return x.cpu().numpy(), conv.cpu().numpy().astype(bool)


def fit_lsi_device(design: LsiDesign, signals, x, converged, status=None, outer=None, active=None,
                   only_qr: bool = False) -> None:
    """The device-resident fit_lsi: torch CUDA tensors in and out; status (0 Cholesky path,
    1 QR fallback, 2 no constraint active), outer steps and active-constraint flags (v, k) are
    optional diagnostics."""
    torch = _torch()
    _lib.check(_lib.lib().lar_fit_lsi(
        design.handle, _lib.ptr(signals), signals.shape[0], int(only_qr), _lib.ptr(x), _lib.ptr(converged),
        _lib.ptr(status), _lib.ptr(outer), _lib.ptr(active), _stream(torch)))
