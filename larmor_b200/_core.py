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


class _Transfers:
    """Copies between the caller's (pageable) numpy arrays and the device through two reusable
    page-locked buffers of CHUNK bytes: while the DMA engine moves one chunk, host threads copy
    the next one into (or the previous one out of) the other buffer, so a large array crosses
    at close to the link's rate instead of through the driver's pageable staging. The buffers
    are allocated once per process and kept; the copies run on the current stream."""

    CHUNK = 32 << 20
    THREADS = 8

    def __init__(self) -> None:
        import threading

        self.buffers = None
        self.events = [None, None]
        self.pool = None
        self.lock = threading.Lock()

    def _setup(self, torch):
        if self.buffers is None:
            from concurrent.futures import ThreadPoolExecutor

            self.buffers = [torch.empty(self.CHUNK, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
            self.views = [b.numpy() for b in self.buffers]
            self.pool = ThreadPoolExecutor(self.THREADS, thread_name_prefix="larmor-copy")

    def _host_copy(self, dst: np.ndarray, src: np.ndarray) -> None:
        """dst[:] = src for flat uint8 views, split over the host threads (numpy releases the GIL
        while it copies)."""
        n = len(src)
        if n < (4 << 20):
            dst[:] = src
            return
        step = -(-n // self.THREADS)
        parts = [(i, min(i + step, n)) for i in range(0, n, step)]
        for f in [self.pool.submit(np.copyto, dst[a:b], src[a:b]) for a, b in parts]:
            f.result()

    def prefault(self, torch, arrays) -> None:
        """Writes zeros over newly allocated host arrays on the copy threads, so that their pages
        are mapped before the copies from the device need them (a first touch costs more than the
        copy itself)."""
        self._setup(torch)
        jobs = []
        for arr in arrays:
            flat = arr.reshape(-1).view(np.uint8)
            step = max(1 << 22, -(-len(flat) // self.THREADS))
            jobs += [self.pool.submit(flat[a:a + step].fill, 0) for a in range(0, len(flat), step)]
        for f in jobs:
            f.result()

    def _wait(self, k: int) -> None:
        if self.events[k] is not None:
            self.events[k].synchronize()
            self.events[k] = None

    def upload(self, torch, a: np.ndarray, dev):
        """A new C-contiguous device tensor with the contents of the host array a."""
        out = torch.empty(a.shape, dtype=getattr(torch, a.dtype.name), device=dev)
        return self.upload_into(torch, a, out)

    def upload_into(self, torch, a: np.ndarray, out):
        """Copies the host array a into the contiguous device tensor out of the same size, on the
        current stream; returns out."""
        if a.nbytes < (1 << 20):
            out.copy_(torch.from_numpy(np.ascontiguousarray(a)))
            return out
        with self.lock:
            return self._upload(torch, a, out)

    def _upload(self, torch, a, out):
        self._setup(torch)
        src = np.ascontiguousarray(a).reshape(-1).view(np.uint8)
        dst = out.view(-1).view(torch.uint8)
        stream = torch.cuda.current_stream()
        for i, start in enumerate(range(0, len(src), self.CHUNK)):
            k = i & 1
            stop = min(start + self.CHUNK, len(src))
            self._wait(k)  # the buffer's previous DMA has finished
            self._host_copy(self.views[k][:stop - start], src[start:stop])
            dst[start:stop].copy_(self.buffers[k][:stop - start], non_blocking=True)
            self.events[k] = torch.cuda.Event()
            self.events[k].record(stream)
        return out

    def download(self, torch, t) -> np.ndarray:
        """A new numpy array with the contents of the device tensor t (waits for t's stream)."""
        t = t.contiguous()
        out = np.empty(tuple(t.shape), dtype=np.dtype(str(t.dtype).replace("torch.", "")))
        return self.download_into(torch, t, out)

    def download_into(self, torch, t, out: np.ndarray) -> np.ndarray:
        """Copies the contiguous device tensor t into the C-contiguous host array out of the same
        size, through the current stream (waits for the copies); returns out."""
        if out.nbytes < (1 << 20):
            out[...] = t.cpu().numpy()
            return out
        with self.lock:
            return self._download(torch, t, out)

    def _download(self, torch, t, out):
        nbytes = out.nbytes
        self._setup(torch)
        src = t.view(-1).view(torch.uint8)
        dst = out.reshape(-1).view(np.uint8)
        stream = torch.cuda.current_stream()
        pending = None
        for i, start in enumerate(range(0, nbytes, self.CHUNK)):
            k = i & 1
            stop = min(start + self.CHUNK, nbytes)
            self._wait(k)
            self.buffers[k][:stop - start].copy_(src[start:stop], non_blocking=True)
            self.events[k] = torch.cuda.Event()
            self.events[k].record(stream)
            if pending is not None:  # the previous chunk, while this one moves
                pk, pa, pb = pending
                self._wait(pk)
                self._host_copy(dst[pa:pb], self.views[pk][:pb - pa])
            pending = (k, start, stop)
        pk, pa, pb = pending
        self._wait(pk)
        self._host_copy(dst[pa:pb], self.views[pk][:pb - pa])
        return out


_transfers = _Transfers()


def _on_device(torch, a, dev):
    """A C-contiguous device tensor of a host array, or the device tensor itself."""
    if isinstance(a, np.ndarray):
        return _transfers.upload(torch, a, dev)
    return a.contiguous()


def _to_host(t) -> np.ndarray:
    """A new numpy array of a device tensor, copied through the page-locked buffers."""
    return _transfers.download(_torch(), t)


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

    def violators(self) -> int:
        """Voxels of the last constrained fit on this design that took the constrained re-fit
        (read after that fit's stream has finished)."""
        n = ctypes.c_int64(0)
        _lib.check(_lib.lib().lar_log_design_violators(self._handle, ctypes.byref(n)))
        return n.value

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
        ls = _on_device(torch, log_s, dev)
        fit_log_signal_device(design, ls, bool(weighted), int(max_iter), float(tol), params, broke)
    return _to_host(params), _to_host(broke).astype(bool)


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
        s = _on_device(torch, signals, dev)
        fit_lsi_device(design, s, x, conv)
    return _to_host(x), _to_host(conv).astype(bool)


def fit_lsi_device(design: LsiDesign, signals, x, converged, status=None, outer=None, active=None,
                   only_qr: bool = False) -> None:
    """The device-resident fit_lsi: torch CUDA tensors in and out; status (0 Cholesky path,
    1 QR fallback, 2 no constraint active), outer steps and active-constraint flags (v, k) are
    optional diagnostics."""
    torch = _torch()
    _lib.check(_lib.lib().lar_fit_lsi(
        design.handle, _lib.ptr(signals), signals.shape[0], int(only_qr), _lib.ptr(x), _lib.ptr(converged),
        _lib.ptr(status), _lib.ptr(outer), _lib.ptr(active), _stream(torch)))


def fit_lsi_plain_fp32_device(design: LsiDesign, signals, x, status=None) -> None:
    """The plain single-precision LSI fit, the comparison baseline of fit_lsi_device: float32
    signals (v, m) in, float32 solutions (v, n) out (torch CUDA tensors); status (v,) uint8: 0
    converged, 1 factor failed, 2 f = 0, 3 step limit (lar_fit_lsi_plain_fp32)."""
    torch = _torch()
    _lib.check(_lib.lib().lar_fit_lsi_plain_fp32(
        design.handle, _lib.ptr(signals), signals.shape[0], _lib.ptr(x), _lib.ptr(status), _stream(torch)))


class _Handle:
    """Owns a C-ABI handle and destroys it with the given function."""

    _destroy = ""

    def __init__(self) -> None:
        self._handle = ctypes.c_void_p()

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._handle

    def __del__(self) -> None:
        handle = getattr(self, "_handle", None)
        if handle is not None and handle.value:
            try:
                getattr(_lib.lib(), self._destroy)(handle)
            except Exception:
                pass


class FodSolver(_Handle):
    """An FOD solver with the matrices it needs from one kernel, copied to the device
    (cpp/src/python/sd.cpp:399-438): the L2NNLS method (mFOD's) and damped Richardson-Lucy (dRL,
    single-tissue fits only)."""

    _destroy = "lar_fod_solver_destroy"

    @staticmethod
    def l2nnls(k, reg, tol_x) -> "FodSolver":
        """Non-negative least squares with a ridge penalty: each voxel's FOD f minimises
        ||k f - s||^2 + reg^2 ||f||^2 with f >= 0; a coefficient enters only when its gradient
        exceeds tol_x.

        Raises:
            TypeError: If k is not a float64 numpy array.
            ValueError: If reg is negative or tol_x is not positive.
        """
        k = _array(k, "k", 2)
        if not reg >= 0.0:
            raise ValueError("reg must be at least 0")
        if not tol_x > 0.0:
            raise ValueError("tol_x must be positive")
        solver = FodSolver()
        solver.n_meas, solver.n_dirs = k.shape
        _lib.check(_lib.lib().lar_l2nnls_create(_lib.ptr(k), k.shape[0], k.shape[1], float(reg), float(tol_x),
                                                ctypes.byref(solver._handle)))
        return solver

    @staticmethod
    def drl(k_t, k_t_k, nu, n_iter, init) -> "FodSolver":
        """Damped Richardson-Lucy (cpp/src/python/sd.cpp:127-145): k_t is K^T (c, m), k_t_k is
        K^T K (c, c); amplitudes below nu have their updates damped; at most n_iter iterations
        per voxel, every amplitude started at init. fit_single_tissue and fit_multi_tissue (GRL) run
        it on the device (lar_drl_create).

        Raises:
            TypeError: If k_t or k_t_k is not a float64 numpy array.
            ValueError: If the shapes do not match, n_iter is negative, or the solver has more
                than 640 directions.
        """
        for name, a in (("k_t", k_t), ("k_t_k", k_t_k)):
            if not isinstance(a, np.ndarray) or a.dtype != np.float64:
                got = type(a).__name__ if not isinstance(a, np.ndarray) else str(a.dtype)
                raise TypeError(f"{name} must be a float64 numpy array, got {got}")
            if a.ndim != 2:
                raise ValueError(f"{name} must have 2 dimensions, got shape {a.shape}")
        k_t, k_t_k = np.ascontiguousarray(k_t), np.ascontiguousarray(k_t_k)
        c, m = k_t.shape
        if k_t_k.shape != (c, c):
            raise ValueError(f"shapes do not match: k_t ({c}, {m}), k_t_k ({k_t_k.shape[0]}, {k_t_k.shape[1]})")
        if n_iter < 0:
            raise ValueError("n_iter must be at least 0")
        solver = FodSolver()
        solver.n_meas, solver.n_dirs = m, c
        _lib.check(_lib.lib().lar_drl_create(_lib.ptr(k_t), _lib.ptr(k_t_k), c, m, float(nu), int(n_iter),
                                             float(init), ctypes.byref(solver._handle)))
        return solver

    def set_precision(self, precision: str) -> "FodSolver":
        """The arithmetic of a dRL solver's fits: "fp64" (the default, the reference's) or
        "tf32x3" (65 to 320 directions: each iteration's product on the tcgen05 tensor cores as
        three TF32 products, FP32 amplitudes; FODs within 1e-4 of the voxel's largest amplitude
        of the FP64 fit); lar_drl_set_precision.

        Raises:
            ValueError: If the solver is not a dRL solver, or tf32x3 does not take its size.
        """
        codes = {"fp64": _lib.LAR_FP64, "tf32x3": _lib.LAR_TF32X3}
        if precision not in codes:
            raise ValueError(f"precision must be one of {', '.join(codes)}, got {precision!r}")
        _lib.check(_lib.lib().lar_drl_set_precision(self._handle, codes[precision]))
        self.precision = precision
        return self

    def check_errors(self) -> None:
        """Raises RuntimeError when a tensor-core fit of this solver stopped at a bounded wait
        (lar_drl_errors)."""
        flag = ctypes.c_int(0)
        _lib.check(_lib.lib().lar_drl_errors(self._handle, ctypes.byref(flag)))
        if flag.value:
            raise RuntimeError("a tensor-core dRL fit stopped at a bounded wait; its FODs are not valid")

    @staticmethod
    def lasso(*_args, **_kwargs):
        raise NotImplementedError("the elastic-net solver is not part of larmor_b200")

    @property
    def n_unconverged(self) -> int:
        return 0


class DeconvKernel(_Handle):
    """One resolution of a multi-tissue kernel, copied to the device
    (cpp/src/python/sd.cpp:260-292)."""

    _destroy = "lar_deconv_kernel_destroy"

    def __init__(self, k_aniso, k_iso, w_k_iso, aniso_blocks) -> None:
        super().__init__()
        k_aniso = _array(k_aniso, "k_aniso", 2)
        m, ca = k_aniso.shape
        if k_iso is None:
            k_iso = np.zeros((m, 0))
            w_k_iso = np.zeros((m, 0))
        k_iso = _array(k_iso, "k_iso", 2)
        w_k_iso = _array(w_k_iso, "w_k_iso", 2)
        if k_iso.shape[0] != m or w_k_iso.shape != k_iso.shape:
            raise ValueError(f"k_aniso {k_aniso.shape}, k_iso {k_iso.shape} and w_k_iso {w_k_iso.shape} "
                             "do not match")
        blocks = np.ascontiguousarray(np.array(list(aniso_blocks), dtype=np.int64).reshape(-1, 2))
        self.m, self.ca, self.ci, self.nb = m, ca, k_iso.shape[1], len(blocks)
        _lib.check(_lib.lib().lar_deconv_kernel_create(
            _lib.ptr(k_aniso), m, ca, _lib.ptr(k_iso if k_iso.size else None),
            _lib.ptr(w_k_iso if w_k_iso.size else None), k_iso.shape[1], _lib.ptr(blocks), len(blocks),
            ctypes.byref(self._handle)))


def fit_multi_tissue(signals, weights, lr, lr_solver, hr, hr_solver, max_outer, fraction_tol, final_tol_x,
                     n_threads):
    """Fits the FODs and tissue fractions of every row of signals (n, m); the shell weights
    (m,) apply to the FOD fits only. Returns the high-resolution FODs (n, ca_hr) and the
    fractions (n, n_aniso_rfs + ci), summing to 1 (cpp/src/python/sd.cpp:310-358).

    Raises:
        TypeError: If signals or weights is not float64.
        ValueError: If signals is not C-contiguous, the shapes do not match, a solver does not
            match its kernel, or n_threads is 0.
    """
    signals = _array(signals, "signals", 2)
    weights = _array(weights, "weights", 1)
    if signals.shape[1] != hr.m or weights.shape[0] != hr.m or lr.m != hr.m:
        raise ValueError(f"signals {signals.shape}, weights {weights.shape[0]} and the kernels' {hr.m} "
                         "measurements do not match")
    _require_threads(n_threads)
    if max_outer < 0:
        raise ValueError("max_outer must be at least 0")
    if signals.shape[0] >= _PIECES * _PIECE_MIN:
        return _fit_multi_tissue_pipelined(signals, weights, lr, lr_solver, hr, hr_solver, max_outer, fraction_tol,
                                           final_tol_x)
    fods, fractions = _fit_multi_tissue_on_device(signals, weights, lr, lr_solver, hr, hr_solver, max_outer,
                                                  fraction_tol, final_tol_x)
    return _to_host(fods), _to_host(fractions)


# The drop-in multi-tissue call cuts a large volume into pieces of voxels (at least _PIECE_MIN
# voxels in all per piece count), so that one piece's upload and another's download overlap a
# third's fit: a small first piece (its upload is the wait before the first fit) and a smaller
# last one (its download is the wait after the last fit).
_PIECE_SHARES = (0.10, 0.30, 0.35, 0.25)
_PIECES = len(_PIECE_SHARES)
_PIECE_MIN = 32768
_copy_streams: dict = {}


def _fit_multi_tissue_pipelined(signals, weights, lr, lr_solver, hr, hr_solver, max_outer, fraction_tol,
                                final_tol_x):
    """fit_multi_tissue of checked host arrays, piece by piece: a piece's signals go up on one
    copy stream while the previous piece is fitted on the caller's stream (every round enqueued
    with its count read on the device, so the host never waits on a fit), and the results come
    down on a second copy stream once their piece is fitted. Each voxel's fit depends on its own
    signals only, so the results equal one call over the whole array."""
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    v, m = signals.shape
    nf = hr.nb + hr.ci
    fods = np.empty((v, hr.ca), dtype=np.float64)
    fractions = np.empty((v, nf), dtype=np.float64)
    d_sig = torch.empty((v, m), dtype=torch.float64, device=dev)
    d_fods = torch.empty((v, hr.ca), dtype=torch.float64, device=dev)
    d_fr = torch.empty((v, nf), dtype=torch.float64, device=dev)
    if dev.index not in _copy_streams:
        _copy_streams[dev.index] = (torch.cuda.Stream(dev), torch.cuda.Stream(dev))
    up, down = _copy_streams[dev.index]
    compute = torch.cuda.current_stream(dev)
    ends = np.rint(np.cumsum(_PIECE_SHARES) * v).astype(np.int64)
    ends[-1] = v
    starts = np.concatenate([[0], ends[:-1]])
    pieces = [(int(a), int(b)) for a, b in zip(starts, ends) if b > a]
    fitted = []
    up.wait_stream(compute)  # the device arrays were allocated on the caller's stream
    for a, b in pieces:
        with torch.cuda.stream(up):
            _transfers.upload_into(torch, signals[a:b], d_sig[a:b])
        compute.wait_stream(up)
        fit_multi_tissue_device(d_sig[a:b], weights, lr, lr_solver, hr, hr_solver, max_outer, fraction_tol,
                                final_tol_x, d_fods[a:b], d_fr[a:b], asynchronous=True)
        done = torch.cuda.Event()
        done.record(compute)
        fitted.append(done)
    # While the GPU fits, the output pages are mapped (fresh host memory faults on first touch).
    _transfers.prefault(torch, (fods, fractions))
    for (a, b), done in zip(pieces, fitted):
        down.wait_event(done)
        with torch.cuda.stream(down):
            _transfers.download_into(torch, d_fods[a:b], fods[a:b])
            _transfers.download_into(torch, d_fr[a:b], fractions[a:b])
    compute.wait_stream(down)
    return fods, fractions


def _fit_multi_tissue_on_device(signals, weights, lr, lr_solver, hr, hr_solver, max_outer, fraction_tol,
                                final_tol_x):
    """fit_multi_tissue of checked host arrays (or a float64 device tensor), the results left on
    the device (torch tensors)."""
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    v = signals.shape[0]
    fods = torch.empty((v, hr.ca), dtype=torch.float64, device=dev)
    fractions = torch.empty((v, hr.nb + hr.ci), dtype=torch.float64, device=dev)
    if v:
        s = _on_device(torch, signals, dev)
        fit_multi_tissue_device(s, weights, lr, lr_solver, hr, hr_solver, max_outer, fraction_tol, final_tol_x,
                                fods, fractions)
    return fods, fractions


def fit_multi_tissue_device(signals, weights, lr, lr_solver, hr, hr_solver, max_outer, fraction_tol,
                            final_tol_x, fods, fractions, rounds=None, status=None, asynchronous=False) -> None:
    """The device-resident fit_multi_tissue (torch CUDA tensors; weights a host array). With
    asynchronous, every round is enqueued with its voxel count read on the device, and the call
    returns without waiting for the GPU (lar_fit_multi_tissue_async)."""
    torch = _torch()
    weights = np.ascontiguousarray(weights, dtype=np.float64)
    entry = _lib.lib().lar_fit_multi_tissue_async if asynchronous else _lib.lib().lar_fit_multi_tissue
    _lib.check(entry(
        _lib.ptr(signals), signals.shape[0], _lib.ptr(weights), lr.handle, lr_solver.handle, hr.handle,
        hr_solver.handle, int(max_outer), float(fraction_tol), float(final_tol_x), _lib.ptr(fods),
        _lib.ptr(fractions), _lib.ptr(rounds), _lib.ptr(status), _stream(torch)))


def fit_multi_tissue_plain_fp32_device(signals, weights, lr, lr_solver, hr, hr_solver, max_outer, fraction_tol,
                                       final_tol_x, fods, fractions, rounds=None, status=None) -> None:
    """The plain single-precision fit of fit_multi_tissue_device, the comparison baseline: float32
    signals (v, m) in, float32 FODs (v, ca_hr) and fractions (v, nb + ci) out (torch CUDA
    tensors; weights a host array); lar_fit_multi_tissue_plain_fp32."""
    torch = _torch()
    weights = np.ascontiguousarray(weights, dtype=np.float64)
    _lib.check(_lib.lib().lar_fit_multi_tissue_plain_fp32(
        _lib.ptr(signals), signals.shape[0], _lib.ptr(weights), lr.handle, lr_solver.handle, hr.handle,
        hr_solver.handle, int(max_outer), float(fraction_tol), float(final_tol_x), _lib.ptr(fods),
        _lib.ptr(fractions), _lib.ptr(rounds), _lib.ptr(status), _stream(torch)))


def lsqnonneg(c, d, tol_x=None):
    """Solves one non-negative least-squares problem, min ||c x - d|| with x >= 0, on the device
    (cpp/src/python/sd.cpp:208-228): c is (m, n) and d (m,); a coefficient enters the solution
    only when its gradient exceeds tol_x, None using 10 * eps * norm(c, 1) * max(m, n).

    Raises:
        TypeError: If c or d is not a float64 numpy array.
        ValueError: If c is not C-contiguous, the shapes do not match, or c has more than 16
            columns.
    """
    c = _array(c, "c", 2)
    if not isinstance(d, np.ndarray) or d.dtype != np.float64:
        raise TypeError(f"d must be a float64 numpy array, got {getattr(d, 'dtype', type(d).__name__)}")
    if d.ndim != 1 or d.shape[0] != c.shape[0]:
        raise ValueError(f"c must be (m, n) and d (m,): got ({c.shape[0]}, {c.shape[1]}) and "
                         f"{d.shape[0] if d.ndim == 1 else d.shape}")
    m, n = c.shape
    if n > 16:
        raise ValueError(f"lsqnonneg takes at most 16 columns, got {n}")
    if n == 0:
        return np.zeros(0)
    if m == 0:
        raise ValueError("c must have at least one row")
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    dc = torch.from_numpy(c).to(dev)
    dd = torch.from_numpy(np.ascontiguousarray(d)).to(dev)
    x = torch.empty(n, dtype=torch.float64, device=dev)
    _lib.check(_lib.lib().lar_lsqnonneg(_lib.ptr(dc), m, n, _lib.ptr(dd), int(tol_x is None),
                                        0.0 if tol_x is None else float(tol_x), _lib.ptr(x), _stream(torch)))
    return x.cpu().numpy()


def fit_single_tissue(signals, solver: FodSolver, n_threads):
    """The FOD (n, c) of every row of signals (n, m) with one solver."""
    signals = _array(signals, "signals", 2)
    if signals.shape[1] != solver.n_meas:
        raise ValueError(f"signals {signals.shape} do not have the solver's {solver.n_meas} measurements")
    _require_threads(n_threads)
    return _to_host(_fit_single_tissue_on_device(signals, solver))


def _fit_single_tissue_on_device(signals, solver: FodSolver):
    """fit_single_tissue of a checked host array (or a float64 device tensor), the FODs left on the
    device (a torch tensor)."""
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    v = signals.shape[0]
    fods = torch.empty((v, solver.n_dirs), dtype=torch.float64, device=dev)
    if v:
        s = _on_device(torch, signals, dev)
        _lib.check(_lib.lib().lar_fit_single_tissue(_lib.ptr(s), v, solver.handle, _lib.ptr(fods), None,
                                                    _stream(torch)))
    return fods


def _row_stride(t) -> int:
    """The row stride of a 2D tensor with unit-stride rows; a one-row tensor's stride along the
    rows is arbitrary (numpy and torch keep 0 for a view like a[None]), so its row length."""
    return t.stride(0) if t.shape[0] > 1 else t.shape[1]


class ShProjector(_Handle):
    """The least-squares projector of amplitudes on a sphere grid onto an SH basis, scaled by
    the grid's density, on the device (the _to_sh step, src/larmor/sd/model.py:412-440)."""

    _destroy = "lar_sh_projector_destroy"

    def __init__(self, projector) -> None:
        super().__init__()
        p = _array(projector, "projector", 2)
        self.ncoef, self.ca = p.shape
        _lib.check(_lib.lib().lar_sh_projector_create(_lib.ptr(p), self.ncoef, self.ca, ctypes.byref(self._handle)))


def project_sh_device(projector: ShProjector, amplitudes, exact_integral: bool):
    """SH coefficients (v, ncoef) of device amplitudes (v, ca), a column slice of a row-major
    tensor allowed; a new device tensor."""
    torch = _torch()
    if (amplitudes.dim() != 2 or amplitudes.shape[1] != projector.ca
            or (amplitudes.shape[0] and amplitudes.stride(1) != 1)):
        raise ValueError(f"amplitudes {tuple(amplitudes.shape)} do not have the projector's {projector.ca} "
                         "directions in unit-stride rows")
    v = amplitudes.shape[0]
    out = torch.empty((v, projector.ncoef), dtype=torch.float64, device=amplitudes.device)
    if v:
        _lib.check(_lib.lib().lar_project_sh(projector.handle, _lib.ptr(amplitudes), v, _row_stride(amplitudes),
                                             int(bool(exact_integral)), _lib.ptr(out), projector.ncoef,
                                             _stream(torch)))
    return out


# ---- single-shell CSD (cpp/src/python/sd.cpp:171-209) -----------------------------------


class CsdProblem(_Handle):
    """The matrices of one shell's CSD fit on the device (lar_csd_create)."""

    _destroy = "lar_csd_destroy"

    def __init__(self, initial, forward, constraint, norm_weight, threshold, max_iter) -> None:
        super().__init__()
        self.c0, self.m = initial.shape
        self.c = forward.shape[1]
        self.k = constraint.shape[0]
        _lib.check(_lib.lib().lar_csd_create(_lib.ptr(initial), self.c0, self.m, _lib.ptr(forward), self.c,
                                             _lib.ptr(constraint), self.k, float(norm_weight), float(threshold),
                                             int(max_iter), ctypes.byref(self._handle)))

    @classmethod
    def cached(cls, initial, forward, constraint, norm_weight, threshold, max_iter) -> "CsdProblem":
        extra = np.array([norm_weight, threshold, max_iter], dtype=np.float64).tobytes() + b"csd"
        return _designs.get(_digest(initial, forward, constraint, extra=extra),
                            lambda: cls(initial, forward, constraint, norm_weight, threshold, max_iter))


def fit_csd_device(problem: CsdProblem, signals):
    """The FODs (v, c) and converged flags (v,) of float64 device signals (v, m), left on the
    device."""
    torch = _torch()
    v = signals.shape[0]
    fods = torch.empty((v, problem.c), dtype=torch.float64, device=signals.device)
    conv = torch.empty((v,), dtype=torch.uint8, device=signals.device)
    if v:
        _lib.check(_lib.lib().lar_fit_csd(problem.handle, _lib.ptr(signals), v, _lib.ptr(fods), _lib.ptr(conv),
                                          _stream(torch)))
    return fods, conv


def _shape2(rows: int, cols: int) -> str:
    return f"({rows}, {cols})"


def fit_csd(signals, initial, forward, constraint, norm_weight, threshold, max_iter, n_threads):
    """Fits every row of signals (n, m) by constrained spherical deconvolution
    (cpp/src/python/sd.cpp:171-209), on the device.

    initial (c0, m) gives the starting FOD's first c0 coefficients, forward (m, c) is the forward
    model M and constraint (k, c) the weighted SH basis on the constraint directions. Each solve
    minimises ||M f - s||^2 + norm_weight ||f||^2 plus the squared constraint rows where the FOD is
    below threshold, until that set of rows repeats or after max_iter solves. Returns the FODs
    (n, c) and whether each voxel's set repeated (n,).

    Raises:
        TypeError: If an array is not float64.
        ValueError: If signals is not C-contiguous, the shapes do not match, max_iter is negative
            or n_threads is 0.
    """
    signals = _array(signals, "signals", 2)
    mats = []
    for name, a in (("initial", initial), ("forward", forward), ("constraint", constraint)):
        if not isinstance(a, np.ndarray) or a.dtype != np.float64:
            got = type(a).__name__ if not isinstance(a, np.ndarray) else str(a.dtype)
            raise TypeError(f"{name} must be a float64 numpy array, got {got}")
        if a.ndim != 2:
            raise ValueError(f"{name} must have 2 dimensions, got shape {a.shape}")
        mats.append(np.ascontiguousarray(a))
    initial, forward, constraint = mats
    m, c = forward.shape
    if (signals.shape[1] != m or initial.shape[1] != m or initial.shape[0] > c or constraint.shape[1] != c):
        raise ValueError(f"shapes do not match: signals {_shape2(*signals.shape)}, initial {_shape2(*initial.shape)}, "
                         f"forward {_shape2(m, c)}, constraint {_shape2(*constraint.shape)}")
    if max_iter < 0:
        raise ValueError("max_iter must be at least 0")
    _require_threads(n_threads)
    torch = _torch()
    problem = CsdProblem.cached(initial, forward, constraint, norm_weight, threshold, max_iter)
    dev = torch.device("cuda", torch.cuda.current_device())
    s = _on_device(torch, signals, dev)
    fods, conv = fit_csd_device(problem, s)
    return _to_host(fods), _to_host(conv).astype(bool)


# ---- FOD peaks (cpp/src/python/sh.cpp) ---------------------------------------------------

MAX_LMAX = 20


def _check_lmax(lmax: int, full: bool, n_coeffs_given: int) -> None:
    """cpp/src/python/sh.cpp:40-53: lmax within 0..20, even unless full, matching the count."""
    if lmax < 0 or lmax > MAX_LMAX or (not full and lmax % 2 != 0):
        raise ValueError(f"lmax must be at most {MAX_LMAX}, and even unless full, got {lmax}")
    expected = (lmax + 1) ** 2 if full else (lmax + 1) * (lmax + 2) // 2
    if expected != n_coeffs_given:
        raise ValueError(f"lmax {lmax} has {expected} coefficients, got {n_coeffs_given}")


def _series(sh) -> np.ndarray:
    """A 1D float64 series of any strides, copied (the bindings' copy_series)."""
    if not isinstance(sh, np.ndarray) or sh.dtype != np.float64:
        got = type(sh).__name__ if not isinstance(sh, np.ndarray) else str(sh.dtype)
        raise TypeError(f"sh must be a float64 numpy array, got {got}")
    if sh.ndim != 1:
        raise ValueError(f"sh must have 1 dimension, got shape {sh.shape}")
    return np.ascontiguousarray(sh)


def sh_derivatives(sh, lmax: int, theta: float, phi: float, full: bool = False) -> tuple[float, ...]:
    """The amplitude f of a series and df/dtheta, df/dphi / sin theta, d2f/dtheta2,
    d2f/dtheta dphi / sin theta, d2f/dphi2 / sin^2 theta at (theta, phi)
    (cpp/src/python/sh.cpp:69-82), computed on the device.

    Raises:
        ValueError: If lmax is above 20, odd without full, or does not match sh.
    """
    series = _series(sh)
    _check_lmax(lmax, full, series.shape[0])
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    s = torch.from_numpy(series).to(dev)
    angles = torch.tensor([float(theta), float(phi)], dtype=torch.float64, device=dev)
    out = torch.empty(6, dtype=torch.float64, device=dev)
    _lib.check(_lib.lib().lar_sh_derivatives(_lib.ptr(s), 1, series.shape[0], lmax, int(bool(full)),
                                             _lib.ptr(angles), ctypes.c_void_p(angles.data_ptr() + 8),
                                             _lib.ptr(out), _stream(torch)))
    return tuple(float(x) for x in out.cpu().numpy())


def climb(sh, lmax: int, start, max_iters: int = 50, tol: float = 1e-4, max_step: float = 0.2,
          full: bool = False) -> tuple[np.ndarray, float]:
    """Climbs from start to the peak whose basin it lies in (cpp/src/python/sh.cpp:84-108),
    on the device: the peak's direction (3,) and amplitude, both NaN if the climb does not
    converge within max_iters.

    Raises:
        ValueError: If lmax is above 20, odd without full, or does not match sh, or max_iters
            is negative.
    """
    series = _series(sh)
    _check_lmax(lmax, full, series.shape[0])
    if max_iters < 0:
        raise ValueError("max_iters must be at least 0")
    st = np.asarray(start, dtype=np.float64).reshape(-1)
    if st.shape != (3,):
        raise ValueError(f"start must hold three numbers, got {st.shape[0]}")
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    s = torch.from_numpy(series).to(dev)
    d_start = torch.from_numpy(np.ascontiguousarray(st)).to(dev)
    dirs = torch.empty(3, dtype=torch.float64, device=dev)
    amps = torch.empty(1, dtype=torch.float64, device=dev)
    _lib.check(_lib.lib().lar_climb(_lib.ptr(s), 1, series.shape[0], lmax, int(bool(full)), _lib.ptr(d_start),
                                    int(max_iters), float(tol), float(max_step), _lib.ptr(dirs), _lib.ptr(amps),
                                    _stream(torch)))
    return dirs.cpu().numpy(), float(amps.cpu().numpy()[0])


class PeakSphere(_Handle):
    """A sphere for the peak search on the device: unit vertices (nv, 3) and the 6 neighbours of
    each (nv, 6), copied (the reference copies its sphere per call, cpp/src/python/sh.cpp:130-147).

    Raises:
        ValueError: If a neighbour index is outside the sphere.
    """

    _destroy = "lar_peak_sphere_destroy"

    def __init__(self, vertices, neighbours) -> None:
        super().__init__()
        v = np.ascontiguousarray(vertices, dtype=np.float64)
        nb = np.ascontiguousarray(neighbours, dtype=np.int64)
        self.nv = v.shape[0]
        _lib.check(_lib.lib().lar_peak_sphere_create(_lib.ptr(v), _lib.ptr(nb), self.nv,
                                                     ctypes.byref(self._handle)))

    @classmethod
    def cached(cls, vertices: np.ndarray, neighbours: np.ndarray) -> "PeakSphere":
        return _designs.get(_digest(vertices, neighbours, extra=b"peak-sphere"), lambda: cls(vertices, neighbours))


def find_peaks_device(sphere: PeakSphere, coeffs, lmax: int, full: bool, on_sphere, n_peaks: int,
                      relative_threshold: float, threshold: float):
    """The peaks of device series (n, C) from their device amplitudes on the sphere (n, nv):
    directions (n, n_peaks, 3) and amplitudes (n, n_peaks), new device tensors."""
    torch = _torch()
    n = coeffs.shape[0]
    if coeffs.dim() != 2 or on_sphere.dim() != 2 or (n and (coeffs.stride(1) != 1 or on_sphere.stride(1) != 1)):
        raise ValueError("coeffs and on_sphere must be 2D tensors with unit-stride rows")
    if on_sphere.shape[0] != n or on_sphere.shape[1] != sphere.nv:
        raise ValueError(f"on_sphere {tuple(on_sphere.shape)} does not have {n} voxels x {sphere.nv} vertices")
    _check_lmax(lmax, full, coeffs.shape[1])
    dirs = torch.empty((n, n_peaks, 3), dtype=torch.float64, device=coeffs.device)
    amps = torch.empty((n, n_peaks), dtype=torch.float64, device=coeffs.device)
    if n:
        _lib.check(_lib.lib().lar_find_peaks(
            sphere.handle, _lib.ptr(coeffs), n, _row_stride(coeffs), lmax, int(bool(full)), _lib.ptr(on_sphere),
            _row_stride(on_sphere), int(n_peaks), float(relative_threshold), float(threshold), _lib.ptr(dirs),
            _lib.ptr(amps), _stream(torch)))
    return dirs, amps


def _shape(a: np.ndarray) -> str:
    return "(" + ", ".join(str(x) for x in a.shape) + ")"


def peaks_chunk(coeffs, lmax: int, on_sphere, vertices, neighbours, n_peaks: int, relative_threshold: float,
                threshold: float, n_threads: int, full: bool = False) -> tuple[np.ndarray, np.ndarray]:
    """Finds the peaks of every voxel of a chunk (cpp/src/python/sh.cpp:112-198), on the device.

    coeffs is (n, C) in the tournier basis, with all degrees if full. on_sphere (n, V) holds the
    amplitudes at the vertices (V, 3), and neighbours (V, 6) the 6 neighbours of each vertex.
    Returns directions (n, n_peaks, 3) and amplitudes (n, n_peaks), largest first, with z >= 0
    unless full, and NaN where a voxel has fewer peaks.

    Raises:
        TypeError: If an array does not have the dtype the reference binds (float64; neighbours
            int64).
        ValueError: If lmax is above 20, odd without full or does not match C, the shapes do
            not match, a neighbour is outside the sphere, n_peaks or n_threads is 0.
    """
    coeffs = _array(coeffs, "coeffs", 2)
    on_sphere = _array(on_sphere, "on_sphere", 2)
    for name, a, dtype in (("vertices", vertices, np.float64), ("neighbours", neighbours, np.int64)):
        if not isinstance(a, np.ndarray) or a.dtype != dtype:
            got = type(a).__name__ if not isinstance(a, np.ndarray) else str(a.dtype)
            raise TypeError(f"{name} must be a {np.dtype(dtype)} numpy array, got {got}")
        if a.ndim != 2:
            raise ValueError(f"{name} must have 2 dimensions, got shape {a.shape}")
    _check_lmax(lmax, full, coeffs.shape[1])
    nv = vertices.shape[0]
    if (vertices.shape[1] != 3 or neighbours.shape[0] != nv or neighbours.shape[1] != 6
            or on_sphere.shape[0] != coeffs.shape[0] or on_sphere.shape[1] != nv):
        raise ValueError(f"shapes do not match: coeffs {_shape(coeffs)}, on_sphere {_shape(on_sphere)}, "
                         f"vertices {_shape(vertices)}, neighbours {_shape(neighbours)}")
    if nv and (neighbours.min() < 0 or neighbours.max() >= nv):
        raise ValueError("a neighbour index is outside the sphere")
    if n_peaks < 1:
        raise ValueError("n_peaks must be at least 1")
    _require_threads(n_threads)
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    sphere = PeakSphere.cached(np.ascontiguousarray(vertices), np.ascontiguousarray(neighbours))
    c = torch.from_numpy(coeffs).to(dev)
    o = torch.from_numpy(on_sphere).to(dev)
    dirs, amps = find_peaks_device(sphere, c, lmax, full, o, n_peaks, relative_threshold, threshold)
    return dirs.cpu().numpy(), amps.cpu().numpy()


# ---- launch accounting (benchmarks) ------------------------------------------------------

def launch_count() -> int:
    """Kernels the library has launched since it was loaded."""
    return int(_lib.lib().lar_launch_count())


def kernel_timing(enable: bool) -> None:
    """Turns per-kernel CUDA-event timing on or off (clearing the records either way)."""
    _lib.check(_lib.lib().lar_kernel_timing(int(bool(enable))))


def kernel_time(name: str) -> tuple[float, int]:
    """(total ms, launches) of the timed launches of one kernel; waits for their events."""
    ms, n = ctypes.c_double(0.0), ctypes.c_int64(0)
    _lib.check(_lib.lib().lar_kernel_time(name.encode(), ctypes.byref(ms), ctypes.byref(n)))
    return ms.value, n.value
