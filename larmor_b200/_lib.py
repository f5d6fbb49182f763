"""Loads liblarmor_b200.so and declares its C ABI (include/larmor_b200.h) for ctypes.

There is no CPU fallback: without the built library, or without a CUDA device, the fits raise.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "liblarmor_b200.so"

_c = ctypes
_p = _c.c_void_p
_i64 = _c.c_int64
_i32 = _c.c_int
_f64 = _c.c_double

# name: (restype, argtypes), in the order of include/larmor_b200.h.
SIGNATURES: dict[str, tuple] = {
    "lar_last_error": (_c.c_char_p, []),
    "lar_version": (_c.c_char_p, []),
    "lar_launch_count": (_i64, []),
    "lar_set_launch_setting": (_i32, [_c.c_char_p, _i64]),
    "lar_get_launch_setting": (_i32, [_c.c_char_p, _p]),
    "lar_kernel_timing": (_i32, [_i32]),
    "lar_kernel_time": (_i32, [_c.c_char_p, _p, _p]),
    "lar_log_design_create": (_i32, [_p, _i64, _i64, _p, _i64, _p]),
    "lar_log_design_destroy": (None, [_p]),
    "lar_log_design_violators": (_i32, [_p, _p]),
    "lar_fit_log_signal": (_i32, [_p, _p, _i64, _i32, _i64, _f64, _i32, _p, _p, _p, _p]),
    "lar_fit_dti_maps": (_i32, [_p, _p, _p, _i64, _i32, _i64, _f64, _i32, _p, _p, _p, _p]),
    "lar_dki_maps": (_i32, [_p, _i64, _p, _p, _p]),
    "lar_fit_dki_maps": (_i32, [_p, _p, _p, _p, _p, _i64, _i32, _i64, _f64, _i32, _p, _p, _p, _p, _p]),
    "lar_lsi_design_create": (_i32, [_p, _i64, _i64, _p, _i64, _f64, _p]),
    "lar_lsi_design_destroy": (None, [_p]),
    "lar_lsi_design_matrices": (_i32, [_p, _p, _p, _p, _p, _p]),
    "lar_fit_lsi": (_i32, [_p, _p, _i64, _i32, _p, _p, _p, _p, _p, _p]),
    "lar_fit_lsi_plain_fp32": (_i32, [_p, _p, _i64, _p, _p, _p]),
    "lar_l2nnls_create": (_i32, [_p, _i64, _i64, _f64, _f64, _p]),
    "lar_fod_solver_destroy": (None, [_p]),
    "lar_deconv_kernel_create": (_i32, [_p, _i64, _i64, _p, _p, _i64, _p, _i64, _p]),
    "lar_deconv_kernel_destroy": (None, [_p]),
    "lar_fit_multi_tissue": (_i32, [_p, _i64, _p, _p, _p, _p, _p, _i64, _f64, _f64, _p, _p, _p, _p, _p]),
    "lar_fit_multi_tissue_async": (_i32, [_p, _i64, _p, _p, _p, _p, _p, _i64, _f64, _f64, _p, _p, _p, _p, _p]),
    "lar_fit_multi_tissue_plain_fp32": (_i32, [_p, _i64, _p, _p, _p, _p, _p, _i64, _f64, _f64, _p, _p, _p, _p, _p]),
    "lar_lsqnonneg": (_i32, [_p, _i64, _i64, _p, _i32, _f64, _p, _p]),
    "lar_batch_create": (_i32, [_p]),
    "lar_batch_destroy": (None, [_p]),
    "lar_batch_add_dti": (_i32, [_p, _p, _p, _p, _i64, _i32, _i64, _f64, _p, _p]),
    "lar_batch_add_dki": (_i32, [_p, _p, _p, _p, _p, _p, _i64, _i32, _i64, _f64, _p, _p, _p, _p]),
    "lar_batch_add_mfod": (_i32, [_p, _p, _i64, _p, _p, _p, _p, _p, _i64, _f64, _f64, _p, _p, _p, _p]),
    "lar_batch_finalize": (_i32, [_p]),
    "lar_batch_run": (_i32, [_p, _i32, _p]),
    "lar_fit_single_tissue": (_i32, [_p, _i64, _p, _p, _p, _p]),
    "lar_sh_projector_create": (_i32, [_p, _i64, _i64, _p]),
    "lar_sh_projector_destroy": (None, [_p]),
    "lar_project_sh": (_i32, [_p, _p, _i64, _i64, _i32, _p, _i64, _p]),
    "lar_drl_create": (_i32, [_p, _p, _i64, _i64, _f64, _i64, _f64, _p]),
    "lar_drl_set_precision": (_i32, [_p, _i32]),
    "lar_drl_errors": (_i32, [_p, _p]),
    "lar_csd_create": (_i32, [_p, _i64, _i64, _p, _i64, _p, _i64, _f64, _f64, _i64, _p]),
    "lar_csd_destroy": (None, [_p]),
    "lar_fit_csd": (_i32, [_p, _p, _i64, _p, _p, _p]),
    "lar_stage_dwi": (_i32, [_p, _i32, _i64, _i64, _i64, _i64, _f64, _f64, _p, _i64, _p, _p, _p, _p, _p, _p, _p]),
    "lar_normalise_signals": (_i32, [_p, _p, _i64, _i64, _p, _p, _p]),
    "lar_unmask_rows": (_i32, [_p, _i64, _i64, _p, _i64, _p, _p]),
    "lar_peak_sphere_create": (_i32, [_p, _p, _i64, _p]),
    "lar_peak_sphere_destroy": (None, [_p]),
    "lar_sh_derivatives": (_i32, [_p, _i64, _i64, _i32, _i32, _p, _p, _p, _p]),
    "lar_climb": (_i32, [_p, _i64, _i64, _i32, _i32, _p, _i32, _f64, _f64, _p, _p, _p]),
    "lar_find_peaks": (_i32, [_p, _p, _i64, _i64, _i32, _i32, _p, _i64, _i32, _f64, _f64, _p, _p, _p]),
    "lar_fit_log_signal_noalloc": (_i32, [_p, _i64, _i64, _p, _i64, _p, _i64, _i32, _i64, _f64, _p, _p, _p]),
}

LAR_OK, LAR_ERR_INVALID, LAR_ERR_CUDA, LAR_ERR_MEMORY = 0, 1, 2, 3
LAR_FP64, LAR_FP32, LAR_TF32X3 = 0, 1, 2
LAR_BATCH_DTI, LAR_BATCH_DKI, LAR_BATCH_MFOD = 1, 2, 4
# Sample types of lar_stage_dwi, by numpy dtype.
LAR_DTYPES = {"float32": 0, "float64": 1, "int16": 2, "uint16": 3, "int8": 4, "uint8": 5, "int32": 6, "uint32": 7}

_lib: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    """The loaded library, with argument types declared."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m larmor_b200.build` "
                "(larmor_b200 has no CPU fallback)"
            )
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status: int) -> None:
    """Raises the Python error of a failed C-ABI call."""
    if status == LAR_OK:
        return
    message = lib().lar_last_error().decode()
    if status == LAR_ERR_INVALID:
        raise ValueError(message)
    if status == LAR_ERR_MEMORY:
        raise MemoryError(message)
    raise RuntimeError(f"CUDA error in larmor_b200: {message}")


def ptr(tensor) -> ctypes.c_void_p:
    """The device (or host) address of a torch tensor or numpy array, for the C ABI."""
    if tensor is None:
        return ctypes.c_void_p(None)
    if hasattr(tensor, "data_ptr"):
        return ctypes.c_void_p(tensor.data_ptr())
    return ctypes.c_void_p(tensor.ctypes.data)
