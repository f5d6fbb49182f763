"""The C-ABI library: it loads without a GPU, exports every function include/*.h declares,
and the Python mirror of larmor._core refuses bad inputs as the reference's bindings do
(before any device work)."""

from __future__ import annotations

import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> set[str]:
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        names.update(re.findall(r"\b(lar_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_function():
    from larmor_b200 import _lib

    lib = _lib.lib()
    names = declared_functions()
    assert len(names) >= 6
    for name in names:
        assert hasattr(lib, name), name
    assert set(_lib.SIGNATURES) == names


def test_version_and_error_string_need_no_gpu():
    import threading

    from larmor_b200 import _lib

    assert b"sm_100a" in _lib.lib().lar_version()
    # The error string is per host thread: a thread that made no failed call reads "".
    seen = []
    t = threading.Thread(target=lambda: seen.append(_lib.lib().lar_last_error()))
    t.start()
    t.join()
    assert seen == [b""]


def test_design_create_refuses_bad_shapes_without_a_gpu():
    import ctypes

    from larmor_b200 import _lib

    x = np.zeros((3, 7))
    handle = ctypes.c_void_p()
    status = _lib.lib().lar_log_design_create(_lib.ptr(x), 3, 7, None, 0, ctypes.byref(handle))
    assert status == _lib.LAR_ERR_INVALID
    assert b"n >= p" in _lib.lib().lar_last_error()


def test_batch_refuses_misuse_without_a_gpu():
    import ctypes

    from larmor_b200 import _lib

    lib = _lib.lib()
    batch = ctypes.c_void_p()
    assert lib.lar_batch_create(ctypes.byref(batch)) == _lib.LAR_OK
    try:
        assert lib.lar_batch_run(batch, _lib.LAR_BATCH_DTI, None) == _lib.LAR_ERR_INVALID
        assert b"finalize" in lib.lar_last_error()
        status = lib.lar_batch_add_dti(batch, None, None, None, 10, 1, 20, 1e-6, None, None)
        assert status == _lib.LAR_ERR_INVALID
        assert b"must not be NULL" in lib.lar_last_error()
    finally:
        lib.lar_batch_destroy(batch)


DESIGN = np.column_stack([np.ones(43), np.random.default_rng(3).normal(size=(43, 6))])


@pytest.mark.parametrize(
    ("x", "g", "log_s", "n_threads", "error", "message"),
    [
        (DESIGN, np.zeros((0, 6)), np.zeros((2, 43)), 1, ValueError, "must be"),
        (DESIGN, np.zeros((0, 7)), np.zeros((2, 40)), 1, ValueError, "must be"),
        (DESIGN, np.zeros((0, 7)), np.zeros((2, 43)), 0, ValueError, "n_threads"),
        (DESIGN, np.zeros((0, 7)), np.zeros((43, 2)).T, 1, ValueError, "C-contiguous"),
        (DESIGN, np.zeros((0, 7)), np.zeros((2, 43), np.float32), 1, TypeError, "float64"),
    ],
    ids=["constraints", "measurements", "threads", "strides", "dtype"],
)
def test_fit_log_signal_refuses_mismatched_inputs(x, g, log_s, n_threads, error, message):
    from larmor_b200 import _core

    with pytest.raises(error, match=message):
        _core.fit_log_signal(x, g, log_s, True, 20, 1e-6, n_threads)


def test_models_refuse_bad_settings():
    from larmor_b200.dwi import DTIModel

    with pytest.raises(ValueError, match="Unknown DTI fit method"):
        DTIModel(fit_method="nlls")
    with pytest.raises(ValueError, match="precision"):
        DTIModel(precision="fp16")
