"""The entry point that allocates no device memory, lar_fit_log_signal_noalloc.

Callers that cannot allocate device memory (an application that owns all device memory through
its own allocator or budget, a plugin host that hands out only its own buffers) use this entry
point instead of lar_fit_log_signal, whose design handle and scratch buffer are allocated with
cudaMalloc. It keeps everything it needs in one static 32 MiB device array. The GPU test calls
it through the C ABI twice in a row (the second call reuses the array the first one left
behind) and checks both results against the existing entry point. This file is collected last,
so a run that stops at the first failure has run every other test before it.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest


def _noalloc(lib_mod, x, g, log_s_dev, params_dev, broke_dev, weighted, stream):
    lib = lib_mod.lib()
    n, p = x.shape
    status = lib.lar_fit_log_signal_noalloc(
        lib_mod.ptr(x), n, p, lib_mod.ptr(g if len(g) else None), g.shape[0], lib_mod.ptr(log_s_dev),
        log_s_dev.shape[0], int(weighted), 20, 1e-6, lib_mod.ptr(params_dev), lib_mod.ptr(broke_dev),
        ctypes.c_void_p(stream))
    lib_mod.check(status)


@pytest.mark.gpu
def test_no_alloc_fit_matches_the_design_handle_fit_on_two_calls_in_a_row(cuda, dki_block):
    import torch

    from larmor_b200 import _core, _lib

    design = np.ascontiguousarray(dki_block["dki_design"])
    g = np.ascontiguousarray(dki_block["dki_constraints"])
    s = dki_block["signals_f32"].astype(np.float64)[dki_block["positive"]]
    scale = np.linalg.norm(design, axis=0)
    dev = torch.device("cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # Call 1: weighted, constrained, the block as it is; call 2: ordinary, constrained, the
    # voxels in reverse order and one fewer, on the array call 1 left behind.
    cases = [(np.log(s), True), (np.log(s[::-1][1:]), False)]
    for log_s, weighted in cases:
        log_s = np.ascontiguousarray(log_s)
        v = len(log_s)
        d_log = torch.from_numpy(log_s).to(dev)
        d_params = torch.full((v, 22), np.nan, dtype=torch.float64, device=dev)
        d_broke = torch.full((v,), 7, dtype=torch.uint8, device=dev)
        _noalloc(_lib, design, g, d_log, d_params, d_broke, weighted, stream)
        torch.cuda.synchronize()
        got = d_params.cpu().numpy()
        got_broke = d_broke.cpu().numpy().astype(bool)
        want, want_broke = _core.fit_log_signal(design, g, log_s, weighted, 20, 1e-6, 1)
        np.testing.assert_array_equal(got_broke, want_broke)
        assert got_broke.sum() > 100
        np.testing.assert_allclose(got * scale, want * scale, rtol=0, atol=1e-10)


@pytest.mark.gpu
def test_no_alloc_fit_without_constraints_matches_the_design_handle_fit(cuda, dki_block):
    """The DTI design with no constraint rows (m = 0): the route with no violator list and no
    counters to clear, twice in a row (weighted, then ordinary on the voxels reversed)."""
    import torch

    from larmor_b200 import _core, _lib

    design = np.ascontiguousarray(dki_block["dti_design"])
    g = np.zeros((0, design.shape[1]))
    s = dki_block["signals_f32"].astype(np.float64)[dki_block["positive"]]
    scale = np.linalg.norm(design, axis=0)
    dev = torch.device("cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for log_s, weighted in [(np.log(s), True), (np.log(s[::-1]), False)]:
        log_s = np.ascontiguousarray(log_s)
        v = len(log_s)
        d_log = torch.from_numpy(log_s).to(dev)
        d_params = torch.full((v, design.shape[1]), np.nan, dtype=torch.float64, device=dev)
        d_broke = torch.full((v,), 7, dtype=torch.uint8, device=dev)
        _noalloc(_lib, design, g, d_log, d_params, d_broke, weighted, stream)
        torch.cuda.synchronize()
        want, want_broke = _core.fit_log_signal(design, g, log_s, weighted, 20, 1e-6, 1)
        got_broke = d_broke.cpu().numpy().astype(bool)
        np.testing.assert_array_equal(got_broke, want_broke)
        assert not got_broke.any()
        np.testing.assert_allclose(d_params.cpu().numpy() * scale, want * scale, rtol=0, atol=1e-10)


def test_no_alloc_fit_refuses_a_design_larger_than_its_array():
    from larmor_b200 import _lib

    x = np.ascontiguousarray(np.random.default_rng(0).normal(size=(80_000, 32)))
    status = _lib.lib().lar_fit_log_signal_noalloc(
        _lib.ptr(x), 80_000, 32, ctypes.c_void_p(None), 0, ctypes.c_void_p(None), 10, 1, 20, 1e-6,
        ctypes.c_void_p(None), ctypes.c_void_p(None), ctypes.c_void_p(None))
    assert status == _lib.LAR_ERR_INVALID
    message = _lib.lib().lar_last_error().decode()
    assert "design itself is too large" in message


def test_no_alloc_fit_refuses_more_voxels_than_its_array_holds():
    from larmor_b200 import _lib

    x = np.ascontiguousarray(np.random.default_rng(0).normal(size=(134, 22)))
    g = np.ascontiguousarray(np.random.default_rng(1).normal(size=(768, 22)))
    status = _lib.lib().lar_fit_log_signal_noalloc(
        _lib.ptr(x), 134, 22, _lib.ptr(g), 768, ctypes.c_void_p(None), 10_000_000, 1, 20, 1e-6,
        ctypes.c_void_p(None), ctypes.c_void_p(None), ctypes.c_void_p(None))
    assert status == _lib.LAR_ERR_INVALID
    message = _lib.lib().lar_last_error().decode()
    assert "32 MiB" in message and "voxels per call" in message
