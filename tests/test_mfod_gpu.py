"""The mFOD multi-tissue fit on the GPU against the oracle and MRIToolkit's MATLAB output
(tests/sd/test_matlab_match.py:143-165), and the single-tissue L2NNLS fit."""

from __future__ import annotations

import numpy as np
import pytest

from test_oracle import mfod_inputs

pytestmark = pytest.mark.gpu


def _gpu_fit(z, signals, rounds=False):
    import torch

    from larmor_b200 import _core

    lr = _core.DeconvKernel(np.ascontiguousarray(z["lr_k_aniso"]), np.ascontiguousarray(z["lr_k_iso"]),
                            np.ascontiguousarray(z["lr_w_k_iso"]), [(0, z["lr_k_aniso"].shape[1])])
    hr = _core.DeconvKernel(np.ascontiguousarray(z["hr_k_aniso"]), np.ascontiguousarray(z["hr_k_iso"]),
                            np.ascontiguousarray(z["hr_w_k_iso"]), [tuple(b) for b in z["hr_blocks"]])
    lr_solver = _core.FodSolver.l2nnls(np.ascontiguousarray(z["lr_w_k_aniso"]), 0.0, 1e-6)
    hr_solver = _core.FodSolver.l2nnls(np.ascontiguousarray(z["hr_w_k_aniso"]), 0.1, 1e-6)
    dev = torch.device("cuda")
    v = len(signals)
    s = torch.from_numpy(np.ascontiguousarray(signals)).to(dev)
    fods = torch.empty((v, hr.ca), dtype=torch.float64, device=dev)
    fr = torch.empty((v, hr.nb + hr.ci), dtype=torch.float64, device=dev)
    rd = torch.empty((v,), dtype=torch.int32, device=dev)
    st = torch.empty((v,), dtype=torch.uint8, device=dev)
    _core.fit_multi_tissue_device(s, z["weights"], lr, lr_solver, hr, hr_solver, 50, 1e-7, 1e-2, fods, fr, rd, st)
    return fods.cpu().numpy(), fr.cpu().numpy(), rd.cpu().numpy(), st.cpu().numpy()


def test_multi_tissue_matches_the_oracle(cuda, oracle, mfod_fixture):
    signals, lr, hr = mfod_inputs(mfod_fixture)
    fods, fractions, rounds, status = _gpu_fit(mfod_fixture, signals)
    rfods, rfr, rrounds = oracle.fit_multi_tissue(signals, mfod_fixture["weights"], lr, hr, n_threads=4, rounds=True)
    assert (status == 0).all()
    np.testing.assert_array_equal(rounds, rrounds)
    # Identical active sets of the final FOD, and values to rounding.
    np.testing.assert_array_equal(fods != 0, rfods != 0)
    scale = np.abs(rfods).max(axis=1, keepdims=True)
    assert (np.abs(fods - rfods) <= 1e-9 * scale).all()
    np.testing.assert_allclose(fractions, rfr, rtol=0, atol=1e-10)


def test_multi_tissue_matches_mritoolkit(cuda, mfod_fixture):
    signals, _, _ = mfod_inputs(mfod_fixture)
    fods, fractions, _, _ = _gpu_fit(mfod_fixture, signals)
    ref_fod = mfod_fixture["matlab_fod"]
    fod_err = np.abs(fods - ref_fod).max(axis=1) / ref_fod.max(axis=1)
    assert fod_err.max() <= 1e-4
    np.testing.assert_allclose(fractions, mfod_fixture["matlab_fractions"], rtol=0, atol=1e-5)


@pytest.mark.parametrize("ridge", [0.0, 0.1])
def test_single_tissue_l2nnls_matches_the_oracle(cuda, oracle, mfod_fixture, ridge):
    from larmor_b200 import _core

    signals, _, _ = mfod_inputs(mfod_fixture)
    k = np.ascontiguousarray(mfod_fixture["hr_w_k_aniso"][:, :300])
    solver = _core.FodSolver.l2nnls(k, ridge, 1e-6)
    fods = _core.fit_single_tissue(np.ascontiguousarray(signals), solver, 1)
    ref = oracle.ridge_nnls(k, ridge, 1e-6, signals, n_threads=4)
    np.testing.assert_array_equal(fods != 0, ref != 0)
    # Values to the forward error of an FP64 normal-equations solve, 10 cond(G_AA) eps of the
    # largest coefficient (cond(G_AA) reaches 8e6 here without the ridge; both fits carry that
    # error, in different rounding).
    gram = k.T @ k + ridge**2 * np.eye(k.shape[1])
    for v in range(signals.shape[0]):
        act = np.nonzero(ref[v])[0]
        if len(act) == 0:
            continue
        tol = 10 * np.linalg.cond(gram[np.ix_(act, act)]) * np.finfo(np.float64).eps
        assert np.abs(fods[v] - ref[v]).max() <= max(tol, 1e-9) * np.abs(ref[v]).max()


def test_sd_model_three_tissue_matches_the_oracle(cuda, oracle):
    from larmor_b200.sd import AnisotropicRF, IsotropicRF, SDModel
    from larmor_b200.sd.model import to_sh
    from larmor_b200.synthetic import mfod_signals, mfod_table
    from larmor_b200.types import Volume

    rng = np.random.default_rng(3)
    gtab = mfod_table(rng)
    sig = mfod_signals(rng, gtab, 64)
    data = sig.reshape(4, 4, 4, -1).astype(np.float32)
    rfs = [AnisotropicRF([1.7e-3, 0.2e-3, 0.2e-3], 0.0), IsotropicRF(0.8e-3), IsotropicRF(3e-3)]
    model = SDModel(rfs, method="mFOD")
    fit = model.fit(Volume(data, np.eye(4)), gtab)
    # The oracle on the same normalised signals and kernels.
    s = data.reshape(-1, data.shape[-1]).astype(np.float64)
    s0 = s[:, gtab.b0_mask].mean(axis=1)
    norm = np.minimum(s / s0[:, None], 1.0)
    from larmor_b200.sd.solvers import L2NNLS

    hr, lr, _, _ = model._prepare(L2NNLS(), gtab.bvals, gtab.bvecs)
    lrd = dict(k_aniso=lr.k_aniso, k_iso=lr.k_iso, w_k_iso=lr.w_k_iso, w_k_aniso=lr.w_k_aniso)
    hrd = dict(k_aniso=hr.k_aniso, k_iso=hr.k_iso, w_k_iso=hr.w_k_iso, w_k_aniso=hr.w_k_aniso,
               blocks=[(b.start, b.stop) for b in hr.aniso_blocks])
    rfods, rfr = oracle.fit_multi_tissue(norm, lr.weights, lrd, hrd)
    ref_sh = to_sh(rfods, fit.lmax, "tournier", exact_integral=True)
    # The maps are float32, as the reference's.
    np.testing.assert_allclose(fit.fods[0].reshape(-1, ref_sh.shape[1]), ref_sh, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(fit.tissue_fractions.reshape(-1, 3), rfr, rtol=0, atol=1e-6)


@pytest.mark.parametrize("lmax", [8, 12])
@pytest.mark.parametrize("exact_integral", [True, False])
def test_sh_projection_matches_the_least_squares_fit(cuda, lmax, exact_integral):
    """The device _to_sh (amplitudes on DIRS_300 to SH) against numpy's lstsq restatement, on
    column blocks of a two-block amplitude array (a strided source) and with more than one
    48-coefficient tile (lmax 12: 91 coefficients)."""
    import torch

    from larmor_b200 import _core
    from larmor_b200.sd.model import sh_projector, to_sh

    rng = np.random.default_rng(11)
    amps = np.abs(rng.normal(size=(1000, 600)))
    amps[rng.random(amps.shape) < 0.8] = 0.0
    d = torch.from_numpy(amps).to("cuda")
    projector = sh_projector(lmax, "tournier")
    for block in (slice(0, 300), slice(300, 600)):
        ref = to_sh(amps[:, block], lmax, "tournier", exact_integral=exact_integral)
        got = _core.project_sh_device(projector, d[:, block], exact_integral).cpu().numpy()
        assert (np.abs(got - ref) <= 1e-12 * np.abs(ref).max(axis=1, keepdims=True)).all()


def test_async_multi_tissue_equals_the_waiting_call(cuda, mfod_fixture):
    """lar_fit_multi_tissue_async (every round enqueued, counts read on the device) gives the
    waiting call's results bit for bit, including the round counts."""
    import torch

    from larmor_b200 import _core

    z = mfod_fixture
    signals, _, _ = mfod_inputs(z)
    fods, fr, rd, st = _gpu_fit(z, signals)
    lr = _core.DeconvKernel(np.ascontiguousarray(z["lr_k_aniso"]), np.ascontiguousarray(z["lr_k_iso"]),
                            np.ascontiguousarray(z["lr_w_k_iso"]), [(0, z["lr_k_aniso"].shape[1])])
    hr = _core.DeconvKernel(np.ascontiguousarray(z["hr_k_aniso"]), np.ascontiguousarray(z["hr_k_iso"]),
                            np.ascontiguousarray(z["hr_w_k_iso"]), [tuple(b) for b in z["hr_blocks"]])
    lr_solver = _core.FodSolver.l2nnls(np.ascontiguousarray(z["lr_w_k_aniso"]), 0.0, 1e-6)
    hr_solver = _core.FodSolver.l2nnls(np.ascontiguousarray(z["hr_w_k_aniso"]), 0.1, 1e-6)
    dev = torch.device("cuda")
    v = len(signals)
    s = torch.from_numpy(np.ascontiguousarray(signals)).to(dev)
    out = dict(fods=torch.zeros((v, hr.ca), dtype=torch.float64, device=dev),
               fr=torch.zeros((v, hr.nb + hr.ci), dtype=torch.float64, device=dev),
               rd=torch.zeros((v,), dtype=torch.int32, device=dev), st=torch.ones((v,), dtype=torch.uint8, device=dev))
    _core.fit_multi_tissue_device(s, z["weights"], lr, lr_solver, hr, hr_solver, 50, 1e-7, 1e-2, out["fods"],
                                  out["fr"], out["rd"], out["st"], asynchronous=True)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out["fods"].cpu().numpy(), fods)
    np.testing.assert_array_equal(out["fr"].cpu().numpy(), fr)
    np.testing.assert_array_equal(out["rd"].cpu().numpy(), rd)
    np.testing.assert_array_equal(out["st"].cpu().numpy(), st)


def test_plain_fp32_fit_stays_near_the_fp64_oracle(cuda, oracle):
    """The plain single-precision fit (the comparison baseline) of 256 voxels of the three-tissue
    generator (WM on the 300 directions, GM, CSF): finite FODs and fractions near the FP64
    oracle's, at the accuracy FP32 arithmetic allows (a median FOD error below 1e-2 of the
    voxel's largest amplitude, fractions within 5e-2)."""
    import torch

    from larmor_b200 import _core
    from larmor_b200.sd.kernel import Kernel
    from larmor_b200.sd.model import compute_shell_weights, low_resolution_dirs
    from larmor_b200.sd.solvers import L2NNLS, Stage, _deconv_kernel
    from larmor_b200.sd.sphere import DIRS_300
    from larmor_b200.synthetic import mfod_model_responses, mfod_signals, mfod_table

    rng = np.random.default_rng(11)
    gtab = mfod_table(rng)
    sig = mfod_signals(rng, gtab, 256).astype(np.float64)
    norm = np.ascontiguousarray(np.minimum(sig / sig[:, gtab.b0_mask].mean(axis=1)[:, None], 1.0))
    rfs = mfod_model_responses()
    w = compute_shell_weights(gtab.bvals, 1.0)
    hr = Kernel(rfs, gtab.bvals, gtab.bvecs, dirs=DIRS_300, weights=w)
    lr = Kernel(rfs, gtab.bvals, gtab.bvecs, dirs=low_resolution_dirs(rfs, len(gtab.bvals)), weights=w)
    k_lr, k_hr = _deconv_kernel(lr), _deconv_kernel(hr)
    lr_solver = L2NNLS()._prepare(lr, gtab.bvals, Stage.LOW_RES)
    hr_solver = L2NNLS()._prepare(hr, gtab.bvals, Stage.HIGH_RES)
    dev = torch.device("cuda")
    v = len(norm)
    s = torch.from_numpy(norm).to(dev).float()
    fods = torch.empty((v, k_hr.ca), dtype=torch.float32, device=dev)
    fr = torch.empty((v, 3), dtype=torch.float32, device=dev)
    rd = torch.empty((v,), dtype=torch.int32, device=dev)
    st = torch.empty((v,), dtype=torch.uint8, device=dev)
    _core.fit_multi_tissue_plain_fp32_device(s, lr.weights, k_lr, lr_solver, k_hr, hr_solver, 50, 1e-7, 1e-2, fods,
                                             fr, rd, st)
    got, got_fr = fods.double().cpu().numpy(), fr.double().cpu().numpy()
    lrd = dict(k_aniso=lr.k_aniso, k_iso=lr.k_iso, w_k_iso=lr.w_k_iso, w_k_aniso=lr.w_k_aniso)
    hrd = dict(k_aniso=hr.k_aniso, k_iso=hr.k_iso, w_k_iso=hr.w_k_iso, w_k_aniso=hr.w_k_aniso,
               blocks=[(b.start, b.stop) for b in hr.aniso_blocks])
    rfods, rfr = oracle.fit_multi_tissue(norm, lr.weights, lrd, hrd, n_threads=4)
    rel = np.abs(got - rfods).max(axis=1) / np.abs(rfods).max(axis=1)
    print(f"plain FP32, {v} voxels: FOD rel max {rel.max():.3e}, median {np.median(rel):.3e}; fractions abs max "
          f"{np.abs(got_fr - rfr).max():.3e}; status nonzero {(st.cpu().numpy() != 0).mean():.4f}")
    assert np.isfinite(got).all() and np.isfinite(got_fr).all()
    assert np.median(rel) <= 1e-2
    assert np.abs(got_fr - rfr).max() <= 5e-2
