"""MSMT-CSD's LSI solve on the GPU against the oracle and the reference's known-answer tests
(tests/sd/test_msmt.py, cpp/tests/sd/test_lsi.cpp)."""

from __future__ import annotations

import numpy as np
import pytest
from scipy.optimize import nnls as scipy_nnls

pytestmark = pytest.mark.gpu


def _design(msmt_fixture):
    from larmor_b200 import _core

    f, g = msmt_fixture["forward"], msmt_fixture["constraints"]
    return _core.LsiDesign(np.ascontiguousarray(f), np.ascontiguousarray(g), float(msmt_fixture["ridge"]))


def _signals(msmt_fixture, v, seed):
    rng = np.random.default_rng(seed)
    f = msmt_fixture["forward"]
    noisy = 300.0 + 200.0 * rng.standard_normal((v // 2, f.shape[0]))
    # Plausible voxels too: non-negative FOD-like coefficients, GM and CSF, some noise.
    coef = np.zeros((v - v // 2, f.shape[1]))
    coef[:, 0] = rng.uniform(0.1, 0.3, len(coef))
    coef[:, 1:45] = 0.05 * rng.standard_normal((len(coef), 44))
    coef[:, 45:] = rng.uniform(0.0, 0.2, (len(coef), 2))
    clean = coef @ f.T
    return np.vstack([noisy, clean + 20.0 * rng.standard_normal(clean.shape)])


def _device_fit(design, signals, only_qr=False):
    import torch

    from larmor_b200 import _core

    dev = torch.device("cuda")
    v = len(signals)
    s = torch.from_numpy(np.ascontiguousarray(signals)).to(dev)
    x = torch.empty((v, design.n), dtype=torch.float64, device=dev)
    conv = torch.empty((v,), dtype=torch.uint8, device=dev)
    status = torch.empty((v,), dtype=torch.uint8, device=dev)
    outer = torch.empty((v,), dtype=torch.int32, device=dev)
    active = torch.empty((v, design.k), dtype=torch.uint8, device=dev)
    _core.fit_lsi_device(design, s, x, conv, status, outer, active, only_qr=only_qr)
    return (x.cpu().numpy(), conv.cpu().numpy().astype(bool), status.cpu().numpy(), outer.cpu().numpy(),
            active.cpu().numpy().astype(bool))


def test_prepared_design_matches_the_oracle(cuda, oracle, msmt_fixture):
    design = _design(msmt_fixture)
    ours = design.matrices()
    ref = oracle.lsi_design(msmt_fixture["forward"], msmt_fixture["constraints"], float(msmt_fixture["ridge"]))
    for key in ("back", "e", "gram", "abs_sums"):
        scale = np.abs(ref[key]).max()
        np.testing.assert_allclose(ours[key], ref[key], rtol=0, atol=1e-12 * scale, err_msg=key)
    # Q is unique up to the signs the pivoted QR fixes; compare q_t directly.
    np.testing.assert_allclose(ours["q_t"], ref["q_t"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("only_qr", [False, True], ids=["cholesky", "qr"])
def test_lsi_matches_the_oracle_with_identical_active_sets(cuda, oracle, msmt_fixture, only_qr):
    design = _design(msmt_fixture)
    signals = _signals(msmt_fixture, 256, seed=1)
    x, conv, status, outer, active = _device_fit(design, signals, only_qr)
    rx, rconv, rstatus, router, ractive = oracle.fit_lsi(
        msmt_fixture["forward"], msmt_fixture["constraints"], float(msmt_fixture["ridge"]), signals,
        only_qr=only_qr, details=True)
    np.testing.assert_array_equal(conv, rconv)
    np.testing.assert_array_equal(status, rstatus)
    np.testing.assert_array_equal(active, ractive)
    if not only_qr:
        np.testing.assert_array_equal(outer, router)
    np.testing.assert_allclose(x, rx, rtol=0, atol=1e-9)
    # Values to the forward error of the active-set solve, 10 cond(H_AA) eps of the voxel's
    # largest coefficient (at least 1e-10 of it): both fits solve H_AA u_A = f_A, with H = E E^T + f f^T
    # reaching cond 3e8 here, in different rounding.
    m = oracle.lsi_design(msmt_fixture["forward"], msmt_fixture["constraints"], float(msmt_fixture["ridge"]))
    for v in range(len(signals)):
        scale = np.abs(rx[v]).max()
        tol = 1e-10
        act = np.nonzero(ractive[v])[0]
        if rstatus[v] == 0 and len(act):
            rot = m["q_t"] @ signals[v]
            f = -m["e"] @ rot
            f /= np.abs(f).max()
            h = (m["gram"] + np.outer(f, f))[np.ix_(act, act)]
            tol = max(tol, 10 * np.linalg.cond(h) * np.finfo(np.float64).eps)
        assert np.abs(x[v] - rx[v]).max() <= tol * scale
    assert active.sum(axis=1).max() > 5


def test_lsi_meets_the_kkt_conditions(cuda, msmt_fixture):
    from larmor_b200 import _core

    design = _design(msmt_fixture)
    fwd, g = msmt_fixture["forward"], msmt_fixture["constraints"]
    ridge2 = float(msmt_fixture["ridge"]) ** 2
    rng = np.random.default_rng(7)
    noisy = 300.0 + 200.0 * rng.standard_normal((8, fwd.shape[0]))
    x, conv = _core.fit_lsi(noisy, design, 1)
    assert conv.all()
    for s, xi in zip(noisy, x):
        values = g @ xi
        assert values.min() > -1e-9
        act = values < 1e-9 * np.abs(values).max()
        assert act.sum() > 5
        grad = fwd.T @ (fwd @ xi - s) + ridge2 * xi
        _, residual = scipy_nnls(g[act].T, grad)
        assert residual < 1e-8 * np.linalg.norm(fwd.T @ s)


def test_lsi_small_known_answers(cuda):
    from larmor_b200 import _core

    d = _core.LsiDesign(np.eye(3), np.eye(3), 0.0)
    x, conv = _core.fit_lsi(np.array([[2.0, -1.0, 3.0]]), d, 1)
    np.testing.assert_allclose(x[0], [2.0, 0.0, 3.0], atol=1e-12)
    d = _core.LsiDesign(np.eye(2), np.array([[-1.0, -1.0]]), 0.0)
    x, _ = _core.fit_lsi(np.array([[0.5, 0.5]]), d, 1)
    np.testing.assert_allclose(x[0], [0.0, 0.0], atol=1e-12)


def test_msmt_model_recovers_a_wm_csf_mixture(cuda, msmt_fixture):
    """tests/sd/test_msmt.py:75: fractions (0.7, 0.3) and the FOD within 1e-6."""
    from larmor_b200.sd import MSMTCSDModel, ZonalSHRF
    from larmor_b200.sd.msmt import forward_matrix
    from larmor_b200.sd.sh import fit_sh
    from larmor_b200.sd.sphere import DIRS_300
    from larmor_b200.types import GradientTable, Volume

    shells = msmt_fixture["shells"]
    wm = ZonalSHRF(bvals=shells, coefficients=msmt_fixture["wm_coefficients"])
    csf = ZonalSHRF(bvals=shells, coefficients=msmt_fixture["csf_coefficients"])
    gtab = GradientTable(msmt_fixture["bvals"], msmt_fixture["bvecs"])
    fibre = np.array([0.6, 0.0, 0.8])
    fod_true = fit_sh(0.7 * 9 / (4 * np.pi) * (DIRS_300 @ fibre) ** 8, DIRS_300, 8)
    fwd = forward_matrix([wm, csf], [8, 0], gtab.bvals, gtab.bvecs)
    csf_coef = 0.3 / np.sqrt(4 * np.pi) * 1000.0 / msmt_fixture["csf_coefficients"][0, 0] * np.sqrt(4 * np.pi)
    signal = fwd @ np.concatenate([fod_true, [0.3 / np.sqrt(4 * np.pi)]])
    volume = Volume(np.tile(signal, (2, 1, 1, 1)), np.eye(4))
    fit = MSMTCSDModel([csf, wm]).fit(volume, gtab, n_jobs=1)
    np.testing.assert_allclose(fit.tissue_fractions[0, 0, 0], (0.7, 0.3), atol=1e-6)
    np.testing.assert_allclose(fit.fods[0][0, 0, 0], fod_true, atol=1e-6)
    assert csf_coef > 0


def _plain_fp32(design, signals):
    import torch

    from larmor_b200 import _core

    dev = torch.device("cuda")
    s32 = torch.from_numpy(np.ascontiguousarray(signals, dtype=np.float32)).to(dev)
    x32 = torch.empty((len(signals), design.n), dtype=torch.float32, device=dev)
    status = torch.empty((len(signals),), dtype=torch.uint8, device=dev)
    _core.fit_lsi_plain_fp32_device(design, s32, x32, status)
    return x32.double().cpu().numpy(), status.cpu().numpy()


def test_plain_fp32_lsi_known_answers_and_a_well_conditioned_problem(cuda):
    """The plain single-precision LSI fit (the comparison baseline: FP32, the active Cholesky
    factor formed anew for every fit, no QR fallback) gives the known answers and, on a
    well-conditioned random problem, the FP64 fit's solutions to single precision."""
    from larmor_b200 import _core

    d = _core.LsiDesign(np.eye(3), np.eye(3), 0.0)
    x, st = _plain_fp32(d, np.array([[2.0, -1.0, 3.0]]))
    np.testing.assert_allclose(x[0], [2.0, 0.0, 3.0], atol=1e-5)
    assert st[0] == 0
    d = _core.LsiDesign(np.eye(2), np.array([[-1.0, -1.0]]), 0.0)
    x, _ = _plain_fp32(d, np.array([[0.5, 0.5]]))
    np.testing.assert_allclose(x[0], [0.0, 0.0], atol=1e-5)
    # x >= 0 and 20 non-negative combinations of x: the feasible cone is the orthant.
    rng = np.random.default_rng(5)
    a = rng.standard_normal((60, 10))
    g = np.vstack([np.eye(10), rng.uniform(0.0, 1.0, (20, 10))])
    d = _core.LsiDesign(a, g, 0.0)
    signals = rng.standard_normal((256, 60))
    x64 = _device_fit(d, signals)[0]
    x32, st = _plain_fp32(d, signals)
    ok = st == 0
    assert ok.mean() >= 0.95
    rel = np.abs(x32 - x64).max(axis=1) / np.abs(x64).max(axis=1)
    print(f"plain FP32 LSI, random orthant problem: rel median {np.median(rel[ok]):.2e}, max {rel[ok].max():.2e}")
    assert np.median(rel[ok]) <= 1e-4


def test_plain_fp32_lsi_on_the_msmt_problem(cuda, msmt_fixture):
    """On MSMT-CSD's problem (47 unknowns, 302 constraints, ~40 active) the least-distance
    system E_A E_A^T + f_A f_A^T is near-singular, so the plain FP32 fit converges but lands far
    from the FP64 solution: this is the baseline the FP64 path is compared with. Its results are
    finite and most voxels converge."""
    design = _design(msmt_fixture)
    signals = _signals(msmt_fixture, 512, seed=11)[256:]  # the plausible half
    x64 = _device_fit(design, signals)[0]
    got, st = _plain_fp32(design, signals)
    ok = st == 0
    assert ok.mean() >= 0.9
    assert np.isfinite(got[ok]).all()
    rel = np.abs(got - x64).max(axis=1) / np.abs(x64).max(axis=1)
    print(f"plain FP32 LSI on MSMT: {ok.mean():.3f} converged, rel median {np.median(rel[ok]):.2e}, "
          f"max {rel[ok].max():.2e}")
