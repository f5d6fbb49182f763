"""GRL: the multi-tissue fit with damped Richardson-Lucy FOD solves at both resolutions.

On the CPU the oracle against the reference's numpy restatement
(tests/sd/reference_solvers.py:fit_multi_tissue_voxel) on the MATLAB and synthetic cases of
tests/sd/test_grl.py (tests/golden/grl.npz); on the GPU fit_multi_tissue with dRL solvers
(drl_kernel on each round's listed voxels, drl_kernel_wide for the 600-direction kernel of two
anisotropic responses) against the same fixtures at the reference's bounds, the solvers DRL
prepares per stage, the asynchronous call, and SDModel's GRL method against the oracle."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN

# The reference's bounds between its compiled fit and the numpy restatement
# (tests/sd/test_grl.py:27-32).
FOD_RTOL = 1e-10
FRACTION_ATOL = 1e-12
CASES = ["matlab", "synthetic"]
LR_ITER, HR_ITER = 200, 600  # asked for; a multi-tissue solve runs one fewer from 1e-6
GRL_FRACTION_TOL = 1e-3
MULTI_TISSUE_INIT = 1e-6


@pytest.fixture(scope="module")
def grl_fixture():
    return dict(np.load(GOLDEN / "grl.npz"))


def _kernel(z, name, tag):
    return {"k_aniso": z[f"{name}_{tag}_k_aniso"], "k_iso": z[f"{name}_{tag}_k_iso"],
            "w_k_iso": z[f"{name}_{tag}_w_k_iso"], "w_k_aniso": z[f"{name}_{tag}_w_k_aniso"],
            "blocks": [tuple(int(x) for x in b) for b in z[f"{name}_{tag}_blocks"]]}


def _oracle_grl(oracle, z, name, rows):
    return oracle.fit_multi_tissue(
        z[f"{name}_signals"][rows], z["weights"], _kernel(z, name, "lr"), _kernel(z, name, "hr"), max_rounds=50,
        fraction_tol=GRL_FRACTION_TOL, final_tol=1e-2, n_threads=8,
        lr_drl={"nu": float(z[f"{name}_lr_nu"]), "n_iter": LR_ITER - 1, "init": MULTI_TISSUE_INIT},
        hr_drl={"nu": float(z[f"{name}_hr_nu"]), "n_iter": HR_ITER - 1, "init": MULTI_TISSUE_INIT})


def _check(fods, fractions, ref_fods, ref_fractions):
    np.testing.assert_allclose(fods, ref_fods, rtol=FOD_RTOL, atol=0)
    np.testing.assert_array_equal(fractions == 0, ref_fractions == 0)
    np.testing.assert_allclose(fractions, ref_fractions, rtol=0, atol=FRACTION_ATOL)


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_the_reference_restatement(oracle, grl_fixture, name):
    """All 216 MATLAB voxels; 40 of the synthetic ones (their 600-direction final solves take the
    CPU most of its time)."""
    z = grl_fixture
    rows = slice(None) if name == "matlab" else slice(0, 40)
    fods, fractions = _oracle_grl(oracle, z, name, rows)
    _check(fods, fractions, z[f"{name}_fods"][rows], z[f"{name}_fractions"][rows])


def test_oracle_grl_does_not_depend_on_thread_count(oracle, grl_fixture):
    """The oracle's GRL of 48 MATLAB voxels, the same bit for bit on 1 and 5 threads."""
    z = grl_fixture
    kw = dict(max_rounds=50, fraction_tol=GRL_FRACTION_TOL, final_tol=1e-2,
              lr_drl={"nu": float(z["matlab_lr_nu"]), "n_iter": LR_ITER - 1, "init": MULTI_TISSUE_INIT},
              hr_drl={"nu": float(z["matlab_hr_nu"]), "n_iter": HR_ITER - 1, "init": MULTI_TISSUE_INIT})
    args = (z["matlab_signals"][:48], z["weights"], _kernel(z, "matlab", "lr"), _kernel(z, "matlab", "hr"))
    one = oracle.fit_multi_tissue(*args, n_threads=1, **kw)
    five = oracle.fit_multi_tissue(*args, n_threads=5, **kw)
    np.testing.assert_array_equal(one[0], five[0])
    np.testing.assert_array_equal(one[1], five[1])


def test_fixture_cases_cover_zero_fractions_and_two_fibre_blocks(grl_fixture):
    """tests/sd/test_grl.py:144-149: the synthetic voxels zero some tissues, and the final fit of
    the two-response kernel has one fraction per block."""
    z = grl_fixture
    fr = z["synthetic_fractions"]
    assert fr.shape[1] == 4 and z["synthetic_hr_k_aniso"].shape[1] == 600
    assert (fr == 0).any(axis=0)[1:].all()
    assert (fr > 0.05).any(axis=0).all()
    np.testing.assert_allclose(fr.sum(axis=1), 1.0, rtol=1e-12)


def test_drl_prepares_each_stage_as_the_reference(monkeypatch):
    """DRL._prepare (src/larmor/sd/solvers.py:123-148): a single-tissue solve starts at 1/c with
    num_iter iterations, a multi-tissue stage at 1e-6 with one iteration fewer than asked
    (num_iter at low resolution, hr_num_iter at high)."""
    from larmor_b200 import _core
    from larmor_b200.sd import DRL
    from larmor_b200.sd import solvers
    from larmor_b200.sd.solvers import Stage

    made = []
    monkeypatch.setattr(solvers, "calibrate_drl_nu", lambda kernel, bvals, adc, scale: 0.25)
    monkeypatch.setattr(_core.FodSolver, "drl", staticmethod(lambda k_t, k_t_k, **kw: made.append(kw) or kw))

    class _K:
        w_k_aniso = np.ones((5, 4))

    drl = DRL(num_iter=120, hr_num_iter=480)
    for stage in (Stage.SINGLE, Stage.LOW_RES, Stage.HIGH_RES):
        drl._prepare(_K(), np.zeros(5), stage)
    assert made == [dict(nu=0.25, n_iter=120, init=0.25), dict(nu=0.25, n_iter=119, init=1e-6),
                    dict(nu=0.25, n_iter=479, init=1e-6)]


def test_grl_model_takes_one_anisotropic_response():
    from larmor_b200.sd import DRL, AnisotropicRF, IsotropicRF, SDModel

    rfs = [AnisotropicRF([1.7e-3, 0.2e-3, 0.2e-3], 0.0), IsotropicRF(0.7e-3), IsotropicRF(3e-3)]
    model = SDModel(rfs, method="GRL")
    assert isinstance(model.method.default_solver(), DRL) and model.is_multi_tissue
    with pytest.raises(ValueError, match="exactly one anisotropic"):
        SDModel([rfs[0], AnisotropicRF([1.5e-3, 0.9e-3, 0.1e-3], 0.0), rfs[1]], method="GRL")


# ---- GPU -----------------------------------------------------------------------------------


def _device_case(z, name, lr_nu, hr_nu):
    from larmor_b200 import _core

    def kern(tag):
        k = _kernel(z, name, tag)
        return _core.DeconvKernel(np.ascontiguousarray(k["k_aniso"]), np.ascontiguousarray(k["k_iso"]),
                                  np.ascontiguousarray(k["w_k_iso"]), k["blocks"])

    def solver(tag, nu, n_iter):
        w = z[f"{name}_{tag}_w_k_aniso"]
        return _core.FodSolver.drl(np.ascontiguousarray(w.T), np.ascontiguousarray(w.T @ w), nu=nu,
                                   n_iter=n_iter - 1, init=MULTI_TISSUE_INIT)

    return kern("lr"), solver("lr", lr_nu, LR_ITER), kern("hr"), solver("hr", hr_nu, HR_ITER)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_grl_matches_the_reference_restatement(cuda, grl_fixture, name):
    """tests/sd/test_grl.py:130-141 on the device: the fixture's nu, MATLAB's iteration counts."""
    from larmor_b200 import _core

    z = grl_fixture
    lr, lr_solver, hr, hr_solver = _device_case(z, name, float(z[f"{name}_lr_nu"]), float(z[f"{name}_hr_nu"]))
    fods, fractions = _core.fit_multi_tissue(np.ascontiguousarray(z[f"{name}_signals"]), z["weights"], lr, lr_solver,
                                             hr, hr_solver, 50, GRL_FRACTION_TOL, 1e-2, 1)
    _check(fods, fractions, z[f"{name}_fods"], z[f"{name}_fractions"])


@pytest.mark.gpu
def test_gpu_grl_with_the_solvers_drl_prepares(cuda, grl_fixture):
    """The synthetic case through DRL()._prepare per stage (nu calibrated on the device) and the
    package's fit_multi_tissue, as tests/sd/test_grl.py:105-108 builds it."""
    from larmor_b200.sd import DRL
    from larmor_b200.sd.kernel import Kernel
    from larmor_b200.sd.rf import AnisotropicRF, IsotropicRF
    from larmor_b200.sd.solvers import Stage, calibrate_drl_nu, fit_multi_tissue
    from larmor_b200.sd.sphere import DIRS_300, get_dirs

    z = grl_fixture
    bvals, bvecs, weights = z["bvals"], z["bvecs"], z["weights"]
    rfs = [AnisotropicRF([1.7e-3, 0.2e-3, 0.2e-3], 0.0), AnisotropicRF([1.5e-3, 0.9e-3, 0.1e-3], 0.0),
           IsotropicRF(0.7e-3), IsotropicRF(3e-3)]
    lr = Kernel(rfs, bvals, bvecs, dirs=get_dirs(min(len(bvals), 45)), weights=weights)
    hr = Kernel(rfs, bvals, bvecs, dirs=DIRS_300, weights=weights)
    np.testing.assert_allclose(hr.w_k_aniso, z["synthetic_hr_w_k_aniso"], rtol=1e-14, atol=0)
    np.testing.assert_allclose(lr.w_k_aniso, z["synthetic_lr_w_k_aniso"], rtol=1e-14, atol=0)
    assert calibrate_drl_nu(lr, bvals) == pytest.approx(float(z["synthetic_lr_nu"]), rel=1e-10)
    assert calibrate_drl_nu(hr, bvals) == pytest.approx(float(z["synthetic_hr_nu"]), rel=1e-10)
    fods, fractions = fit_multi_tissue(z["synthetic_signals"], lr, hr, DRL()._prepare(lr, bvals, Stage.LOW_RES),
                                       DRL()._prepare(hr, bvals, Stage.HIGH_RES), fraction_tol=GRL_FRACTION_TOL)
    _check(fods, fractions, z["synthetic_fods"], z["synthetic_fractions"])


@pytest.mark.gpu
def test_gpu_grl_async_equals_the_waiting_call(cuda, grl_fixture):
    """lar_fit_multi_tissue_async with dRL stages (every round enqueued, the listed dRL reading its
    voxel count on the device) gives the waiting call's results bit for bit."""
    import torch

    from larmor_b200 import _core

    z = grl_fixture
    lr, lr_solver, hr, hr_solver = _device_case(z, "matlab", float(z["matlab_lr_nu"]), float(z["matlab_hr_nu"]))
    signals = np.ascontiguousarray(z["matlab_signals"])
    fods, fractions = _core.fit_multi_tissue(signals, z["weights"], lr, lr_solver, hr, hr_solver, 50,
                                             GRL_FRACTION_TOL, 1e-2, 1)
    dev = torch.device("cuda")
    v = len(signals)
    s = torch.from_numpy(signals).to(dev)
    out_f = torch.zeros((v, hr.ca), dtype=torch.float64, device=dev)
    out_p = torch.zeros((v, hr.nb + hr.ci), dtype=torch.float64, device=dev)
    rd = torch.zeros((v,), dtype=torch.int32, device=dev)
    _core.fit_multi_tissue_device(s, z["weights"], lr, lr_solver, hr, hr_solver, 50, GRL_FRACTION_TOL, 1e-2, out_f,
                                  out_p, rd, None, asynchronous=True)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out_f.cpu().numpy(), fods)
    np.testing.assert_array_equal(out_p.cpu().numpy(), fractions)
    assert 1 <= rd.min().item() and rd.max().item() <= 50


@pytest.mark.gpu
def test_gpu_grl_sd_model_matches_the_oracle(cuda, oracle):
    """SDModel(method="GRL") with one anisotropic and two isotropic responses against the oracle's
    GRL of the same S0-normalised signals and the kernels and nu the model prepares."""
    from larmor_b200.sd import DRL, AnisotropicRF, IsotropicRF, SDModel
    from larmor_b200.sd.model import to_sh
    from larmor_b200.sd.solvers import calibrate_drl_nu
    from larmor_b200.synthetic import mfod_signals, mfod_table
    from larmor_b200.types import Volume

    rng = np.random.default_rng(5)
    gtab = mfod_table(rng)
    data = mfod_signals(rng, gtab, 64).reshape(4, 4, 4, -1).astype(np.float32)
    rfs = [AnisotropicRF([1.7e-3, 0.2e-3, 0.2e-3], 0.0), IsotropicRF(0.8e-3), IsotropicRF(3e-3)]
    model = SDModel(rfs, method="GRL")
    fit = model.fit(Volume(data, np.eye(4)), gtab)
    s = data.reshape(-1, data.shape[-1]).astype(np.float64)
    norm = np.minimum(s / s[:, gtab.b0_mask].mean(axis=1)[:, None], 1.0)
    hr, lr, _, _ = model._prepare(DRL(), gtab.bvals, gtab.bvecs)
    lrd = dict(k_aniso=lr.k_aniso, k_iso=lr.k_iso, w_k_iso=lr.w_k_iso, w_k_aniso=lr.w_k_aniso)
    hrd = dict(k_aniso=hr.k_aniso, k_iso=hr.k_iso, w_k_iso=hr.w_k_iso, w_k_aniso=hr.w_k_aniso,
               blocks=[(b.start, b.stop) for b in hr.aniso_blocks])
    rfods, rfr = oracle.fit_multi_tissue(
        norm, lr.weights, lrd, hrd, max_rounds=50, fraction_tol=GRL_FRACTION_TOL, final_tol=1e-2, n_threads=8,
        lr_drl={"nu": calibrate_drl_nu(lr, gtab.bvals), "n_iter": LR_ITER - 1, "init": MULTI_TISSUE_INIT},
        hr_drl={"nu": calibrate_drl_nu(hr, gtab.bvals), "n_iter": HR_ITER - 1, "init": MULTI_TISSUE_INIT})
    ref_sh = to_sh(rfods, fit.lmax, "tournier", exact_integral=True)
    # The maps are float32, as the reference's.
    np.testing.assert_allclose(fit.fods[0].reshape(-1, ref_sh.shape[1]), ref_sh, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(fit.tissue_fractions.reshape(-1, 3), rfr, rtol=0, atol=1e-6)


@pytest.mark.gpu
def test_gpu_grl_does_not_depend_on_thread_count(cuda, grl_fixture):
    """tests/sd/test_grl.py:152-161: the fit is the same bit for bit for any n_threads."""
    from larmor_b200 import _core

    z = grl_fixture
    lr, lr_solver, hr, hr_solver = _device_case(z, "matlab", float(z["matlab_lr_nu"]), float(z["matlab_hr_nu"]))
    signals = np.ascontiguousarray(z["matlab_signals"])
    one = _core.fit_multi_tissue(signals, z["weights"], lr, lr_solver, hr, hr_solver, 50, GRL_FRACTION_TOL, 1e-2, 1)
    for n_threads in (2, 7):
        got = _core.fit_multi_tissue(signals, z["weights"], lr, lr_solver, hr, hr_solver, 50, GRL_FRACTION_TOL, 1e-2,
                                     n_threads)
        np.testing.assert_array_equal(got[0], one[0])
        np.testing.assert_array_equal(got[1], one[1])


@pytest.mark.gpu
@pytest.mark.parametrize(("mismatch", "resolution"),
                         [("directions", "low-resolution"), ("measurements", "high-resolution")])
def test_gpu_grl_refuses_a_solver_that_does_not_match_its_kernel(cuda, grl_fixture, mismatch, resolution):
    """tests/sd/test_grl.py:316-335: a dRL solver with another kernel's directions, or one
    measurement short, is refused with the reference's message."""
    from larmor_b200 import _core

    z = grl_fixture
    lr, lr_solver, hr, hr_solver = _device_case(z, "matlab", float(z["matlab_lr_nu"]), float(z["matlab_hr_nu"]))
    if mismatch == "directions":
        lr_solver = hr_solver  # 300 directions against the low-resolution kernel's 33
    else:
        k = z["matlab_hr_w_k_aniso"][:-1]
        hr_solver = _core.FodSolver.drl(np.ascontiguousarray(k.T), np.ascontiguousarray(k.T @ k), nu=0.01,
                                        n_iter=10, init=0.1)
    with pytest.raises(ValueError, match=f"the {resolution} solver .* does not match its kernel"):
        _core.fit_multi_tissue(np.ascontiguousarray(z["matlab_signals"]), z["weights"], lr, lr_solver, hr,
                               hr_solver, 50, GRL_FRACTION_TOL, 1e-2, 1)


# ---- lsqnonneg (the fraction fits' NNLS, one problem) --------------------------------------


def _fraction_problems():
    """tests/sd/test_grl.py:165-177: 200 seeded problems of 2-6 decaying-exponential columns on
    32 measurements (b = 0, 1000, 2000, 3000 x 8), a third of the true fractions 0, plus noise."""
    rng = np.random.default_rng(1)
    b = np.repeat([0.0, 1000.0, 2000.0, 3000.0], 8)
    problems = []
    for _ in range(200):
        n = int(rng.integers(2, 7))
        c = np.exp(-np.outer(b, np.sort(rng.uniform(0.1e-3, 3e-3, n))))
        x = rng.dirichlet(np.ones(n))
        x[rng.random(n) < 0.3] = 0.0
        d = c @ x + rng.uniform(0.0, 0.02) * rng.standard_normal(len(b))
        problems.append((np.ascontiguousarray(c), d))
    return problems


def test_oracle_nnls_matches_scipy_on_the_fraction_problems(oracle):
    """The oracle's solve_nnls against scipy's nnls at the reference's bound (atol 1e-10)."""
    from scipy.optimize import nnls

    for c, d in _fraction_problems():
        x, _ = oracle.nnls(c, d)
        expected, _ = nnls(c, d)
        np.testing.assert_array_equal(x == 0, expected == 0)
        np.testing.assert_allclose(x, expected, rtol=0, atol=1e-10)


def test_lsqnonneg_refuses_bad_arguments():
    """tests/sd/test_grl.py:223-225, and the binding's type and width checks (before any
    device work)."""
    from larmor_b200 import _core

    with pytest.raises(ValueError, match="c must be"):
        _core.lsqnonneg(np.ones((32, 3)), np.ones(31))
    with pytest.raises(TypeError):
        _core.lsqnonneg(np.ones((32, 3), dtype=np.float32), np.ones(32))
    with pytest.raises(ValueError, match="C-contiguous"):
        _core.lsqnonneg(np.asfortranarray(np.ones((32, 3))), np.ones(32))
    with pytest.raises(ValueError, match="at most 16 columns"):
        _core.lsqnonneg(np.ones((32, 17)), np.ones(32))


@pytest.mark.gpu
@pytest.mark.parametrize(("against", "tol_x", "atol"), [("scipy", None, 1e-10), ("oracle", None, 1e-10),
                                                        ("oracle", 1e-2, 1e-13)])
def test_gpu_lsqnonneg_matches_the_reference_nnls(cuda, oracle, against, tol_x, atol):
    """tests/sd/test_grl.py:185-208: the same zero coefficients and values within atol, against
    scipy (exact NNLS) and the oracle's solve_nnls (MATLAB's TolX rule)."""
    from scipy.optimize import nnls

    from larmor_b200 import _core

    n_zeros = 0
    for c, d in _fraction_problems():
        x = _core.lsqnonneg(c, d, tol_x)
        expected = nnls(c, d)[0] if against == "scipy" else oracle.nnls(c, d, tol_x)[0]
        np.testing.assert_array_equal(x == 0, expected == 0)
        np.testing.assert_allclose(x, expected, rtol=0, atol=atol)
        n_zeros += int((x == 0).sum())
    assert n_zeros > 0


@pytest.mark.gpu
def test_gpu_lsqnonneg_tol_x_zeroes_a_small_coefficient(cuda):
    """tests/sd/test_grl.py:211-220: a 0.5% compartment is kept at the default TolX and dropped
    at 1e-2."""
    from larmor_b200 import _core

    b = np.repeat([0.0, 1000.0, 2000.0, 3000.0], 8)
    c = np.ascontiguousarray(np.exp(-np.outer(b, [0.7e-3, 3e-3])))
    d = c @ np.array([0.995, 0.005])
    assert (_core.lsqnonneg(c, d) > 0).all()
    x = _core.lsqnonneg(c, d, 1e-2)
    assert x[1] == 0
    np.testing.assert_allclose(x[0], 1.0, atol=1e-2)


@pytest.mark.gpu
def test_gpu_grl_on_the_tensor_cores_stays_within_the_fod_tolerance(cuda, grl_fixture):
    """The MATLAB case (one 300-direction response) with the final high-resolution solve in the
    tensor-core mode (tf32x3), the low-resolution rounds (44 directions) in FP64. Each of the
    599 multiplicative iterations carries the FP32-level error of its product (~1e-6 relative),
    and the iteration carries it along: the FODs stay within 5e-4 of the voxel's largest
    amplitude (median ~5e-5; 1e-4 holds at dRL's 200 iterations, test_drl.py) and the fractions
    within 1e-4 of the reference's."""
    from larmor_b200 import _core

    z = grl_fixture
    name = "matlab"
    lr, lr_solver, hr, hr_solver = _device_case(z, name, float(z[f"{name}_lr_nu"]), float(z[f"{name}_hr_nu"]))
    hr_solver.set_precision("tf32x3")
    fods, fractions = _core.fit_multi_tissue(np.ascontiguousarray(z[f"{name}_signals"]), z["weights"], lr, lr_solver,
                                             hr, hr_solver, 50, GRL_FRACTION_TOL, 1e-2, 1)
    hr_solver.check_errors()
    ref, ref_fr = z[f"{name}_fods"], z[f"{name}_fractions"]
    rel = np.abs(fods - ref).max(axis=1) / np.abs(ref).max(axis=1)
    print(f"GRL tensor-core final solve: FOD rel max {rel.max():.3e}, fractions abs max "
          f"{np.abs(fractions - ref_fr).max():.3e}")
    assert rel.max() <= 5e-4 and np.median(rel) <= 1e-4
    assert np.abs(fractions - ref_fr).max() <= 1e-4


def _wide_and_rank_deficient_problems():
    """Seeded problems the fraction fits never build: fewer rows than columns (the QR's wide
    case, rank at most the row count) and duplicated columns (rank-deficient), where the
    column-pivoted QR's rank threshold decides which columns get zero."""
    rng = np.random.default_rng(12)
    problems = []
    for _ in range(40):
        m, n = int(rng.integers(2, 6)), int(rng.integers(6, 12))
        c = np.abs(rng.standard_normal((m, n)))
        problems.append((np.ascontiguousarray(c), c @ np.abs(rng.standard_normal(n)) + 0.1 * rng.standard_normal(m)))
    for _ in range(40):
        m, n = 24, int(rng.integers(3, 8))
        base = np.exp(-np.outer(np.linspace(0, 3e3, m), rng.uniform(0.1e-3, 3e-3, n)))
        dup = int(rng.integers(0, n))
        c = np.ascontiguousarray(np.concatenate([base, base[:, dup:dup + 1]], axis=1))
        problems.append((c, c @ rng.dirichlet(np.ones(n + 1)) + 0.01 * rng.standard_normal(m)))
    return problems


@pytest.mark.gpu
def test_gpu_lsqnonneg_matches_the_oracle_on_wide_and_rank_deficient_problems(cuda, oracle):
    """The device NNLS against the oracle's (the reference's ColPivHouseholderQR rank rule) on
    wide problems (m < n) and problems with a duplicated column: the same zero coefficients and
    values within 1e-10 of the largest."""
    from larmor_b200 import _core

    for c, d in _wide_and_rank_deficient_problems():
        x = _core.lsqnonneg(c, d)
        expected = oracle.nnls(c, d)[0]
        np.testing.assert_array_equal(x == 0, expected == 0)
        np.testing.assert_allclose(x, expected, rtol=0, atol=1e-10 * max(1.0, np.abs(expected).max()))
