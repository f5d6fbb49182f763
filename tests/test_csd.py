"""Single-shell CSD: the problem's matrices against the reference's own (tests/golden/csd.npz),
the oracle's solve against the reference's known-answer tests (tests/sd/test_csd.py: the
directions of one fibre and of crossings, the suppressed negative lobes) and against its fixed
point, the settings' checks on the CPU; on the GPU the lar_fit_csd solve against the oracle and
the same known-answer tests through CSDModel."""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import GOLDEN

SOLVERS = [
    dict(),
    dict(init_lmax=2, neg_lambda=0.5, threshold=0.1, max_iter=20),
    dict(norm_lambda=2.0),
]


@pytest.fixture(scope="module")
def csd_fixture():
    return dict(np.load(GOLDEN / "csd.npz"))


def _solver(z, i):
    from larmor_b200.sd import CSDSolver

    kw = dict(SOLVERS[i]) if i < 3 else dict(directions=z["p3_directions"])
    return CSDSolver(**kw)


def _problem(z, i):
    from larmor_b200.sd.csd_solver import csd_problem

    return csd_problem(z["bvecs"][1:], z["response"], int(z[f"p{i}_lmax"]), _solver(z, i))


@pytest.mark.parametrize("i", [0, 1, 2, 3])
def test_problem_matrices_are_the_reference_ones(csd_fixture, i):
    z = csd_fixture
    p = _problem(z, i)
    for name in ("initial", "forward", "constraint"):
        np.testing.assert_array_equal(getattr(p, name), z[f"p{i}_{name}"])
    assert p.norm_weight == float(z[f"p{i}_norm_weight"])
    assert p.threshold == float(z[f"p{i}_threshold"])
    assert p.max_iter == int(z[f"p{i}_max_iter"])


def _peak_directions(oracle, peaks_fixture, fods):
    from larmor_b200.sd.sh import build_basis_matrix
    from larmor_b200.sd.sphere import get_theta_phi

    v, nb = peaks_fixture["vertices"], peaks_fixture["neighbours"]
    t, p = get_theta_phi(v)
    on = np.ascontiguousarray(fods @ build_basis_matrix(t, p, 8).T)
    return oracle.peaks_chunk(np.ascontiguousarray(fods), 8, on, v, nb, 3, 0.1, 0.0)


def _check_known_answers(fods, z, dirs, amps):
    """tests/sd/test_csd.py:67-87: each fibre within 2 degrees of a peak, as many peaks as
    fibres; the constrained FOD of the noisy crossing keeps less than a third of the linear
    estimate's relative negative lobe."""
    for i in range(4):
        fib = z["fibres"][i]
        fib = fib[np.isfinite(fib[:, 0])]
        found = dirs[i][np.isfinite(amps[i])]
        assert len(found) == len(fib)
        cos = np.abs(found @ fib.T).max(axis=0)
        assert np.degrees(np.arccos(cos.clip(max=1))).max() < 2.0


def _negative_ratio(fod):
    from larmor_b200.sd.sh import build_basis_matrix
    from larmor_b200.sd.sphere import get_dirs, get_theta_phi

    amp = build_basis_matrix(*get_theta_phi(get_dirs(2000)), 8) @ fod
    return -amp.min() / amp.max()


def test_oracle_passes_the_reference_known_answer_tests(oracle, csd_fixture, peaks_fixture):
    z = csd_fixture
    p = _problem(z, 0)
    sig = np.maximum(z["signals"], 0.0)
    fods, conv = oracle.fit_csd(sig, p.initial, p.forward, p.constraint, p.norm_weight, p.threshold, p.max_iter)
    assert conv.all()
    dirs, amps = _peak_directions(oracle, peaks_fixture, fods)
    _check_known_answers(fods, z, dirs, amps)
    linear, _ = oracle.fit_csd(sig[4:], p.initial, p.forward, p.constraint, p.norm_weight, p.threshold, 0)
    assert _negative_ratio(fods[4]) < _negative_ratio(linear[0]) / 3


def _synthetic_shell(z, n, seed, noise=40.0):
    """n voxels of 1-3 fibres (Dirichlet(2) fractions) of the fixture's response on its shell,
    Gaussian noise of `noise` signal units."""
    from larmor_b200.sd.rf import ZonalSHRF

    rng = np.random.default_rng(seed)
    rf = ZonalSHRF(bvals=np.array([1000.0]), coefficients=z["response"][None])
    b, g = z["bvals"][1:], z["bvecs"][1:]
    out = np.zeros((n, len(b)))
    k = rng.integers(1, 4, size=n)
    w = rng.dirichlet([2.0, 2.0, 2.0], size=n) * (np.arange(3)[None] < k[:, None])
    w /= w.sum(axis=1, keepdims=True)
    dirs = rng.normal(size=(n, 3, 3))
    dirs /= np.linalg.norm(dirs, axis=2, keepdims=True)
    for f in range(3):
        out += w[:, f:f + 1] * rf.signal(b, g, dirs[:, f]).T
    return out + rng.normal(0, noise, out.shape)


@pytest.mark.parametrize("i", [0, 1, 2, 3])
def test_oracle_solutions_are_fixed_points(oracle, csd_fixture, i):
    """Where the set repeated, the FOD solves the normal equations of that set: with S the rows
    where C f < threshold, (M^T M + norm_weight I + C_S^T C_S) f = M^T s."""
    z = csd_fixture
    p = _problem(z, i)
    sig = np.maximum(_synthetic_shell(z, 200, 7 + i), 0.0)
    fods, conv = oracle.fit_csd(sig, p.initial, p.forward, p.constraint, p.norm_weight, p.threshold, p.max_iter,
                                n_threads=4)
    assert conv.mean() > 0.9
    gram = p.forward.T @ p.forward + p.norm_weight * np.eye(p.forward.shape[1])
    for f, s in zip(fods[conv], sig[conv]):
        rows = p.constraint[p.constraint @ f < p.threshold]
        x = np.linalg.solve(gram + rows.T @ rows, p.forward.T @ s)
        np.testing.assert_allclose(f, x, rtol=0, atol=1e-10 * np.abs(x).max())


def test_max_iter_zero_is_the_linear_estimate(oracle, csd_fixture):
    z = csd_fixture
    p = _problem(z, 1)
    sig = np.maximum(z["signals"], 0.0)
    fods, conv = oracle.fit_csd(sig, p.initial, p.forward, p.constraint, p.norm_weight, p.threshold, 0)
    expected = np.zeros_like(fods)
    expected[:, : p.initial.shape[0]] = sig @ p.initial.T
    np.testing.assert_allclose(fods, expected, rtol=1e-13, atol=1e-12)
    assert conv.all()


def test_settings_and_models_that_cannot_be_solved_are_refused():
    from larmor_b200.sd import CSDModel, CSDSolver, IsotropicRF, ZonalSHRF
    from larmor_b200.sd.csd_solver import csd_problem

    with pytest.raises(ValueError, match="non-zero"):
        CSDSolver(directions=np.array([[0.0, 0.0, 1.0], [0.0, 0.0, 0.0]]))
    for kw in (dict(neg_lambda=-1.0), dict(norm_lambda=math.inf), dict(threshold=math.nan), dict(max_iter=-1),
               dict(init_lmax=3)):
        with pytest.raises(ValueError):
            CSDSolver(**kw)
    with pytest.raises(ValueError, match="ZonalSHRF"):
        CSDModel(IsotropicRF(3e-3))
    with pytest.raises(ValueError, match="lmax"):
        CSDModel(lmax=7)
    response = np.array([1800.0, -700.0, 180.0, -35.0, 5.0])
    rng = np.random.default_rng(1)
    dirs = rng.normal(size=(60, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    # lmax 10 has 66 coefficients for 60 measurements: singular without the norm penalty.
    with pytest.raises(ValueError, match="singular"):
        csd_problem(dirs, response, 10, CSDSolver(norm_lambda=0.0))
    with pytest.raises(ValueError, match="at least 6"):
        csd_problem(dirs[:5], response, 8, CSDSolver())
    with pytest.raises(ValueError, match="positive l = 0"):
        csd_problem(dirs, -response, 8, CSDSolver())
    _ = ZonalSHRF


def test_fit_csd_binding_refuses_bad_arguments(csd_fixture):
    from larmor_b200 import _core

    z = csd_fixture
    p = _problem(z, 0)
    args = dict(signals=np.zeros((3, 60)), initial=p.initial, forward=p.forward, constraint=p.constraint,
                norm_weight=p.norm_weight, threshold=p.threshold, max_iter=50, n_threads=1)
    for name, value, message in [("signals", np.zeros((3, 59)), "shapes do not match"),
                                 ("signals", np.zeros((60, 6)).T, "C-contiguous"),
                                 ("constraint", np.zeros((300, 44)), "shapes do not match"),
                                 ("max_iter", -1, "max_iter must be at least 0"),
                                 ("n_threads", 0, "n_threads must be at least 1")]:
        bad = dict(args)
        bad[name] = value
        with pytest.raises(ValueError, match=message):
            _core.fit_csd(**bad)
    bad = dict(args)
    bad["signals"] = np.zeros((3, 60), dtype=np.float32)
    with pytest.raises(TypeError):
        _core.fit_csd(**bad)


# ---- GPU -----------------------------------------------------------------------------------


def _gpu_vs_oracle(oracle, p, sig, rtol=1e-9):
    from larmor_b200 import _core

    fods, conv = _core.fit_csd(sig, p.initial, p.forward, p.constraint, p.norm_weight, p.threshold, p.max_iter, 1)
    ref, rconv = oracle.fit_csd(sig, p.initial, p.forward, p.constraint, p.norm_weight, p.threshold, p.max_iter,
                                n_threads=8)
    # Rounding can flip a direction sitting on the threshold in one iteration; the fits then
    # take another path to the same fixed point. Converged flags agree on all but a few voxels,
    # and the FODs of voxels converged in both agree to rounding amplified by the system's
    # condition.
    both = conv & rconv
    assert (conv == rconv).mean() > 0.999
    scale = np.abs(ref).max(axis=1, keepdims=True)
    err = (np.abs(fods - ref) / scale)[both]
    assert np.quantile(err.max(axis=1), 0.999) <= rtol
    return fods, conv


@pytest.mark.gpu
@pytest.mark.parametrize("i", [0, 1, 2, 3])
def test_gpu_solve_matches_the_oracle(cuda, oracle, csd_fixture, i):
    z = csd_fixture
    p = _problem(z, i)
    sig = np.ascontiguousarray(np.maximum(_synthetic_shell(z, 5000, 30 + i), 0.0))
    _gpu_vs_oracle(oracle, p, sig)


@pytest.mark.gpu
def test_gpu_linear_estimate_and_known_answers(cuda, oracle, csd_fixture, peaks_fixture):
    from larmor_b200 import _core

    z = csd_fixture
    p = _problem(z, 0)
    sig = np.ascontiguousarray(np.maximum(z["signals"], 0.0))
    lin, conv = _core.fit_csd(sig, p.initial, p.forward, p.constraint, p.norm_weight, p.threshold, 0, 1)
    assert conv.all()
    expected = np.zeros_like(lin)
    expected[:, : p.initial.shape[0]] = sig @ p.initial.T
    np.testing.assert_allclose(lin, expected, rtol=1e-13, atol=1e-12)
    fods, conv = _core.fit_csd(sig, p.initial, p.forward, p.constraint, p.norm_weight, p.threshold, 50, 1)
    assert conv.all()
    dirs, amps = _peak_directions(oracle, peaks_fixture, fods)
    _check_known_answers(fods, z, dirs, amps)
    assert _negative_ratio(fods[4]) < _negative_ratio(lin[4]) / 3


@pytest.mark.gpu
def test_csd_model_fits_a_volume_like_the_oracle(cuda, oracle, csd_fixture):
    """CSDModel end to end: a 12x10x8 volume of the fixture's shell plus two b0s and a second
    shell it leaves out, NaN samples in some voxels; the FODs against the oracle's solve of the
    same samples, and the peaks of the single fibres."""
    from larmor_b200.sd import CSDModel, ZonalSHRF
    from larmor_b200.types import GradientTable, Volume

    z = csd_fixture
    rng = np.random.default_rng(12)
    n = 12 * 10 * 8
    shell = _synthetic_shell(z, n, 40)
    other = shell * 0.5
    data = np.concatenate([np.full((n, 2), 2000.0), shell, other], axis=1).astype(np.float32)
    data[rng.random(n) < 0.02, 70] = np.nan  # in the fitted shell: NaN FODs
    data[rng.random(n) < 0.02, 5] = np.nan  # in the shell left out: no effect
    b = np.concatenate([[0.0, 0.0], z["bvals"][1:], np.full(60, 2000.0)])
    g = np.concatenate([np.zeros((2, 3)), z["bvecs"][1:], z["bvecs"][1:]])
    gtab = GradientTable(b, g)
    response = ZonalSHRF(bvals=np.array([1000.0, 2000.0]), coefficients=np.vstack([z["response"] * 0.0,
                                                                                  z["response"]]))
    # The fitted shell is b = 2000 (the highest): its response row is the fixture's.
    vol = Volume(data.reshape(12, 10, 8, -1), np.eye(4))
    mask = np.ones((12, 10, 8), dtype=bool)
    mask[0, 0, :] = False
    fit = CSDModel(response).fit(vol, gtab, mask)
    p = _problem(z, 0)
    sig = data[mask.reshape(-1)][:, 62:].astype(np.float64)
    finite = np.isfinite(sig).all(axis=1)
    ref, _ = oracle.fit_csd(np.maximum(sig[finite], 0.0), p.initial, p.forward, p.constraint, p.norm_weight,
                            p.threshold, p.max_iter, n_threads=8)
    got = fit.fods[0][mask]
    assert (~finite).any()
    assert np.isnan(got[~finite]).all() and not np.isnan(got[finite]).any()
    # The model's maps are float32, as the reference's: the FP64 solve rounded once.
    assert fit.fods[0].dtype == np.float32
    scale = np.abs(ref).max(axis=1, keepdims=True)
    assert np.quantile((np.abs(got[finite] - ref) / scale).max(axis=1), 0.99) <= 2e-7
    assert (fit.fods[0][~mask] == 0).all()
