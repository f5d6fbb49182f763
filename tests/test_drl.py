"""Damped Richardson-Lucy: the oracle against the reference's numpy solver on the cases of
tests/sd/test_drl.py (tests/golden/drl.npz: the calibration, single-tissue and multi-tissue-start
settings, rtol 1e-10), the settings' and bindings' checks on the CPU; on the GPU the dRL solver
(FodSolver.drl + fit_single_tissue, drl_kernel on the FP64 tensor cores) against the same
fixtures, the oracle, the calibration of nu and a single-tissue SDModel fit."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN

RTOL = 1e-10  # the reference's bound between its compiled and numpy solvers
SETTINGS = ["calibration", "single", "multi_start"]


@pytest.fixture(scope="module")
def drl_fixture():
    return dict(np.load(GOLDEN / "drl.npz"))


def _products(k):
    return np.ascontiguousarray(k.T), np.ascontiguousarray(k.T @ k)


@pytest.mark.parametrize("name", SETTINGS)
def test_oracle_matches_the_reference_solver(oracle, drl_fixture, name):
    z = drl_fixture
    k_t, k_t_k = _products(z["k"])
    got = oracle.drl(z["signals"], k_t, k_t_k, float(z[f"{name}_nu"]), 200, float(z[f"{name}_start"]), n_threads=4)
    np.testing.assert_allclose(got, z[f"{name}_fods"], rtol=RTOL, atol=0)


def test_fixture_voxels_converge_at_different_iterations(oracle, drl_fixture):
    """tests/sd/test_drl.py:119-129: some voxels stop within 100 iterations, some do not."""
    z = drl_fixture
    k_t, k_t_k = _products(z["k"])
    nu, start = float(z["single_nu"]), float(z["single_start"])
    half = oracle.drl(z["signals"], k_t, k_t_k, nu, 100, start)
    full = oracle.drl(z["signals"], k_t, k_t_k, nu, 200, start)
    converged = np.all(half == full, axis=1).sum()
    assert 0 < converged < len(z["signals"])


@pytest.mark.parametrize("settings", [{"num_iter": 0}, {"hr_num_iter": 0}, {"num_iter": -1}, {"target_adc": 0.0},
                                      {"target_adc": float("nan")}, {"nu_scale": 0.0}, {"nu_scale": float("inf")}])
def test_drl_refuses_bad_settings(settings):
    from larmor_b200.sd import DRL

    with pytest.raises(ValueError, match="must be"):
        DRL(**settings)


def test_drl_binding_refuses_bad_arguments(drl_fixture):
    from larmor_b200 import _core

    k_t, k_t_k = _products(drl_fixture["k"])
    with pytest.raises(ValueError, match="shapes do not match"):
        _core.FodSolver.drl(k_t, np.ascontiguousarray(k_t_k[:, :-1]), nu=0.1, n_iter=10, init=0.1)
    with pytest.raises(ValueError, match="n_iter must be at least 0"):
        _core.FodSolver.drl(k_t, k_t_k, nu=0.1, n_iter=-1, init=0.1)
    with pytest.raises(TypeError):
        _core.FodSolver.drl(k_t.astype(np.float32), k_t_k, nu=0.1, n_iter=10, init=0.1)


# ---- GPU -----------------------------------------------------------------------------------


def _device_drl(signals, k, nu, n_iter, start):
    from larmor_b200 import _core

    k_t, k_t_k = _products(k)
    solver = _core.FodSolver.drl(k_t, k_t_k, nu=nu, n_iter=n_iter, init=start)
    return _core.fit_single_tissue(np.ascontiguousarray(signals), solver, 1)


@pytest.mark.gpu
@pytest.mark.parametrize("name", SETTINGS)
def test_gpu_drl_matches_the_reference_solver(cuda, drl_fixture, name):
    z = drl_fixture
    got = _device_drl(z["signals"], z["k"], float(z[f"{name}_nu"]), 200, float(z[f"{name}_start"]))
    np.testing.assert_allclose(got, z[f"{name}_fods"], rtol=RTOL, atol=0)


@pytest.mark.gpu
def test_gpu_drl_convergence_and_edge_cases(cuda, drl_fixture):
    from larmor_b200 import _core

    z = drl_fixture
    nu, start = float(z["single_nu"]), float(z["single_start"])
    half = _device_drl(z["signals"], z["k"], nu, 100, start)
    full = _device_drl(z["signals"], z["k"], nu, 200, start)
    converged = np.all(half == full, axis=1).sum()
    assert 0 < converged < len(z["signals"])
    # No iteration: the start itself.
    np.testing.assert_array_equal(_device_drl(z["signals"][:5], z["k"], nu, 0, start), np.full((5, 300), start))
    k_t, k_t_k = _products(z["k"])
    solver = _core.FodSolver.drl(k_t, k_t_k, nu=nu, n_iter=200, init=start)
    assert _core.fit_single_tissue(np.zeros((0, 33)), solver, 1).shape == (0, 300)
    with pytest.raises(ValueError, match="measurements"):
        _core.fit_single_tissue(np.ascontiguousarray(z["signals"][:, :-1]), solver, 1)
    with pytest.raises(ValueError, match="n_threads"):
        _core.fit_single_tissue(z["signals"], solver, 0)


@pytest.mark.gpu
@pytest.mark.parametrize(("n_meas", "n_dirs", "n_vox"),
                         [(33, 300, 1000), (280, 300, 1000), (60, 45, 1000), (90, 130, 1000), (33, 600, 203),
                          (60, 450, 203)])
def test_gpu_drl_matches_the_oracle_on_more_voxels(cuda, oracle, n_meas, n_dirs, n_vox):
    """Voxel counts that are not a multiple of the tile (32 voxels; 8 past 320 directions) of random
    non-negative kernels, fibre and isotropic-like signals, NaN in a few."""
    rng = np.random.default_rng(n_meas + n_dirs)
    k = np.abs(rng.normal(size=(n_meas, n_dirs))) * np.exp(-rng.uniform(0, 3, size=(n_meas, 1)))
    fods = np.zeros((n_vox, n_dirs))
    for f in fods:
        f[rng.choice(n_dirs, size=rng.integers(1, 4), replace=False)] = rng.dirichlet([1.0, 1.0, 1.0])[:1]
    signals = fods @ k.T + rng.uniform(0, 0.05, size=(n_vox, 1)) * np.abs(rng.normal(size=(n_vox, n_meas)))
    signals[:n_vox // 2:97, 3] = np.nan
    k_t, k_t_k = _products(k)
    nu = 0.02
    got = _device_drl(signals, k, nu, 150, 1.0 / n_dirs)
    ref = oracle.drl(signals, k_t, k_t_k, nu, 150, 1.0 / n_dirs, n_threads=8)
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    np.testing.assert_allclose(got, ref, rtol=1e-9, atol=0)


@pytest.mark.gpu
def test_gpu_calibration_and_single_tissue_model(cuda, oracle, drl_fixture):
    """calibrate_drl_nu on the device against the fixture's nu (the reference's numpy solver), and
    SDModel with one anisotropic response and the DRL solver against the oracle's solve of the
    same S0-normalised signals."""
    from larmor_b200.sd import DRL, SDModel
    from larmor_b200.sd.kernel import Kernel
    from larmor_b200.sd.rf import AnisotropicRF
    from larmor_b200.sd.solvers import calibrate_drl_nu
    from larmor_b200.sd.sphere import DIRS_300
    from larmor_b200.synthetic import mfod_signals, mfod_table
    from larmor_b200.types import Volume

    z = drl_fixture

    class _K:
        k = z["k"]

    assert calibrate_drl_nu(_K(), z["bvals"]) == pytest.approx(float(z["nu"]), rel=1e-10)
    rng = np.random.default_rng(4)
    gtab = mfod_table(rng)
    data = mfod_signals(rng, gtab, 64).reshape(4, 4, 4, -1).astype(np.float32)
    wm = AnisotropicRF([1.7e-3, 0.2e-3, 0.2e-3], 0.0)
    model = SDModel([wm], method="GRL", solver=DRL(num_iter=120))
    fit = model.fit(Volume(data, np.eye(4)), gtab)
    kernel = Kernel([wm], gtab.bvals, gtab.bvecs, dirs=DIRS_300, weights=None)
    nu = calibrate_drl_nu(kernel, gtab.bvals)
    sig = data.reshape(-1, data.shape[-1]).astype(np.float64)
    norm = np.minimum(sig / sig[:, gtab.b0_mask].mean(axis=1)[:, None], 1.0)
    k_t, k_t_k = _products(kernel.w_k_aniso)
    amps = oracle.drl(norm, k_t, k_t_k, nu, 120, 1.0 / kernel.w_k_aniso.shape[1])
    from larmor_b200.sd.model import to_sh

    ref = to_sh(amps, fit.lmax, "tournier", exact_integral=True)
    got = fit.fods[0].reshape(-1, ref.shape[1])
    assert (np.abs(got - ref).max(axis=1) / np.abs(ref).max(axis=1)).max() < 1e-5


# ---- the tensor-core mode (precision tf32x3) -------------------------------------------------

# The tensor-core mode computes each product as three TF32 products (FP32 accuracy) and keeps
# the amplitudes in FP32: its FODs are held to the project's FOD tolerance, 1e-4 of the voxel's
# largest amplitude, against the FP64 fit, not to the FP64 path's 1e-10.
TC_FOD_REL = 1e-4


def _tc_fit(signals, k, nu, n_iter, start, precision):
    from larmor_b200 import _core

    k_t, k_t_k = _products(k)
    solver = _core.FodSolver.drl(k_t, k_t_k, nu=nu, n_iter=n_iter, init=start)
    if precision != "fp64":
        solver.set_precision(precision)
    got = _core.fit_single_tissue(np.ascontiguousarray(signals), solver, 1)
    solver.check_errors()
    return got


def _rel(got, ref):
    return np.abs(got - ref).max(axis=1) / np.abs(ref).max(axis=1)


@pytest.mark.gpu
@pytest.mark.parametrize("name", SETTINGS)
def test_tensor_core_drl_matches_the_reference_solver(cuda, drl_fixture, name):
    z = drl_fixture
    got = _tc_fit(z["signals"], z["k"], float(z[f"{name}_nu"]), 200, float(z[f"{name}_start"]), "tf32x3")
    rel = _rel(got, z[f"{name}_fods"])
    print(f"tensor-core dRL, {name}: FOD rel max {rel.max():.3e}, median {np.median(rel):.3e}")
    assert rel.max() <= TC_FOD_REL


@pytest.mark.gpu
@pytest.mark.parametrize(("n_meas", "n_dirs", "n_vox"), [(280, 300, 1000), (90, 130, 203), (60, 72, 97)])
def test_tensor_core_drl_matches_the_oracle_on_more_voxels(cuda, oracle, n_meas, n_dirs, n_vox):
    """Tiles of 48 voxels with a ragged last one, one to three 128-direction tiles, NaN signals."""
    rng = np.random.default_rng(7 * n_meas + n_dirs)
    k = np.abs(rng.normal(size=(n_meas, n_dirs))) * np.exp(-rng.uniform(0, 3, size=(n_meas, 1)))
    fods = np.zeros((n_vox, n_dirs))
    for f in fods:
        f[rng.choice(n_dirs, size=rng.integers(1, 4), replace=False)] = rng.dirichlet([1.0, 1.0, 1.0])[:1]
    signals = fods @ k.T + rng.uniform(0, 0.05, size=(n_vox, 1)) * np.abs(rng.normal(size=(n_vox, n_meas)))
    signals[:n_vox // 2:37, 3] = np.nan
    k_t, k_t_k = _products(k)
    got = _tc_fit(signals, k, 0.02, 150, 1.0 / n_dirs, "tf32x3")
    ref = oracle.drl(signals, k_t, k_t_k, 0.02, 150, 1.0 / n_dirs, n_threads=8)
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    ok = ~np.isnan(ref).any(axis=1)
    rel = _rel(got[ok], ref[ok])
    print(f"tensor-core dRL {n_meas}x{n_dirs}, {n_vox} voxels: FOD rel max {rel.max():.3e}, "
          f"median {np.median(rel):.3e}")
    assert rel.max() <= TC_FOD_REL


@pytest.mark.gpu
def test_tensor_core_drl_refuses_sizes_it_does_not_take(cuda, drl_fixture):
    from larmor_b200 import _core

    k = drl_fixture["k"][:, :40]
    k_t, k_t_k = _products(k)
    solver = _core.FodSolver.drl(k_t, k_t_k, nu=0.1, n_iter=10, init=0.1)
    with pytest.raises(ValueError, match="65 to 320 directions"):
        solver.set_precision("tf32x3")
    with pytest.raises(ValueError, match="precision must be"):
        solver.set_precision("fp16")
