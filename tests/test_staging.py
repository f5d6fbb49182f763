"""Device input staging (lar_stage_dwi, lar_normalise_signals): the oracle's restatement of the
reference's input preparation against the reference's own outputs (tests/golden/staging.npz),
and on the GPU the staging kernels against the oracle, on the fixture's volumes and on a larger
seeded one. The signals and the largest value are exact (the same float32 operations); S0 and
the floors follow sums taken in another order, so they agree to a few ulps."""

from __future__ import annotations

import numpy as np
import pytest

NAMES = ["int", "float", "b0only"]


@pytest.fixture(scope="module")
def staging_fixture():
    from conftest import GOLDEN

    return dict(np.load(GOLDEN / "staging.npz"))


def _volume(z, name):
    from larmor_b200.types import GradientTable, Volume

    n = len(z[f"{name}_bvals"])
    bvecs = np.zeros((n, 3))
    bvecs[:, 0] = 1.0
    gtab = GradientTable(z[f"{name}_bvals"], bvecs)
    vol = Volume(z[f"{name}_data"], np.eye(4), slope=float(z[f"{name}_slope"]),
                 intercept=float(z[f"{name}_intercept"]))
    return vol, gtab


@pytest.mark.parametrize("name", NAMES)
def test_oracle_staging_matches_the_reference(staging_fixture, name):
    from oracle import staging

    z = staging_fixture
    mask = z["mask"]
    args = (z[f"{name}_data"], float(z[f"{name}_slope"]), float(z[f"{name}_intercept"]), z[f"{name}_is_b0"])
    np.testing.assert_array_equal(staging.estimate_s0(*args, mask), z[f"{name}_s0"])
    got = staging.stage(*args, mask)
    np.testing.assert_array_equal(got["signals"].astype(np.float64), z[f"{name}_signals"])
    assert got["largest"] == z[f"{name}_largest"]
    sig = got["signals"].astype(np.float64)
    floored = np.where(np.isfinite(sig) & (sig > 0), sig, got["floor"][:, None])
    np.testing.assert_array_equal(floored, z[f"{name}_floored"])


def test_fixture_covers_every_repair_case(staging_fixture):
    """The int volume has voxels repaired from 3x3x3, from 5x5x5 and not at all."""
    from oracle import staging

    z = staging_fixture
    mask = z["mask"]
    is_b0 = z["int_is_b0"]
    vals = staging.scaled(z["int_data"], 0.25, 3.0, always=True).astype(np.float64)
    own = vals[..., is_b0].mean(axis=-1)[mask]
    s0 = z["int_s0"][mask]
    repaired = own != s0
    assert np.isnan(s0).sum() >= 1 and (repaired & np.isfinite(s0)).sum() >= 10


def test_staging_refuses_unreadable_sample_types(staging_fixture):
    from larmor_b200.dwi.inputs import stage_dwi
    from larmor_b200.types import Volume

    vol, gtab = _volume(staging_fixture, "float")
    half = Volume(vol.data.astype(np.float16), np.eye(4))
    with pytest.raises(ValueError, match="staging reads"):
        stage_dwi(half, gtab, staging_fixture["mask"])


def _check_staged(staged, expected):
    signals = staged.signals.cpu().numpy()
    np.testing.assert_array_equal(signals, expected["signals"])
    np.testing.assert_array_equal(staged.finite.cpu().numpy().astype(bool), expected["finite"])
    assert float(staged.largest.cpu().numpy()[0]) == expected["largest"]
    if expected["s0"] is None:
        assert staged.s0 is None
    else:
        s0 = staged.s0.cpu().numpy()
        np.testing.assert_array_equal(np.isnan(s0), np.isnan(expected["s0"]))
        np.testing.assert_allclose(s0, expected["s0"], rtol=1e-13, atol=0)
    np.testing.assert_allclose(staged.floor.cpu().numpy(), expected["floor"], rtol=1e-13, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_device_staging_matches_the_oracle(cuda, staging_fixture, name):
    from larmor_b200.dwi.inputs import stage_dwi
    from oracle import staging

    z = staging_fixture
    vol, gtab = _volume(z, name)
    staged = stage_dwi(vol, gtab, z["mask"])
    expected = staging.stage(vol.data, vol.slope, vol.intercept, gtab.b0_mask, z["mask"])
    _check_staged(staged, expected)
    # And the reference's own numbers.
    np.testing.assert_array_equal(staged.signals.cpu().numpy().astype(np.float64), z[f"{name}_signals"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_estimate_s0_matches_the_reference_on_the_grid(cuda, staging_fixture, name):
    """dwi.estimate_s0 (the mask's S0 and repair staged on the device, the plain b0 mean outside
    the mask) against the reference's estimate_s0 over the whole grid."""
    from larmor_b200.dwi import estimate_s0

    z = staging_fixture
    vol, gtab = _volume(z, name)
    got = estimate_s0(vol, gtab, z["mask"])
    ref = z[f"{name}_s0"]
    assert got.shape == ref.shape
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["uint16", "int32", "uint8", "float64"])
def test_device_staging_of_a_larger_volume(cuda, dtype):
    """A 48x40x30 volume of 6 b0s + 40 dw samples with dark-b0 patches of several sizes, in
    several sample types and a scaling."""
    from larmor_b200.dwi.inputs import stage_dwi
    from larmor_b200.types import GradientTable, Volume
    from oracle import staging

    rng = np.random.default_rng(21)
    shape = (48, 40, 30)
    n_b0, n_dw = 6, 40
    s0 = rng.uniform(100, 200, size=shape)
    dw = s0[..., None] * np.exp(-rng.uniform(0.3, 2.5, size=shape + (n_dw,)))
    sig = np.concatenate([np.repeat(s0[..., None], n_b0, axis=-1), dw], axis=-1)
    for k in range(25):
        c = rng.integers(0, np.array(shape) - 1)
        w = rng.integers(1, 8)
        sig[c[0]:c[0] + w, c[1]:c[1] + w, c[2]:c[2] + w, :n_b0] = rng.uniform(0, 5)
    sig[21:28, 17:24, 12:19, :n_b0] = 1.0  # a 7x7x7 dark block: its centre has no plausible voxel within 5x5x5
    if dtype == "float64":
        data = sig
        slope, intercept = 1.0, 0.0
    else:
        slope, intercept = 0.5, 1.0
        data = np.clip(np.rint((sig - intercept) / slope), 0, np.iinfo(dtype).max).astype(dtype)
    grid = np.stack(np.meshgrid(*[np.linspace(-1, 1, k) for k in shape], indexing="ij"), axis=-1)
    mask = (grid**2).sum(axis=-1) <= 1.0
    bvals = np.concatenate([np.zeros(n_b0), np.full(n_dw, 1000.0)])
    bvecs = np.zeros((n_b0 + n_dw, 3))
    bvecs[:, 2] = 1.0
    gtab = GradientTable(bvals, bvecs)
    vol = Volume(data, np.eye(4), slope=slope, intercept=intercept)
    staged = stage_dwi(vol, gtab, mask)
    expected = staging.stage(vol.data, vol.slope, vol.intercept, gtab.b0_mask, mask)
    assert np.isnan(expected["s0"]).any()
    _check_staged(staged, expected)


@pytest.mark.gpu
def test_device_normalisation_matches_numpy(cuda, staging_fixture):
    from larmor_b200.dwi.inputs import normalise_signals, stage_dwi

    z = staging_fixture
    vol, gtab = _volume(z, "float")
    staged = stage_dwi(vol, gtab, z["mask"])
    out, finite = normalise_signals(staged.signals, staged.s0)
    q = staged.signals.cpu().numpy().astype(np.float64) / staged.s0.cpu().numpy()[:, None]
    fin = np.isfinite(q).all(axis=1)
    np.testing.assert_array_equal(finite.cpu().numpy().astype(bool), fin)
    np.testing.assert_array_equal(out.cpu().numpy()[fin], np.minimum(q[fin], 1.0))
    assert (~fin).any()
