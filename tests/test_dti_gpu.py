"""DTI on the GPU against the oracle and the reference's golden fits, through the C ABI."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scaled(design):
    return np.linalg.norm(design, axis=0)


@pytest.mark.parametrize("method", ["ols", "wls"])
def test_core_fit_log_signal_matches_the_oracle_on_the_cfin_block(cuda, oracle, dki_block, method):
    from larmor_b200 import _core

    s = dki_block["signals_f32"].astype(np.float64)[dki_block["positive"]]
    design = dki_block["dti_design"]
    log_s = np.ascontiguousarray(np.log(s))
    params, broke = _core.fit_log_signal(design, np.zeros((0, 7)), log_s, method == "wls", 20, 1e-6, 1)
    ref, _ = oracle.fit_log_signal(design, None, log_s, method == "wls")
    assert not broke.any()
    # Same algorithm in FP64; the sums run in another order.
    np.testing.assert_allclose(params * _scaled(design), ref * _scaled(design), rtol=0, atol=1e-10)
    # And against the reference's own numpy oracle.
    np.testing.assert_allclose(params * _scaled(design), dki_block[f"np_dti_{method}"].T * _scaled(design),
                               rtol=0, atol=1e-10)


@pytest.mark.parametrize("weighted", [False, True])
def test_noise_free_and_underflow_cases(cuda, oracle, weighted):
    from larmor_b200 import _core
    from test_oracle import TENSOR_PARAMS, _tensor_design

    design = _tensor_design()
    log_s = np.ascontiguousarray(TENSOR_PARAMS @ design.T)
    params, _ = _core.fit_log_signal(design, np.zeros((0, 7)), log_s, weighted, 20, 1e-6, 1)
    np.testing.assert_allclose(params, TENSOR_PARAMS, rtol=1e-9, atol=1e-15)
    broken = np.vstack([TENSOR_PARAMS[0], [0.0, 0.42, 0.0, 0.0, 0.42, 0.0, 0.42]])
    log_s = np.ascontiguousarray(broken @ design.T)
    wls, _ = _core.fit_log_signal(design, np.zeros((0, 7)), log_s, True, 20, 1e-6, 1)
    ols, _ = _core.fit_log_signal(design, np.zeros((0, 7)), log_s, False, 20, 1e-6, 1)
    assert np.isfinite(wls).all()
    np.testing.assert_array_equal(wls[1], ols[1])


@pytest.mark.parametrize("method", ["ols", "wls"])
def test_dti_maps_match_the_reference_metrics(cuda, dki_block, method):
    from larmor_b200.dwi.dti import fit_dti_signals

    s = dki_block["signals_f32"][dki_block["positive"]]
    maps, npd = fit_dti_signals(dki_block["dti_design"], s, np.full(len(s), 1.0), method == "wls")
    ref = dki_block[f"metrics_dti_{method}"]  # fa, md, ad, rd, ev(3), pe(3), float32 maps
    np.testing.assert_allclose(maps[6], ref[:, 0], rtol=0, atol=2e-6)      # FA
    np.testing.assert_allclose(maps[7], ref[:, 1], rtol=1e-6, atol=1e-12)  # MD
    np.testing.assert_allclose(maps[8], ref[:, 2], rtol=1e-6, atol=1e-12)  # AD
    np.testing.assert_allclose(maps[9], ref[:, 3], rtol=1e-6, atol=1e-12)  # RD
    np.testing.assert_allclose(maps[13:16].T, ref[:, 4:7], rtol=1e-6, atol=1e-12)
    align = np.abs(np.sum(maps[10:13].T * ref[:, 7:10], axis=1))
    gap = ref[:, 4] - ref[:, 5]
    assert np.all(align[gap > 1e-5] > 1 - 1e-5)
    np.testing.assert_array_equal(npd, dki_block[f"metrics_dti_{method}_npd"])


@pytest.mark.parametrize("method", ["ols", "wls"])
def test_dti_model_matches_mrtrix_on_the_cfin_block(cuda, dki_block, method):
    """tests/dwi/test_dti.py:148-162, through DTIModel on the block's masked signals."""
    from larmor_b200.dwi.dti import fit_dti_signals

    s = dki_block["signals_f32"]
    kept = (s > 0).all(axis=1)
    if method == "wls":
        kept &= dki_block["mrtrix_dt_wls_settled"]
    maps, _ = fit_dti_signals(dki_block["dti_design"], s[kept], np.ones(kept.sum()), method == "wls")
    ref = dki_block[f"mrtrix_dt_{method}"][kept].astype(np.float64)
    mats = ref[:, [0, 1, 2, 1, 3, 4, 2, 4, 5]].reshape(-1, 3, 3)
    scale = np.abs(np.linalg.eigvalsh(mats)).max(axis=1)
    err = np.abs(maps[0:6].T - ref).max(axis=1) / scale
    assert err.max() < 1e-5


def test_dti_model_on_the_synthetic_volume_matches_the_oracle(cuda, oracle):
    from larmor_b200.dwi import DTIModel
    from larmor_b200.dwi.dti import dti_design
    from larmor_b200.synthetic import dti_volume

    w = dti_volume(shape=(24, 24, 16))
    fit = DTIModel(fit_method="wls").fit(w.volume, w.gtab, w.mask)
    s = w.volume.data[w.mask].astype(np.float64)
    params, _ = oracle.fit_log_signal(dti_design(w.gtab), None, np.log(s), True)
    np.testing.assert_allclose(fit.dt[w.mask], params[:, 1:7], rtol=1e-6, atol=1e-12)
    assert (fit.fa[~w.mask] == 0).all()
    # Float32 maps of the same FP64 fit: MD and FA within float32 rounding of the oracle's.
    md = params[:, [1, 4, 6]].sum(axis=1) / 3
    np.testing.assert_allclose(fit.md[w.mask], md, rtol=1e-6)


def test_fp32_variant_stays_near_the_fp64_fit(cuda, oracle):
    from larmor_b200.dwi import DTIModel
    from larmor_b200.synthetic import dti_volume

    w = dti_volume(shape=(24, 24, 16))
    f64 = DTIModel(fit_method="wls").fit(w.volume, w.gtab, w.mask)
    f32 = DTIModel(fit_method="wls", precision="fp32").fit(w.volume, w.gtab, w.mask)
    assert np.abs(f32.fa - f64.fa).max() < 1e-3
    assert np.abs(f32.md - f64.md).max() < 1e-6


@pytest.mark.parametrize("shells", [2, 3])
def test_large_tables_use_smaller_ctas_and_match_the_oracle(cuda, oracle, shells):
    """Tables of 200-290 measurements (2-3 shells of 90 directions) do not fit 64 voxels per CTA
    in shared memory; the fit takes 32 or 16 voxels per CTA and still matches the oracle."""
    from larmor_b200 import _core
    from larmor_b200.dwi.dti import dti_design
    from larmor_b200.synthetic import random_rotations, unit_directions
    from larmor_b200.types import GradientTable

    rng = np.random.default_rng(40 + shells)
    dirs = [unit_directions(rng, 90) for _ in range(shells)]
    bvals = np.concatenate([np.zeros(18)] + [np.full(90, 1000.0 * (k + 1)) for k in range(shells)])
    bvecs = np.vstack([np.zeros((18, 3))] + dirs)
    design = dti_design(GradientTable(bvals, bvecs))
    v = 700
    rot = random_rotations(rng, v)
    ev = np.stack([rng.uniform(1.2e-3, 2e-3, v), *(2 * [rng.uniform(0.2e-3, 0.6e-3, v)])], axis=1)
    tensors = np.einsum("vij,vj,vkj->vik", rot, ev, rot)
    g = GradientTable(bvals, bvecs)
    s = 1000.0 * np.exp(-g.bvals[None, :] * np.einsum("ni,vij,nj->vn", g.bvecs, tensors, g.bvecs))
    s = np.abs(s + rng.normal(0, 20.0, s.shape) + 1j * rng.normal(0, 20.0, s.shape))
    log_s = np.ascontiguousarray(np.log(s))
    params, broke = _core.fit_log_signal(design, np.zeros((0, 7)), log_s, True, 20, 1e-6, 1)
    ref, _ = oracle.fit_log_signal(design, None, log_s, True)
    sc = np.linalg.norm(design, axis=0)
    np.testing.assert_allclose(params * sc, ref * sc, rtol=0, atol=1e-10)
