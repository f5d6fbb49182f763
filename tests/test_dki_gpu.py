"""DKI on the GPU against the oracle, the reference's numpy oracle and its metric functions."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fit(dki_block, method, constrained):
    from larmor_b200 import _core

    s = dki_block["signals_f32"].astype(np.float64)[dki_block["positive"]]
    design = dki_block["dki_design"]
    g = dki_block["dki_constraints"] if constrained else np.zeros((0, 22))
    log_s = np.ascontiguousarray(np.log(s))
    return _core.fit_log_signal(design, g, log_s, method == "wls", 20, 1e-6, 1), log_s


@pytest.mark.parametrize("constrained", [False, True], ids=["plain", "constrained"])
@pytest.mark.parametrize("method", ["ols", "wls"])
def test_dki_fit_matches_the_reference_numpy_oracle(cuda, oracle, dki_block, method, constrained):
    """tests/dwi/test_dki.py:581-602: atol 1e-10 on column-scaled parameters, same flags."""
    (params, broke), log_s = _fit(dki_block, method, constrained)
    design = dki_block["dki_design"]
    scale = np.linalg.norm(design, axis=0)
    key = f"np_dki_{method}" + ("_constrained" if constrained else "")
    np.testing.assert_allclose(params * scale, dki_block[key].T * scale, rtol=0, atol=1e-10)
    expected_broke = dki_block[f"np_dki_{method}_broke"] if constrained else np.zeros(len(params), bool)
    np.testing.assert_array_equal(broke, expected_broke)
    g = dki_block["dki_constraints"] if constrained else None
    ref, ref_broke = oracle.fit_log_signal(design, g, log_s, method == "wls")
    np.testing.assert_allclose(params * scale, ref * scale, rtol=0, atol=1e-10)
    np.testing.assert_array_equal(broke, ref_broke)


@pytest.mark.parametrize("method", ["ols", "wls"])
def test_kurtosis_maps_match_the_reference_metrics(cuda, dki_block, method):
    import torch

    from larmor_b200.dwi.dki import dki_maps_device

    (params, _), _ = _fit(dki_block, method, True)
    dev = torch.device("cuda")
    p = torch.from_numpy(params).to(dev)
    maps = torch.empty((36, len(params)), dtype=torch.float32, device=dev)
    npd = torch.empty((len(params),), dtype=torch.uint8, device=dev)
    dki_maps_device(p, maps, npd)
    maps = maps.cpu().numpy()
    ref = dki_block[f"metrics_dki_{method}"]  # mk, ak, rk, ka in float64
    for row, col, name in ((32, 0, "mk"), (33, 1, "ak"), (34, 2, "rk"), (35, 3, "ka")):
        np.testing.assert_allclose(maps[row], ref[:, col], rtol=2e-6, atol=1e-6, err_msg=name)


@pytest.mark.parametrize("method", ["ols", "wls"])
def test_dki_model_matches_mrtrix_on_the_cfin_block(cuda, dki_block, method):
    """tests/dwi/test_dki.py:337-363: DT rel 1e-5, KT rel 5e-5 against dwi2tensor."""
    from larmor_b200.dwi.dki import fit_dki_signals
    from larmor_b200.types import GradientTable

    gtab = GradientTable(dki_block["bvals"], dki_block["bvecs"])
    s = dki_block["signals_f32"]
    s64 = s.astype(np.float64)
    is_b0 = gtab.b0_mask
    s0 = s64[:, is_b0].mean(axis=1)
    kept = (s64 > 0).all(axis=1) & (s64[:, ~is_b0] <= s0[:, None]).all(axis=1)
    assert kept.sum() == 511
    if method == "wls":
        kept &= dki_block["mrtrix_dkt_wls_settled"]
    maps, _, _ = fit_dki_signals(dki_block["dki_design"], np.zeros((0, 22)), s[kept], s0[kept],
                                 1e-3 * s0[kept], is_b0, method == "wls")
    ref_dt = dki_block[f"mrtrix_dkt_dt_{method}"][kept].astype(np.float64)
    ref_kt = dki_block[f"mrtrix_dkt_kt_{method}"][kept].astype(np.float64)
    mats = ref_dt[:, [0, 1, 2, 1, 3, 4, 2, 4, 5]].reshape(-1, 3, 3)
    dt_err = np.abs(maps[0:6].T - ref_dt).max(axis=1) / np.abs(np.linalg.eigvalsh(mats)).max(axis=1)
    kt_err = np.abs(maps[16:31].T - ref_kt).max(axis=1) / np.abs(ref_kt).max(axis=1)
    assert dt_err.max() < 1e-5
    assert kt_err.max() < 5e-5


def test_dki_model_on_a_synthetic_volume_matches_the_oracle(cuda, oracle):
    from larmor_b200.dwi import DKIModel
    from larmor_b200.dwi.dki import dki_constraints, dki_design
    from larmor_b200.synthetic import dki_volume
    from oracle import staging

    w = dki_volume(shape=(20, 20, 12))
    fit = DKIModel().fit(w.volume, w.gtab, w.mask)
    s = w.volume.data[w.mask].astype(np.float64)
    s0 = staging.estimate_s0(w.volume.data, w.volume.slope, w.volume.intercept, w.gtab.b0_mask, w.mask)[w.mask]
    is_b0 = w.gtab.b0_mask
    own = s[:, is_b0].mean(axis=1)
    repaired = ~np.isclose(s0, own, rtol=1e-9, atol=0.0)
    s[np.ix_(repaired, is_b0)] = s0[repaired, None]
    s[:, ~is_b0] = np.minimum(s[:, ~is_b0], s0[:, None])
    bad = ~(np.isfinite(s) & (s > 0))
    s[bad] = np.broadcast_to(1e-3 * s0[:, None], s.shape)[bad]
    params, broke = oracle.fit_log_signal(dki_design(w.gtab), dki_constraints(w.gtab), np.log(s), True)
    assert broke.any()
    np.testing.assert_allclose(fit.dt[w.mask], params[:, 1:7], rtol=1e-5, atol=1e-11)
    np.testing.assert_allclose(fit.s0[w.mask], np.exp(params[:, 0]), rtol=1e-6)
