"""FOD peaks: the oracle against the reference's numpy peak oracle and MRtrix sh2peaks
(tests/golden/peaks.npz; the cases and bounds of tests/sd/test_peaks_compiled.py and
tests/sd/test_peaks_reference.py), the argument checks of the bindings on the CPU, and on the
GPU the sm_100a derivatives, climbs and peak search against the same fixtures and the oracle,
with the edge cases the reference tests."""

from __future__ import annotations

import math

import numpy as np
import pytest

X, Y, Z = np.eye(3)
LMAX = 8

# The reference's bounds (tests/sd/test_peaks_compiled.py): climbs from arbitrary starts that
# wander over flat regions end up to ~4e-10 apart between two implementations; amplitudes are
# taken at near-stationary points.
CLIMB_DIR_ATOL = 1e-9
CLIMB_AMP_ATOL = 1e-14
# (num_peaks, relative_threshold, threshold) -> direction atol, amplitude rtol.
PEP_BOUNDS = [(1e-12, 1e-12), (1e-12, 1e-12), (1e-9, 1e-11)]


def _unit(v) -> np.ndarray:
    u = np.asarray(v, dtype=np.float64)
    return u / np.linalg.norm(u)


def _fibre_sh(direction, lmax: int = LMAX) -> np.ndarray:
    from larmor_b200.sd.sh import build_basis_matrix, get_sh_indices

    ls, _ = get_sh_indices(lmax)
    theta = math.acos(float(np.clip(direction[2], -1.0, 1.0)))
    phi = math.atan2(float(direction[1]), float(direction[0]))
    b = build_basis_matrix(np.array([theta]), np.array([phi]), lmax)
    return b[0] * np.exp(-0.02 * ls * (ls + 1))


def _to_full(sh: np.ndarray, lmax: int) -> np.ndarray:
    """A symmetric series in the all-degrees layout (odd degrees zero)."""
    full = np.zeros((lmax + 1) ** 2)
    k = 0
    for ell in range(0, lmax + 1, 2):
        n = 2 * ell + 1
        full[ell * ell: ell * ell + n] = sh[k: k + n]
        k += n
    return full


def _check_climbs(climb, shs, lmax, starts, dirs, amps, **settings):
    for i, sh in enumerate(shs):
        for j, st in enumerate(starts):
            d, a = climb(sh, lmax, st, **settings)
            assert math.isnan(a) == math.isnan(amps[i, j]), (i, j)
            np.testing.assert_array_equal(np.isnan(d), np.isnan(dirs[i, j]))
            if not math.isnan(amps[i, j]):
                np.testing.assert_allclose(d, dirs[i, j], rtol=0, atol=CLIMB_DIR_ATOL)
                assert abs(a - amps[i, j]) <= CLIMB_AMP_ATOL * np.abs(sh).sum()


def _check_derivatives(derivatives, z):
    for lmax in range(0, 21, 2):
        shs, theta, phi = z[f"deriv_l{lmax}_sh"], z[f"deriv_l{lmax}_theta"], z[f"deriv_l{lmax}_phi"]
        for i, sh in enumerate(shs):
            for j, (t, p) in enumerate(zip(theta, phi)):
                expected = z[f"deriv_l{lmax}_values"][i, j]
                got = np.array(derivatives(sh, lmax, float(t), float(p)))
                np.testing.assert_allclose(got, expected, rtol=0, atol=1e-13 * np.abs(expected).max())


def _check_pep(dirs, amps, z, k):
    dir_atol, amp_rtol = PEP_BOUNDS[k]
    np.testing.assert_array_equal(np.isnan(amps), np.isnan(z[f"pep{k}_amps"]))
    np.testing.assert_allclose(dirs, z[f"pep{k}_dirs"], rtol=0, atol=dir_atol)
    np.testing.assert_allclose(amps, z[f"pep{k}_amps"], rtol=amp_rtol)


def _check_mrtrix_largest(dirs, amps, z):
    """tests/sd/test_peaks_reference.py:19-41: the largest peak against sh2peaks."""
    ref = z["mrtrix_peaks"][:, :3]
    has = np.isfinite(amps[:, 0])
    ref_has = np.isfinite(ref).all(axis=1)
    np.testing.assert_array_equal(has, ref_has)
    assert ref_has.any()
    ref_amp = np.linalg.norm(ref[has], axis=1)
    cos = np.abs(np.sum(dirs[has, 0] * (ref[has] / ref_amp[:, None]), axis=1))
    assert np.all(cos >= math.cos(math.radians(0.01)))
    np.testing.assert_allclose(amps[has, 0], ref_amp, rtol=1e-5)


# ---- the oracle against the reference's outputs (CPU) -------------------------------------


def test_oracle_derivatives_match_the_reference(oracle, peaks_fixture):
    _check_derivatives(oracle.sh_derivatives, peaks_fixture)


def test_oracle_climbs_match_the_reference(oracle, peaks_fixture):
    z = peaks_fixture
    block = z["fod_block"]
    _check_climbs(oracle.climb, block[z["climb_block_voxels"]], LMAX, z["climb_block_starts"],
                  z["climb_block_dirs"], z["climb_block_amps"])
    for lmax in (2, 8, 16, 20):
        _check_climbs(oracle.climb, z[f"climb_l{lmax}_sh"], lmax, z[f"climb_l{lmax}_starts"],
                      z[f"climb_l{lmax}_dirs"], z[f"climb_l{lmax}_amps"])
    for k, (iters, tol, step) in enumerate(z["climb_settings"]):
        _check_climbs(oracle.climb, block[z["climb_settings_voxels"]], LMAX, z["climb_settings_starts"],
                      z[f"climb_settings{k}_dirs"], z[f"climb_settings{k}_amps"], max_iters=int(iters), tol=tol,
                      max_step=step)


@pytest.mark.parametrize("k", [0, 1, 2])
def test_oracle_peak_search_matches_the_reference(oracle, peaks_fixture, k):
    z = peaks_fixture
    num, rel, thr = z["pep_settings"][k]
    dirs, amps = oracle.peaks_chunk(z["fod_block"], LMAX, z["on_sphere"], z["vertices"], z["neighbours"], int(num),
                                    rel, thr, n_threads=4)
    _check_pep(dirs, amps, z, k)


def test_oracle_largest_peak_matches_mrtrix_sh2peaks(oracle, peaks_fixture):
    z = peaks_fixture
    dirs, amps = oracle.peaks_chunk(z["fod_block"], LMAX, z["on_sphere"], z["vertices"], z["neighbours"], 3, 0.1,
                                    0.0, n_threads=4)
    _check_mrtrix_largest(dirs, amps, z)


def test_oracle_full_series_of_a_symmetric_fod(oracle, peaks_fixture):
    """A symmetric series written with all degrees: the same derivatives, and each peak of the
    symmetric search found twice, once per lobe, with its sign kept."""
    z = peaks_fixture
    sh = z["fod_block"][100]
    full = _to_full(sh, LMAX)
    for t, p in [(0.3, 0.2), (1.2, -2.0), (0.0, 0.5), (math.pi, 1.0)]:
        np.testing.assert_allclose(oracle.sh_derivatives(full, LMAX, t, p, full=True),
                                   oracle.sh_derivatives(sh, LMAX, t, p), rtol=0, atol=1e-13)
    from larmor_b200.sd.sh import build_basis_matrix
    from larmor_b200.sd.sphere import get_theta_phi

    v, nb = z["vertices"], z["neighbours"]
    theta, phi = get_theta_phi(v)
    on = (build_basis_matrix(theta, phi, LMAX, full=True) @ full)[None]
    d6, a6 = oracle.peaks_chunk(full[None], LMAX, on, v, nb, 6, 0.1, 0.0, full=True)
    d3, a3 = oracle.peaks_chunk(sh[None], LMAX, z["on_sphere"][100:101], v, nb, 3, 0.1, 0.0)
    n = int(np.isfinite(a3).sum())
    assert int(np.isfinite(a6).sum()) == 2 * n
    for d, a in zip(d3[0, :n], a3[0, :n]):
        for sign in (1.0, -1.0):
            best = np.argmax(d6[0, : 2 * n] @ (sign * d))
            assert d6[0, best] @ (sign * d) > 1 - 1e-10
            assert a6[0, best] == pytest.approx(a, rel=1e-9)


def test_packaged_icosphere_is_the_reference_table(peaks_fixture):
    from larmor_b200.sd.peaks import _build_icosphere

    v, nb = _build_icosphere()
    np.testing.assert_array_equal(v, peaks_fixture["vertices"])
    np.testing.assert_array_equal(nb, peaks_fixture["neighbours"])
    np.testing.assert_allclose(np.linalg.norm(v, axis=1), 1.0, atol=1e-15)
    # Neighbourhood is symmetric; the 12 original vertices have 5 neighbours and list
    # themselves as the sixth.
    own = nb == np.arange(len(v))[:, None]
    assert own.sum(axis=1).tolist() == [1] * 12 + [0] * 630
    for i in range(len(v)):
        for j in nb[i]:
            assert i in nb[j]


# ---- the bindings' checks (CPU: they raise before any device work) ------------------------

BAD_LMAX = r"lmax must be at most 20, and even unless full, got|lmax \d+ has \d+ coefficients, got"


@pytest.mark.parametrize(("lmax", "num_coeffs", "full"), [
    (7, 36, False), (22, 276, False), (8, 28, False), (6, 45, False), (21, 484, True), (8, 45, True),
    (7, 64, False), (7, 36, True)])
def test_bindings_refuse_a_bad_lmax(peaks_fixture, lmax, num_coeffs, full):
    from larmor_b200 import _core

    sh = np.zeros(num_coeffs)
    v, nb = peaks_fixture["vertices"], peaks_fixture["neighbours"]
    with pytest.raises(ValueError, match=BAD_LMAX):
        _core.climb(sh, lmax, Z, full=full)
    with pytest.raises(ValueError, match=BAD_LMAX):
        _core.sh_derivatives(sh, lmax, 0.3, 0.2, full=full)
    with pytest.raises(ValueError, match=BAD_LMAX):
        _core.peaks_chunk(sh[None], lmax, np.zeros((1, 642)), v, nb, 3, 0.1, 0.0, 1, full=full)


def _good_chunk_args(z) -> dict:
    return {"coeffs": np.zeros((2, 45)), "lmax": LMAX, "on_sphere": np.zeros((2, 642)), "vertices": z["vertices"],
            "neighbours": z["neighbours"], "n_peaks": 3, "relative_threshold": 0.1, "threshold": 0.0,
            "n_threads": 1}


def _neighbours_with(z, value: int) -> np.ndarray:
    out = z["neighbours"].copy()
    out[5, 2] = value
    return out


@pytest.mark.parametrize("case", [
    "vertices_4_columns", "neighbours_5_columns", "neighbours_fewer_rows", "on_sphere_fewer_voxels",
    "on_sphere_fewer_vertices", "negative_neighbour", "neighbour_past_the_end", "zero_peaks", "zero_threads",
    "fortran_coeffs", "strided_on_sphere"])
def test_peaks_chunk_refuses_bad_arguments(peaks_fixture, case):
    from larmor_b200 import _core

    z = peaks_fixture
    bad = {
        "vertices_4_columns": ("vertices", np.zeros((642, 4)), "shapes do not match"),
        "neighbours_5_columns": ("neighbours", z["neighbours"][:, :5].copy(), "shapes do not match"),
        "neighbours_fewer_rows": ("neighbours", z["neighbours"][:600], "shapes do not match"),
        "on_sphere_fewer_voxels": ("on_sphere", np.zeros((1, 642)), "shapes do not match"),
        "on_sphere_fewer_vertices": ("on_sphere", np.zeros((2, 600)), "shapes do not match"),
        "negative_neighbour": ("neighbours", _neighbours_with(z, -1), "neighbour index is outside the sphere"),
        "neighbour_past_the_end": ("neighbours", _neighbours_with(z, 642), "neighbour index is outside the sphere"),
        "zero_peaks": ("n_peaks", 0, "n_peaks must be at least 1"),
        "zero_threads": ("n_threads", 0, "n_threads must be at least 1"),
        "fortran_coeffs": ("coeffs", np.asfortranarray(np.zeros((2, 45))), "C-contiguous"),
        "strided_on_sphere": ("on_sphere", np.zeros((4, 642))[::2], "C-contiguous"),
    }
    name, value, message = bad[case]
    args = _good_chunk_args(z)
    args[name] = value
    with pytest.raises(ValueError, match=message):
        _core.peaks_chunk(**args)


def test_bindings_refuse_other_dtypes_and_negative_iterations(peaks_fixture):
    from larmor_b200 import _core

    z = peaks_fixture
    with pytest.raises(TypeError):
        _core.climb(np.zeros(45, dtype=np.float32), LMAX, Z)
    with pytest.raises(ValueError, match="max_iters must be at least 0"):
        _core.climb(np.zeros(45), LMAX, Z, max_iters=-1)
    args = _good_chunk_args(z)
    args["neighbours"] = z["neighbours"].astype(np.int32)
    with pytest.raises(TypeError):
        _core.peaks_chunk(**args)


@pytest.mark.parametrize(("kwargs", "message"), [
    (dict(num_peaks=0), "num_peaks must be at least 1"),
    (dict(chunk_size=0), "chunk_size must be at least 1"),
    (dict(n_jobs=0), "n_jobs must be"),
    (dict(relative_threshold=1.5), "relative_threshold must be between 0 and 1"),
    (dict(mask=np.ones((3, 2), dtype=bool)), "mask has shape"),
])
def test_find_peaks_refuses_bad_arguments(kwargs, message):
    from larmor_b200.sd import find_peaks

    with pytest.raises(ValueError, match=message):
        find_peaks(np.zeros((2, 3, 45)), **kwargs)


def test_find_peaks_refuses_lmax_above_20():
    from larmor_b200.sd import find_peaks

    with pytest.raises(ValueError, match="lmax must be at most 20"):
        find_peaks(np.zeros((1, 23 * 24 // 2)))
    with pytest.raises(ValueError, match="fit no layout"):
        find_peaks(np.zeros((1, 44)))


# ---- the GPU path --------------------------------------------------------------------------


@pytest.mark.gpu
def test_gpu_derivatives_match_the_reference(cuda, peaks_fixture):
    from larmor_b200 import _core

    _check_derivatives(_core.sh_derivatives, peaks_fixture)


@pytest.mark.gpu
def test_gpu_batched_derivatives_match_the_oracle(cuda, oracle):
    """lar_sh_derivatives over many (series, angle) rows at once, symmetric and full series."""
    import torch

    from larmor_b200 import _lib

    rng = np.random.default_rng(5)
    for lmax, full in [(8, False), (12, False), (20, False), (3, True), (8, True), (20, True)]:
        c = (lmax + 1) ** 2 if full else (lmax + 1) * (lmax + 2) // 2
        n = 500
        sh = rng.normal(size=(n, c))
        theta = np.concatenate([rng.uniform(0, np.pi, n - 4), [0.0, 1e-6, np.pi - 2e-5, np.pi]])
        phi = rng.uniform(-np.pi, np.pi, n)
        d = {k: torch.from_numpy(np.ascontiguousarray(a)).cuda() for k, a in dict(sh=sh, t=theta, p=phi).items()}
        out = torch.empty((n, 6), dtype=torch.float64, device="cuda")
        _lib.check(_lib.lib().lar_sh_derivatives(_lib.ptr(d["sh"]), n, c, lmax, int(full), _lib.ptr(d["t"]),
                                                 _lib.ptr(d["p"]), _lib.ptr(out), None))
        got = out.cpu().numpy()
        for i in range(n):
            exp = np.array(oracle.sh_derivatives(sh[i], lmax, theta[i], phi[i], full=full))
            np.testing.assert_allclose(got[i], exp, rtol=0, atol=1e-13 * np.abs(exp).max())


@pytest.mark.gpu
def test_gpu_climbs_match_the_reference(cuda, peaks_fixture):
    from larmor_b200 import _core

    z = peaks_fixture
    block = z["fod_block"]
    _check_climbs(_core.climb, block[z["climb_block_voxels"]], LMAX, z["climb_block_starts"],
                  z["climb_block_dirs"], z["climb_block_amps"])
    for lmax in (2, 8, 16, 20):
        _check_climbs(_core.climb, z[f"climb_l{lmax}_sh"], lmax, z[f"climb_l{lmax}_starts"],
                      z[f"climb_l{lmax}_dirs"], z[f"climb_l{lmax}_amps"])
    for k, (iters, tol, step) in enumerate(z["climb_settings"]):
        _check_climbs(_core.climb, block[z["climb_settings_voxels"]], LMAX, z["climb_settings_starts"],
                      z[f"climb_settings{k}_dirs"], z[f"climb_settings{k}_amps"], max_iters=int(iters), tol=tol,
                      max_step=step)


def _crossing(separation_deg: float):
    s = math.radians(separation_deg)
    b = np.array([math.cos(s), math.sin(s), 0.0])
    return _fibre_sh(X) + _fibre_sh(b), _unit(X + b)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["peak_at_pole", "antipode_at_pole", "peak_on_equator", "ring_of_minima",
                                  "ring_at_pole", "saddle_60", "saddle_90"])
def test_gpu_climb_on_stationary_points(cuda, oracle, name):
    from larmor_b200 import _core

    cases = {
        "peak_at_pole": (_fibre_sh(Z), Z), "antipode_at_pole": (_fibre_sh(Z), -Z),
        "peak_on_equator": (_fibre_sh(X), X), "ring_of_minima": (_fibre_sh(X), Y), "ring_at_pole": (_fibre_sh(X), Z),
        "saddle_60": _crossing(60.0), "saddle_90": _crossing(90.0),
    }
    sh, start = cases[name]
    d, f = _core.climb(sh, LMAX, start)
    d_ref, f_ref = oracle.climb(sh, LMAX, start)
    np.testing.assert_allclose(d, d_ref, rtol=0, atol=1e-14)
    np.testing.assert_allclose(d, start, rtol=0, atol=1e-12)
    assert f == pytest.approx(f_ref, rel=0, abs=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("k", [0, 1, 2])
def test_gpu_peaks_chunk_matches_the_reference(cuda, peaks_fixture, k):
    from larmor_b200 import _core

    z = peaks_fixture
    num, rel, thr = z["pep_settings"][k]
    dirs, amps = _core.peaks_chunk(z["fod_block"], LMAX, z["on_sphere"], z["vertices"], z["neighbours"], int(num),
                                   rel, thr, 1)
    _check_pep(dirs, amps, z, k)


@pytest.mark.gpu
@pytest.mark.parametrize("k", [0, 1, 2])
def test_gpu_find_peaks_matches_the_reference(cuda, peaks_fixture, k):
    """The whole device path: amplitudes on the icosphere computed on the GPU, then the search."""
    from larmor_b200.sd import find_peaks

    z = peaks_fixture
    num, rel, thr = z["pep_settings"][k]
    found = find_peaks(z["fod_block"].reshape(8, 8, 8, 45), num_peaks=int(num), relative_threshold=rel,
                       threshold=thr)
    _check_pep(found.directions.reshape(512, int(num), 3), found.amplitudes.reshape(512, int(num)), z, k)


@pytest.mark.gpu
def test_gpu_find_peaks_matches_mrtrix_sh2peaks(cuda, peaks_fixture):
    from larmor_b200.sd import find_peaks

    z = peaks_fixture
    found = find_peaks(z["fod_block"])
    _check_mrtrix_largest(found.directions, found.amplitudes, z)


@pytest.mark.gpu
@pytest.mark.parametrize(("lmax", "full"), [(8, False), (12, False), (4, True), (8, True)])
def test_gpu_peak_search_matches_the_oracle_on_random_fods(cuda, oracle, peaks_fixture, lmax, full):
    """20k synthetic FODs of 1-3 fibres plus noise (full: with odd-degree noise too), the same
    sphere amplitudes given to both: identical peak slots, values to the climbs' rounding."""
    from larmor_b200 import _core
    from larmor_b200.sd.sh import build_basis_matrix, get_sh_indices
    from larmor_b200.sd.sphere import get_theta_phi

    rng = np.random.default_rng(lmax + 100 * full)
    n = 20000
    ls, _ = get_sh_indices(lmax, full)
    fibres = rng.normal(size=(n, 3, 3))
    fibres /= np.linalg.norm(fibres, axis=2, keepdims=True)
    theta, phi = get_theta_phi(fibres.reshape(-1, 3))
    b = build_basis_matrix(theta, phi, lmax, full=full).reshape(n, 3, -1)
    b = np.where((ls % 2 == 0)[None, None], b, 0.0) * np.exp(-0.02 * ls * (ls + 1))
    w = rng.dirichlet([2.0, 2.0, 2.0], size=n) * (rng.random((n, 3)) < [1.0, 0.7, 0.4])
    coeffs = np.ascontiguousarray(np.einsum("nf,nfc->nc", w, b) + 0.02 * rng.normal(size=(n, len(ls))))
    v, nb = peaks_fixture["vertices"], peaks_fixture["neighbours"]
    tv, pv = get_theta_phi(v)
    on = np.ascontiguousarray(coeffs @ build_basis_matrix(tv, pv, lmax, full=full).T)
    num = 6 if full else 3
    dirs, amps = _core.peaks_chunk(coeffs, lmax, on, v, nb, num, 0.1, 0.0, 1, full=full)
    rd, ra = oracle.peaks_chunk(coeffs, lmax, on, v, nb, num, 0.1, 0.0, n_threads=8, full=full)
    np.testing.assert_array_equal(np.isnan(amps), np.isnan(ra))
    np.testing.assert_allclose(dirs, rd, rtol=0, atol=1e-9)
    np.testing.assert_allclose(amps, ra, rtol=1e-11)


def _chunk(sh, on_sphere, vertices, neighbours, num_peaks=4, relative_threshold=0.0, threshold=0.0):
    from larmor_b200 import _core

    return _core.peaks_chunk(np.ascontiguousarray(sh[None]), LMAX, np.ascontiguousarray(on_sphere[None]), vertices,
                             neighbours, num_peaks, relative_threshold, threshold, 1)


def _two_starts(a, b):
    return np.array([a, b]), np.array([[1, 0, 0, 0, 0, 0], [0, 1, 1, 1, 1, 1]], dtype=np.int64)


@pytest.mark.gpu
def test_gpu_search_does_not_start_from_non_positive_maxima(cuda, peaks_fixture):
    from larmor_b200.sd.peaks import _get_amplitudes

    v, nb = peaks_fixture["vertices"], peaks_fixture["neighbours"]
    sh = _fibre_sh(X)
    for on in (np.zeros(642), -np.ones(642), _get_amplitudes(sh[None], LMAX, False)[0] - 2.0):
        dirs, amps = _chunk(sh, on, v, nb)
        assert np.all(np.isnan(dirs)) and np.all(np.isnan(amps))


@pytest.mark.gpu
def test_gpu_search_starts_from_both_vertices_of_a_tie(cuda):
    v, nb = _two_starts(X, Y)
    sh = _fibre_sh(X) + _fibre_sh(Y)
    tie, _ = _chunk(sh, np.array([1.0, 1.0]), v, nb)
    lower, _ = _chunk(sh, np.array([1.0, 0.9]), v, nb)
    assert int(np.sum(np.isfinite(tie[0, :, 0]))) == 2
    assert int(np.sum(np.isfinite(lower[0, :, 0]))) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("vertex", [0, 7, 11, 12, 300, 641])
def test_gpu_search_starts_only_from_the_single_maximum(cuda, oracle, peaks_fixture, vertex):
    v, nb = peaks_fixture["vertices"], peaks_fixture["neighbours"]
    sh = _fibre_sh(X) + _fibre_sh(Y) + _fibre_sh(Z)
    expected, f = oracle.climb(sh, LMAX, v[vertex])
    assert f > 0
    dirs, amps = _chunk(sh, v @ v[vertex], v, nb)
    assert int(np.sum(np.isfinite(amps))) == 1
    assert abs(float(dirs[0, 0] @ expected)) == pytest.approx(1.0, abs=1e-12)
    assert amps[0, 0] == pytest.approx(f, abs=1e-12)


def _on_ring(azimuth_deg: float) -> np.ndarray:
    t, p = math.radians(50.0), math.radians(azimuth_deg)
    return np.array([math.sin(t) * math.cos(p), math.sin(t) * math.sin(p), math.cos(t)])


@pytest.mark.gpu
@pytest.mark.parametrize(("azimuth_deg", "count"), [(6.0, 1), (12.0, 2)])
def test_gpu_search_merges_peaks_closer_than_0_99_in_cos(cuda, azimuth_deg, count):
    v, nb = _two_starts(_on_ring(0.0), _on_ring(azimuth_deg))
    dirs, _ = _chunk(_fibre_sh(Z), np.array([1.0, 1.0]), v, nb)
    assert int(np.sum(np.isfinite(dirs[0, :, 0]))) == count


@pytest.mark.gpu
def test_gpu_search_drops_maxima_of_non_positive_amplitude(cuda, oracle):
    sh = -_fibre_sh(X)
    start = _unit((0.0, 0.53, 0.85))
    _, f = oracle.climb(sh, LMAX, start)
    assert f < 0
    v, nb = _two_starts(start, start)
    dirs, amps = _chunk(sh, np.array([1.0, 1.0]), v, nb, relative_threshold=1.0, threshold=-math.inf)
    assert np.all(np.isnan(dirs)) and np.all(np.isnan(amps))


@pytest.mark.gpu
def test_gpu_non_finite_first_amplitude_and_empty_chunks(cuda, peaks_fixture):
    from larmor_b200 import _core

    z = peaks_fixture
    on = z["on_sphere"][:4].copy()
    on[1, 0] = np.nan
    on[2, 0] = np.inf
    dirs, amps = _core.peaks_chunk(z["fod_block"][:4].copy(), LMAX, on, z["vertices"], z["neighbours"], 3, 0.1, 0.0, 1)
    assert np.all(np.isnan(amps[1:3])) and np.all(np.isnan(dirs[1:3]))
    assert np.isfinite(amps[0, 0]) and np.isfinite(amps[3, 0])
    dirs, amps = _core.peaks_chunk(np.zeros((0, 45)), LMAX, np.zeros((0, 642)), z["vertices"], z["neighbours"], 3,
                                   0.1, 0.0, 1)
    assert dirs.shape == (0, 3, 3) and amps.shape == (0, 3)


@pytest.mark.gpu
def test_gpu_isotropic_fod_merges_every_start(cuda, oracle, peaks_fixture):
    """A constant positive FOD: every vertex is a local maximum and every climb stops where it
    starts, so the found list grows to hundreds of entries before the merge; the slots match
    the oracle's."""
    from larmor_b200 import _core

    z = peaks_fixture
    sh = np.zeros((1, 45))
    sh[0, 0] = 1.0
    on = np.full((1, 642), 1.0 / math.sqrt(4 * math.pi))
    dirs, amps = _core.peaks_chunk(sh, LMAX, on, z["vertices"], z["neighbours"], 5, 0.0, 0.0, 1)
    rd, ra = oracle.peaks_chunk(sh, LMAX, on, z["vertices"], z["neighbours"], 5, 0.0, 0.0)
    np.testing.assert_array_equal(np.isnan(amps), np.isnan(ra))
    np.testing.assert_allclose(dirs, rd, rtol=0, atol=1e-12)
    np.testing.assert_allclose(amps, ra, rtol=1e-12)
