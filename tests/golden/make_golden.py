"""Generates the golden fixtures of tests/golden from the reference (larmor-dmri 2.2.0).

Run in a container that has the reference checkout, whose path is the one required argument:

    python tests/golden/make_golden.py /path/to/reference

The reference's compiled core cannot be built without Eigen and nanobind, and its Python layer
needs Python >= 3.14. Its numpy/scipy code does run on 3.12 from a temporary copy of its source
tree with three mechanical changes, made here in the copy only:

1. `from __future__ import annotations` at the top of every module (3.14 defers annotations);
2. `except A, B:` rewritten to `except (A, B):` (3.14 syntax);
3. stand-ins for `larmor._core` (whose fits this project replaces) and `skimage.morphology`.

What the fixtures hold, all from the reference's own code and data:
- dki_block.npz: the CFIN 8x8x8x133 test block's masked signals (tests/data/dki), its gradient
  table, the DTI and DKI design and constraint matrices the models build, the MRtrix dwi2tensor
  golden fits (mrtrix_dt_ref.npz, mrtrix_dkt_ref.npz) and the outputs of the reference's numpy
  oracle tests/dwi/reference_fitting.py (ols_fit, wls_fit, constrain) on those signals, plus the
  reference's metric functions (compute_dti_metrics, compute_kurtosis_metrics) on the numpy fits.
- mfod.npz: the MRIToolkit mFOD fixture (tests/data/mfod: 512 voxels, the MATLAB FODs and
  fractions) with the high- and low-resolution kernels Larmor builds for it (sd/kernel.py), its
  shell weights and the SH projection matrices of sd/model.py:_to_sh.
- msmt.npz: the forward and constraint matrices and ridge of MSMT-CSD (sd/msmt.py) for the
  responses of tests/data/msmt on a seeded three-shell table, as tests/sd/test_msmt.py builds them.
- peaks.npz: the FOD block of the reference's peak tests with MRtrix sh2peaks' peaks of it, the
  642-vertex icosphere of find_peaks and the outputs of the reference's numpy peak oracle
  (tests/sd/reference_peaks.py) on the cases of tests/sd/test_peaks_compiled.py; the icosphere
  is also written to larmor_b200/data/icosphere642.npz, where the package reads it.
- staging.npz: the reference's input preparation (estimate_s0, signal_rows,
  largest_finite_signal, floor_bad_samples) on three seeded volumes: int16 with slope and
  intercept and dark-b0 voxels to repair, float32 with non-finite and non-positive samples, and a
  table of b0s only.
- csd.npz: the matrices of single-shell CSD (csd_problem) for four settings on the 60-direction
  shell of tests/sd/test_csd.py, and that test's synthetic voxels.
- drl.npz: damped Richardson-Lucy (the reference's numpy drl_solver) on the voxels, kernel and
  calibrated nu of tests/sd/test_drl.py, for its three settings.
- grl.npz: GRL (the multi-tissue fit with dRL) by the reference's numpy restatement on the MATLAB
  and synthetic cases of tests/sd/test_grl.py, with both kernels' matrices.
- dirs300.npy: the reference's 300 FOD directions (src/larmor/data/dir300.txt), a table the
  SD models must share exactly; also written to larmor_b200/data/dirs300.npy, where the
  package reads it.
"""

from __future__ import annotations

import re
import shutil
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent


def _patched_copy(reference: Path) -> Path:
    tmp = Path(tempfile.mkdtemp(prefix="larmor_ref_"))
    src = tmp / "src"
    shutil.copytree(reference / "src", src, ignore=shutil.ignore_patterns("viewer"))
    for path in src.rglob("*.py"):
        text = path.read_text()
        text = re.sub(r"except (\w+(?:\.\w+)*), (\w+(?:\.\w+)*):", r"except (\1, \2):", text)
        if "from __future__ import annotations" not in text:
            lines = text.split("\n")
            # After the module docstring, if any.
            insert = 0
            if lines and lines[0].startswith('"""'):
                if lines[0].count('"""') >= 2 and len(lines[0]) > 3:
                    insert = 1
                else:
                    for i in range(1, len(lines)):
                        if '"""' in lines[i]:
                            insert = i + 1
                            break
            lines.insert(insert, "from __future__ import annotations")
            text = "\n".join(lines)
        path.write_text(text)
    return tmp


def _install_stubs() -> None:
    core = types.ModuleType("larmor._core")
    core.MAX_LMAX = 20

    def _missing(*_args, **_kwargs):
        raise RuntimeError("the reference's compiled core is not built here")

    for name in ("fit_log_signal", "LsiDesign", "fit_lsi", "FodSolver", "DeconvKernel",
                 "fit_multi_tissue", "fit_single_tissue"):
        setattr(core, name, _missing)
    sys.modules["larmor._core"] = core
    skimage = types.ModuleType("skimage")
    morphology = types.ModuleType("skimage.morphology")
    morphology.reconstruction = _missing
    skimage.morphology = morphology
    sys.modules["skimage"] = skimage
    sys.modules["skimage.morphology"] = morphology


def _staging_fixture() -> None:
    """staging.npz: the reference's input preparation (src/larmor/dwi/inputs.py) on three seeded
    volumes: estimate_s0 over the grid, signal_rows of the mask voxels, largest_finite_signal and
    floor_bad_samples with the mask voxels' S0.
    - "int": int16 samples scaled by slope 0.25 and intercept 3. It has dark-b0 voxels that repair
      from the 3x3x3 neighbourhood, from the 5x5x5 one, or not at all, some on the grid's edge.
    - "float": float32 samples with NaN, infinite, zero and negative values.
    - "b0only": float64 samples rounded by the float32 conversion, with a table of b0s only, whose
      S0 is the plain mean b0."""
    from larmor.dwi.inputs import estimate_s0, floor_bad_samples, largest_finite_signal, signal_rows
    from larmor.types import GradientTable, Volume

    rng = np.random.default_rng(11)
    shape = (14, 12, 10)
    out = {}

    def table(n_b0, n_dw):
        dirs = rng.normal(size=(n_dw, 3))
        dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
        bvals = np.concatenate([np.zeros(n_b0), np.full(n_dw, 1000.0)])
        bvecs = np.vstack([np.zeros((n_b0, 3)), dirs]) if n_dw else np.zeros((n_b0, 3))
        return GradientTable(bvals, bvecs)

    grid = np.stack(np.meshgrid(*[np.linspace(-1, 1, k) for k in shape], indexing="ij"), axis=-1)
    mask = (grid**2).sum(axis=-1) <= 1.15
    mask[0, 5:8, 3:6] = True  # mask voxels on the grid's edge

    def decays(n_b0, n_dw):
        s0 = rng.uniform(800, 1200, size=shape)
        adc = rng.uniform(0.5e-3, 2.5e-3, size=shape + (n_dw,))
        dw = s0[..., None] * np.exp(-1000.0 * adc)
        return np.concatenate([np.repeat(s0[..., None], n_b0, axis=-1), dw], axis=-1)

    # "int": dark b0s: one isolated voxel, a 3x3x3 block (its centre repairs from 5x5x5), a
    # 7x7x7 block (its centre has no plausible voxel within 5x5x5), edge voxels.
    sig = decays(3, 24)
    dark = np.zeros(shape, dtype=bool)
    dark[7, 6, 5] = True
    dark[3:6, 2:5, 2:5] = True
    dark[4:11, 3:10, 2:9] |= True
    dark[0, 6, 4] = True
    sig[dark, :3] = rng.uniform(0, 60, size=(int(dark.sum()), 3))
    raw = np.rint((sig - 3.0) / 0.25).astype(np.int16)
    volumes = {"int": (Volume(raw, np.eye(4), slope=0.25, intercept=3.0), table(3, 24))}
    # "float": float32 with NaN, inf, zero and negative samples.
    sig = decays(2, 30).astype(np.float32)
    bad = rng.random(sig.shape) < 0.01
    sig[bad] = rng.choice(np.array([np.nan, np.inf, -np.inf, 0.0, -5.0], dtype=np.float32), size=int(bad.sum()))
    sig[2, 3:5, 2:8, :2] = 1.0  # dark b0s with finite samples
    volumes["float"] = (Volume(sig, np.eye(4)), table(2, 30))
    # "b0only": a table of b0s only.
    sig = decays(4, 0) * (1 + 1e-9 * rng.normal(size=shape + (4,)))
    volumes["b0only"] = (Volume(sig.astype(np.float64), np.eye(4)), table(4, 0))
    for name, (vol, gtab) in volumes.items():
        voxels = np.nonzero(mask)
        s0 = estimate_s0(vol, gtab, mask)
        rows = signal_rows(vol, voxels, slice(None))
        largest = largest_finite_signal(vol, voxels)
        floored = rows.copy()
        floor_bad_samples(floored, s0[mask], largest=largest)
        out.update({f"{name}_data": vol.data, f"{name}_slope": vol.slope, f"{name}_intercept": vol.intercept,
                    f"{name}_bvals": gtab.bvals, f"{name}_is_b0": gtab.b0_mask, f"{name}_s0": s0,
                    f"{name}_signals": rows, f"{name}_largest": largest, f"{name}_floored": floored})
    out["mask"] = mask
    np.savez_compressed(OUT / "staging.npz", **out)


def _csd_fixture() -> None:
    """csd.npz: the matrices of single-shell CSD the reference builds
    (src/larmor/sd/csd_solver.py:csd_problem) on the 60-direction b=1000 shell and the white matter
    response of tests/sd/test_csd.py (RESPONSE, _gradients), for four solver settings, and that
    test's synthetic voxels (_voxels: one fibre, 90 and 60 degree crossings, a noisy crossing)."""
    from larmor.sd import CSDSolver, ZonalSHRF
    from larmor.sd.csd_solver import csd_problem
    from larmor.types import GradientTable

    response = np.array([1800.0, -700.0, 180.0, -35.0, 5.0])
    rng = np.random.default_rng(1)
    dirs = rng.normal(size=(60, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    gtab = GradientTable(np.r_[0.0, [1000.0] * 60], np.r_[np.zeros((1, 3)), dirs])
    out = dict(response=response, bvals=gtab.bvals, bvecs=gtab.bvecs)
    own = np.random.default_rng(5).normal(size=(120, 3))
    settings = [(8, CSDSolver()), (8, CSDSolver(init_lmax=2, neg_lambda=0.5, threshold=0.1, max_iter=20)),
                (10, CSDSolver(norm_lambda=2.0)), (6, CSDSolver(directions=own))]
    for i, (lmax, solver) in enumerate(settings):
        pr = csd_problem(gtab.bvecs[1:], response, lmax, solver)
        out.update({f"p{i}_lmax": lmax, f"p{i}_initial": pr.initial, f"p{i}_forward": pr.forward,
                    f"p{i}_constraint": pr.constraint, f"p{i}_norm_weight": pr.norm_weight,
                    f"p{i}_threshold": pr.threshold, f"p{i}_max_iter": pr.max_iter})
    out["p3_directions"] = own
    rf = ZonalSHRF(bvals=np.array([1000.0]), coefficients=response[None])
    rad90, rad60 = np.radians(90.0), np.radians(60.0)
    fibre_sets = [np.array([[1.0, 0, 0]]), np.array([[1.0, 0, 0], [np.cos(rad90), np.sin(rad90), 0]]),
                  np.array([[1.0, 0, 0], [np.cos(rad60), np.sin(rad60), 0]]), np.array([[1.0, 0, 0], [0, 1.0, 0]])]
    rows = np.array([rf.signal(gtab.bvals[1:], gtab.bvecs[1:], f).mean(axis=1) for f in fibre_sets])
    noisy = rows[3] + np.random.default_rng(2).normal(0, 40.0, rows.shape[1])
    out["signals"] = np.vstack([rows, noisy[None]])
    out["fibres"] = np.array([np.pad(f, ((0, 2 - len(f)), (0, 0)), constant_values=np.nan) for f in fibre_sets]
                             + [np.array([[1.0, 0, 0], [0, 1.0, 0]])])
    np.savez_compressed(OUT / "csd.npz", **out)


def _drl_fixture(reference: Path) -> None:
    """drl.npz: damped Richardson-Lucy on the cases of tests/sd/test_drl.py. The white matter
    kernel on the MATLAB gradient table of tests/data/grl_obj.mat (DIRS_300, the shell weights);
    the test's 300 seeded voxels (noisy one- to three-fibre voxels with CSF, and isotropic ones);
    nu calibrated as calibrate_drl_nu does (an undamped 200-iteration solve of the isotropic signal
    exp(-b_max 0.7e-3), nu = 0.2 max(fod)), with the reference's numpy solver in place of the
    compiled one; and the reference's numpy solver (tests/sd/reference_solvers.py:drl_solver) on
    the voxels for the test's three settings: calibration (uniform start, undamped), single-tissue
    (uniform start, damped) and multi-tissue start (1e-6 start, damped), 200 iterations each."""
    from scipy.io import loadmat

    sys.path.insert(0, str(reference / "tests" / "sd"))
    from reference_solvers import DRL_INIT, drl_solver

    from larmor.sd import AnisotropicRF
    from larmor.sd.kernel import Kernel
    from larmor.sd.sphere import DIRS_300

    grl = loadmat(reference / "tests" / "data" / "grl_obj.mat", simplify_cells=True)["grl_obj"]
    bvals = np.asarray(grl["bvals"], dtype=np.float64)
    wm = AnisotropicRF(eigen_vals=[1.7e-3, 0.2e-3, 0.2e-3], mean_kurtosis=0.0)
    kernel = Kernel([wm], bvals=bvals, bvecs=grl["bvecs"].astype(np.float64), dirs=DIRS_300,
                    weights=grl["shell_weight"])
    k = np.ascontiguousarray(kernel.k)
    k_t, k_t_k = np.ascontiguousarray(k.T), np.ascontiguousarray(k.T @ k)
    n_cols = k.shape[1]
    iso = np.full(len(bvals), np.exp(-max(bvals) * 0.7e-3))
    nu = float(0.2 * np.max(drl_solver(np.full(n_cols, 1.0 / n_cols), iso, k_t, k_t_k, 0.0, 200)))
    rng = np.random.default_rng(0)
    n_vox = 300
    n_fibre = 2 * n_vox // 3
    fods = np.zeros((n_fibre, n_cols))
    for fod in fods:
        cols = rng.choice(n_cols, size=rng.integers(1, 4), replace=False)
        fod[cols] = rng.dirichlet(np.ones(len(cols)))
    csf = rng.uniform(0.0, 0.3, size=(n_fibre, 1))
    fibre = (1 - csf) * fods @ kernel.k_aniso.T + csf * np.exp(-bvals * 3e-3)
    fibre += rng.uniform(0.0, 0.05, (n_fibre, 1)) * rng.standard_normal(fibre.shape)
    adc = rng.uniform(0.5e-3, 3e-3, size=(n_vox - n_fibre, 1))
    signals = np.ascontiguousarray(np.vstack([fibre, np.exp(-bvals * adc)])[rng.permutation(n_vox)])
    out = dict(bvals=bvals, k=k, signals=signals, nu=nu, drl_init=DRL_INIT)
    for name, start, damping in (("calibration", 1.0 / n_cols, 0.0), ("single", 1.0 / n_cols, nu),
                                 ("multi_start", DRL_INIT, nu)):
        init = np.full(n_cols, start)
        out[f"{name}_fods"] = np.array([drl_solver(init, sv, k_t, k_t_k, damping, 200) for sv in signals])
        out[f"{name}_start"], out[f"{name}_nu"] = start, damping
    np.savez_compressed(OUT / "drl.npz", **out)


def _grl_fixture(reference: Path) -> None:
    """grl.npz: GRL (the multi-tissue fit with damped Richardson-Lucy) on the two cases of
    tests/sd/test_grl.py, by the reference's numpy restatement
    (tests/sd/reference_solvers.py:fit_multi_tissue_voxel, 200 low- and 600 high-resolution
    iterations asked for):
    - "matlab": the 216 masked voxels of tests/data/grl_obj.mat, normalised by their b0s, with the
      kernels of run_grl.m's responses (tests/conftest.py:_rfs, kernel_lr, kernel_hr) and MATLAB's
      nu;
    - "synthetic": test_grl.py's 150 seeded voxels of two anisotropic responses and two isotropic
      ones, with nu calibrated as calibrate_drl_nu does (the numpy solver in place of the compiled
      one).
    Each case stores both kernels' matrices and blocks, the shell weights, the nu values, the
    signals and the reference's high-resolution FODs and fractions."""
    from scipy.io import loadmat

    sys.path.insert(0, str(reference / "tests" / "sd"))
    from reference_solvers import drl_solver, fit_multi_tissue_voxel

    from larmor.sd import AnisotropicRF, IsotropicRF
    from larmor.sd.kernel import Kernel
    from larmor.sd.model import normalize_by_b0
    from larmor.sd.sphere import DIRS_300, get_dirs
    from larmor.types import GradientTable

    grl = loadmat(reference / "tests" / "data" / "grl_obj.mat", simplify_cells=True)["grl_obj"]
    bvals = grl["bvals"].astype(np.float64)
    bvecs = grl["bvecs"].astype(np.float64)
    weights = grl["shell_weight"]

    def kernels(rfs):
        lr = Kernel(rfs, bvals, bvecs, dirs=get_dirs(min(len(bvals), 45)), weights=weights)
        hr = Kernel(rfs, bvals, bvecs, dirs=DIRS_300, weights=weights)
        return lr, hr

    def calibrate(kernel):
        signal = np.full(len(bvals), np.exp(-max(bvals) * 0.7e-3))
        k = kernel.k
        fod = drl_solver(np.full(k.shape[1], 1.0 / k.shape[1]), signal, k.T, k.T @ k, 0.0, 200)
        return float(0.2 * np.max(fod))

    out = {"bvals": bvals, "bvecs": bvecs, "weights": np.asarray(weights, dtype=np.float64)}
    # matlab
    rfs = [AnisotropicRF(eigen_vals=[1.7e-3, 0.2e-3, 0.2e-3], mean_kurtosis=0.0), IsotropicRF(diffusivity=0.7e-3),
           IsotropicRF(diffusivity=3e-3)]
    lr, hr = kernels(rfs)
    vox = np.argwhere(grl["mask"] == 1)
    is_b0 = GradientTable(grl["bvals"], grl["bvecs"]).b0_mask
    signals = normalize_by_b0(grl["img"][vox[:, 0], vox[:, 1], vox[:, 2]].astype(np.float64), is_b0)
    cases = {"matlab": (signals, lr, hr, float(grl["NN_L"]), float(grl["NN_H"]))}
    # synthetic
    rfs2 = [AnisotropicRF(eigen_vals=[1.7e-3, 0.2e-3, 0.2e-3], mean_kurtosis=0.0),
            AnisotropicRF(eigen_vals=[1.5e-3, 0.9e-3, 0.1e-3], mean_kurtosis=0.0),
            IsotropicRF(diffusivity=0.7e-3), IsotropicRF(diffusivity=3e-3)]
    lr2, hr2 = kernels(rfs2)
    rng = np.random.default_rng(0)
    n_dirs = len(DIRS_300)
    syn = np.empty((150, len(bvals)))
    for signal in syn:
        fod = np.zeros(n_dirs)
        cols = rng.choice(n_dirs, size=rng.integers(1, 4), replace=False)
        fod[cols] = rng.dirichlet(np.ones(len(cols)))
        f = rng.dirichlet(np.ones(4))
        if rng.random() < 0.2:
            f[rng.integers(4)] = 0.0
            f /= f.sum()
        signal[:] = (f[0] * hr2.k_aniso[:, :n_dirs] @ fod + f[1] * hr2.k_aniso[:, n_dirs:] @ fod
                     + f[2] * np.exp(-bvals * 0.7e-3) + f[3] * np.exp(-bvals * 3e-3))
        signal += rng.uniform(0.0, 0.03) * rng.standard_normal(len(bvals))
    cases["synthetic"] = (syn, lr2, hr2, calibrate(lr2), calibrate(hr2))
    for name, (sig, klr, khr, lr_nu, hr_nu) in cases.items():
        fits = [fit_multi_tissue_voxel(sv, klr, khr, lr_nu, hr_nu) for sv in sig]
        for tag, k in (("lr", klr), ("hr", khr)):
            out[f"{name}_{tag}_k"] = k.k
            out[f"{name}_{tag}_k_aniso"] = k.k_aniso
            out[f"{name}_{tag}_k_iso"] = k.k_iso
            out[f"{name}_{tag}_w_k_aniso"] = k.w_k_aniso
            out[f"{name}_{tag}_w_k_iso"] = k.w_k_iso
            out[f"{name}_{tag}_blocks"] = np.array([(b.start, b.stop) for b in k.aniso_blocks])
        out.update({f"{name}_signals": np.ascontiguousarray(sig), f"{name}_lr_nu": lr_nu, f"{name}_hr_nu": hr_nu,
                    f"{name}_fods": np.array([f[0] for f in fits]), f"{name}_fractions": np.array([f[1] for f in fits])})
    np.savez_compressed(OUT / "grl.npz", **out)


def _peaks_fixture(reference: Path) -> None:
    """peaks.npz: the FOD block of the reference's peak tests (tests/data/peaks/fod.mif, 8x8x8,
    lmax 8) with MRtrix sh2peaks' peaks of it (peaks_ref.mif), the 642-vertex icosphere and the
    block's amplitudes on it (src/larmor/sd/peaks.py:_build_icosphere, _get_amplitudes), and the
    outputs of the reference's numpy peak oracle (tests/sd/reference_peaks.py) on the cases of
    tests/sd/test_peaks_compiled.py: derivatives at random and polar angles, climbs from random
    starts on the block and on random series, climbs under other settings, and the peak search
    of every voxel under three threshold settings."""
    sys.path.insert(0, str(reference / "tests" / "sd"))
    import reference_peaks as rp

    from larmor.io import load_volume
    from larmor.sd.peaks import _build_icosphere, _get_amplitudes
    from larmor.sd.sh import get_sh_indices

    data = reference / "tests" / "data" / "peaks"
    fod = load_volume(data / "fod.mif")
    fod.to_closest_canonical()
    block = np.ascontiguousarray(fod.as_float(dtype=np.float64).reshape(-1, fod.data.shape[-1]))
    ref = load_volume(data / "peaks_ref.mif")
    ref.to_closest_canonical()
    mrtrix = ref.as_float(dtype=np.float64).reshape(len(block), -1)
    vertices, neighbours = _build_icosphere()
    on_sphere = _get_amplitudes(block, 8, full=False)
    out = dict(fod_block=block, mrtrix_peaks=mrtrix, vertices=vertices,
               neighbours=neighbours.astype(np.int64), on_sphere=on_sphere)

    def random_sh(lmax, seed):
        return np.random.default_rng(seed).normal(size=len(get_sh_indices(lmax)[0]))

    def random_starts(n, seed):
        st = np.random.default_rng(seed).normal(size=(n, 3))
        return st / np.linalg.norm(st, axis=1, keepdims=True)

    # Derivatives: lmax 0..20, three random series each, at random angles and at the poles.
    for lmax in range(0, 21, 2):
        rng = np.random.default_rng(lmax)
        theta = np.concatenate([rng.uniform(0, np.pi, 40), [0.0, 1e-6, 5e-5, 2e-4, np.pi - 1e-6, np.pi]])
        phi = rng.uniform(-np.pi, np.pi, len(theta))
        shs = np.array([random_sh(lmax, seed) for seed in range(3)])
        vals = np.array([[rp.derivatives(sh, lmax, float(t), float(q)) for t, q in zip(theta, phi)] for sh in shs])
        out[f"deriv_l{lmax}_sh"], out[f"deriv_l{lmax}_theta"], out[f"deriv_l{lmax}_phi"] = shs, theta, phi
        out[f"deriv_l{lmax}_values"] = vals

    def climbs(shs, lmax, starts, **settings):
        dirs = np.empty((len(shs), len(starts), 3))
        amps = np.empty((len(shs), len(starts)))
        for i, sh in enumerate(shs):
            for j, st in enumerate(starts):
                dirs[i, j], amps[i, j] = rp.climb(sh, lmax, st, **settings)
        return dirs, amps

    # Climbs from random starts on 20 voxels of the block, and on random series.
    voxels = np.random.default_rng(0).choice(len(block), 20, replace=False)
    starts = random_starts(20, 1)
    out["climb_block_voxels"], out["climb_block_starts"] = voxels, starts
    out["climb_block_dirs"], out["climb_block_amps"] = climbs(block[voxels], 8, starts)
    for lmax in (2, 8, 16, 20):
        shs = np.array([random_sh(lmax, seed) for seed in range(4)])
        st = random_starts(15, lmax)
        out[f"climb_l{lmax}_sh"], out[f"climb_l{lmax}_starts"] = shs, st
        out[f"climb_l{lmax}_dirs"], out[f"climb_l{lmax}_amps"] = climbs(shs, lmax, st)
    # Other settings: one capped step, a smaller cap, too few iterations, no tolerance.
    settings = [dict(tol=1.0), dict(tol=1.0, max_step=0.05), dict(max_iters=3), dict(tol=0.0)]
    starts = random_starts(10, 2)
    rows = np.arange(0, len(block), 37)
    out["climb_settings_voxels"], out["climb_settings_starts"] = rows, starts
    for k, st in enumerate(settings):
        out[f"climb_settings{k}_dirs"], out[f"climb_settings{k}_amps"] = climbs(block[rows], 8, starts, **st)
    out["climb_settings"] = np.array([[st.get("max_iters", 50), st.get("tol", 1e-4), st.get("max_step", 0.2)]
                                      for st in settings])
    # The peak search of every voxel.
    for k, (num, rel, thr) in enumerate([(3, 0.1, 0.0), (2, 0.3, 0.2), (6, 0.0, 0.0)]):
        res = [rp.pep(block[i], 8, on_sphere[i], vertices, neighbours, num, rel, thr) for i in range(len(block))]
        out[f"pep{k}_dirs"] = np.array([r[0] for r in res])
        out[f"pep{k}_amps"] = np.array([r[1] for r in res])
    out["pep_settings"] = np.array([[3, 0.1, 0.0], [2, 0.3, 0.2], [6, 0.0, 0.0]])
    np.savez_compressed(OUT / "peaks.npz", **out)
    # The icosphere ships with the package too: find_peaks' start vertices, whose order is the
    # order in which climbs are merged.
    np.savez_compressed(OUT.parents[1] / "larmor_b200" / "data" / "icosphere642.npz", vertices=vertices,
                        neighbours=neighbours.astype(np.int64))


def main(reference: Path) -> None:
    tmp = _patched_copy(reference)
    sys.path.insert(0, str(tmp / "src"))
    _install_stubs()
    import larmor  # noqa: F401

    sys.modules["larmor"]._core = sys.modules["larmor._core"]
    sys.path.insert(0, str(reference / "tests" / "dwi"))
    from reference_fitting import constrain, ols_fit, wls_fit
    from scipy.io import loadmat

    from larmor.dwi.dki import _constraint_matrix, _design_matrix, compute_kurtosis_metrics
    from larmor.dwi.dti import compute_dti_metrics
    from larmor.io import load_dwi
    from larmor.sd import AnisotropicRF, IsotropicRF, NoddiRF
    from larmor.sd.kernel import Kernel
    from larmor.sd.model import compute_shell_weights, low_resolution_dirs
    from larmor.sd.msmt import constraint_matrix, forward_matrix, NORM_REG
    from larmor.sd.rf import ZonalSHRF
    from larmor.sd.sh import build_basis_matrix
    from larmor.sd.sphere import DIRS_300, get_theta_phi

    # ---- DKI/DTI block ------------------------------------------------------------------
    dki_dir = reference / "tests" / "data" / "dki"
    volume, gtab = load_dwi(dki_dir / "dwi.nii.gz", bvals=dki_dir / "bvals",
                            bvecs=dki_dir / "bvecs", frame="fsl")
    dt_ref = np.load(dki_dir / "mrtrix_dt_ref.npz")
    dkt_ref = np.load(dki_dir / "mrtrix_dkt_ref.npz")
    mask = dkt_ref["mask"]
    s = volume.as_float()[mask].astype(np.float64)
    positive = (s > 0).all(axis=1)
    sp = s[positive]
    dti_design = np.column_stack([np.ones(len(gtab.bvals)), -gtab.b_matrix])
    dki_design = _design_matrix(gtab)
    dki_g = _constraint_matrix(gtab)
    out = dict(
        signals_f32=volume.as_float()[mask].astype(np.float32),
        mask=mask,
        dt_mask=dt_ref["mask"],
        bvals=gtab.bvals,
        bvecs=gtab.bvecs,
        b_matrix=gtab.b_matrix,
        b0_mask=gtab.b0_mask,
        dti_design=dti_design,
        dki_design=dki_design,
        dki_constraints=dki_g,
        positive=positive,
        mrtrix_dt_ols=dt_ref["dt_ols"], mrtrix_dt_wls=dt_ref["dt_wls"],
        mrtrix_dt_wls_settled=dt_ref["wls_settled"],
        mrtrix_dkt_dt_ols=dkt_ref["dt_ols"], mrtrix_dkt_dt_wls=dkt_ref["dt_wls"],
        mrtrix_dkt_kt_ols=dkt_ref["kt_ols"], mrtrix_dkt_kt_wls=dkt_ref["kt_wls"],
        mrtrix_dkt_wls_settled=dkt_ref["wls_settled"],
    )
    # The reference's numpy oracle on the positive voxels (tests/dwi/test_dki.py:581-602).
    for name, fit in (("ols", ols_fit), ("wls", wls_fit)):
        out[f"np_dti_{name}"] = fit(dti_design, sp)
        p = fit(dki_design, sp)
        out[f"np_dki_{name}"] = p
        pc, broke = constrain(dki_design, np.log(sp), p, gtab, name == "wls")
        out[f"np_dki_{name}_constrained"] = pc
        out[f"np_dki_{name}_broke"] = broke
    # The reference's metric functions on its numpy DTI and DKI fits.
    unit = np.ones((len(sp), 1, 1), dtype=bool)
    for name in ("ols", "wls"):
        d = out[f"np_dti_{name}"][1:7]
        dt, fa, md, ad, rd, pe, ev, npd = compute_dti_metrics(d, unit)
        out[f"metrics_dti_{name}"] = np.column_stack(
            [fa[:, 0, 0], md[:, 0, 0], ad[:, 0, 0], rd[:, 0, 0], ev[:, 0, 0], pe[:, 0, 0]]).astype(np.float64)
        out[f"metrics_dti_{name}_npd"] = npd[:, 0, 0]
        p = out[f"np_dki_{name}_constrained"]
        d = p[1:7]
        md_ = (d[0] + d[3] + d[5]) / 3
        w = np.divide(p[7:], md_**2, out=np.zeros_like(p[7:]), where=md_ > 0)
        mk, ak, rk, ka = compute_kurtosis_metrics(d, w)
        out[f"metrics_dki_{name}"] = np.column_stack([mk, ak, rk, ka])
    np.savez_compressed(OUT / "dki_block.npz", **out)

    # ---- mFOD (MRIToolkit fixture) -------------------------------------------------------
    mfod_dir = reference / "tests" / "data" / "mfod"
    kref = loadmat(mfod_dir / "mfod_kernel.mat", simplify_cells=True)["kernel"]
    ref = loadmat(mfod_dir / "mfod_ref.mat", simplify_cells=True)["ref"]
    bvals = kref["bvals"].astype(np.float64)
    bvecs = kref["bvecs"].astype(np.float64)
    rfs = [AnisotropicRF([1.7e-3, 0.2e-3, 0.2e-3], 0.0), NoddiRF(), IsotropicRF(3e-3)]
    weights = compute_shell_weights(bvals, 1.0)
    hr = Kernel(rfs, bvals, bvecs, dirs=DIRS_300, weights=weights)
    lr = Kernel(rfs, bvals, bvecs, dirs=low_resolution_dirs(rfs, len(bvals)), weights=weights)
    theta, phi = get_theta_phi(DIRS_300)
    basis8 = build_basis_matrix(theta, phi, 8)
    np.savez_compressed(
        OUT / "mfod.npz",
        bvals=bvals, bvecs=bvecs, weights=weights,
        signal=ref["signal"].astype(np.float64), ijk=ref["ijk"],
        matlab_fod=ref["fod"].astype(np.float64), matlab_fractions=ref["fractions"].astype(np.float64),
        hr_k_aniso=hr.k_aniso, hr_k_iso=hr.k_iso, hr_w_k_aniso=hr.w_k_aniso, hr_w_k_iso=hr.w_k_iso,
        hr_blocks=np.array([(b.start, b.stop) for b in hr.aniso_blocks]),
        lr_k_aniso=lr.k_aniso, lr_k_iso=lr.k_iso, lr_w_k_aniso=lr.w_k_aniso, lr_w_k_iso=lr.w_k_iso,
        sh_basis_tournier_l8=basis8,
    )

    # ---- MSMT-CSD matrices (tests/sd/test_msmt.py's set-up: _gradients, _tensor_response,
    # _isotropic_response) -------------------------------------------------------------------
    from larmor.sd.sphere import get_dirs
    from larmor.types import GradientTable

    shells = np.array([0.0, 1000.0, 2000.0, 3000.0])
    dirs40 = get_dirs(40)
    tb = [np.zeros((2, 3))]
    for k in range(3):
        ang = 0.4 * k
        rot = np.array([[np.cos(ang), -np.sin(ang), 0.0], [np.sin(ang), np.cos(ang), 0.0], [0.0, 0.0, 1.0]])
        tb.append(dirs40 @ rot.T)
    tgtab = GradientTable(np.concatenate([[0.0, 0.0], np.repeat(shells[1:], 40)]), np.vstack(tb))

    def tensor_response(s0, par, perp):
        nodes, wts = np.polynomial.legendre.leggauss(64)
        th = np.arccos(nodes)
        rows = []
        for b in shells:
            profile = s0 * np.exp(-b * (perp + (par - perp) * nodes**2))
            zonal = build_basis_matrix(th, np.zeros_like(th), 8)[:, [0, 3, 10, 21, 36]]
            rows.append(2 * np.pi * (wts * profile) @ zonal)
        return ZonalSHRF(bvals=shells, coefficients=np.array(rows))

    def isotropic_response(s0, diff):
        sig = s0 * np.exp(-shells * diff)
        return ZonalSHRF(bvals=shells, coefficients=np.sqrt(4 * np.pi) * sig[:, None])

    rfs_msmt = [tensor_response(1000.0, 1.7e-3, 0.2e-3), isotropic_response(1500.0, 0.8e-3),
                isotropic_response(2000.0, 3e-3)]
    lmaxes = [8, 0, 0]
    fwd = forward_matrix(rfs_msmt, lmaxes, tgtab.bvals, tgtab.bvecs)
    g = constraint_matrix(lmaxes, DIRS_300)
    np.savez_compressed(
        OUT / "msmt.npz", forward=fwd, constraints=g,
        ridge=float(np.sqrt(NORM_REG * np.max(np.sum(fwd**2, axis=0)))),
        bvals=tgtab.bvals, bvecs=tgtab.bvecs, shells=shells,
        wm_coefficients=rfs_msmt[0].coefficients, gm_coefficients=rfs_msmt[1].coefficients,
        csf_coefficients=rfs_msmt[2].coefficients)
    _peaks_fixture(reference)
    _staging_fixture()
    _csd_fixture()
    _drl_fixture(reference)
    _grl_fixture(reference)
    np.save(OUT / "dirs300.npy", np.asarray(DIRS_300, dtype=np.float64))
    # The same table ships with the package: the SD models' FOD directions.
    np.save(OUT.parents[1] / "larmor_b200" / "data" / "dirs300.npy", np.asarray(DIRS_300, dtype=np.float64))
    shutil.rmtree(tmp)
    print("wrote", sorted(p.name for p in OUT.glob("*.np*")))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/reference")
    main(Path(sys.argv[1]))
