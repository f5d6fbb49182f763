"""ORACLE — test infrastructure only. Only tests/ and the smoke check import this module; the
product path (larmor_b200) never does.

A numpy restatement of Larmor's input preparation for the voxelwise fits
(src/larmor/dwi/inputs.py of larmor-dmri 2.2.0), the steps the device staging replaces:
    scaled      Volume.as_float / signal_rows: float32 conversion, then * slope + intercept in
                float32 (src/larmor/types/volume.py:91-123, src/larmor/dwi/inputs.py:137-172)
    estimate_s0 the mean b0, repaired from plausible mask voxels within 3x3x3, then 5x5x5
                (src/larmor/dwi/inputs.py:78-134)
    largest     largest_finite_signal (src/larmor/dwi/inputs.py:212-224)
    floors      floor_bad_samples' per-voxel floor (src/larmor/dwi/inputs.py:227-252)

Pinned against the reference's own outputs on three volumes: tests/golden/staging.npz, written
by tests/golden/make_golden.py; tests/test_staging.py checks this module against them.
"""

from __future__ import annotations

import numpy as np
from scipy.ndimage import uniform_filter

SIGNAL_FLOOR = 1e-3
NEIGHBOURHOODS = (3, 5)


def scaled(data: np.ndarray, slope: float, intercept: float, *, always: bool) -> np.ndarray:
    """The float32 values of data * slope + intercept, each step in float32. as_float scales
    whenever it converts (always=True); signal_rows only when the scaling is not the identity."""
    out = data.astype(np.float32)
    if always or slope != 1.0 or intercept != 0.0:
        out = out * np.float32(slope)
        out = out + np.float32(intercept)
    return out


def estimate_s0(data, slope, intercept, is_b0, mask) -> np.ndarray:
    """S0 over the grid (src/larmor/dwi/inputs.py:78-134)."""
    is_b0 = np.asarray(is_b0, dtype=bool)
    values = data if (data.dtype == np.float32 and slope == 1.0 and intercept == 0.0) else \
        scaled(data, slope, intercept, always=True)
    b0_sum = values[..., is_b0].sum(axis=-1, dtype=np.float64)
    s0 = b0_sum / is_b0.sum()
    n_dw = int((~is_b0).sum())
    if n_dw == 0:
        return s0
    mean_dw = (values.sum(axis=-1, dtype=np.float64) - b0_sum) / n_dw
    finite = np.isfinite(s0) & np.isfinite(mean_dw)
    plausible = mask & finite & (s0 > mean_dw)
    to_repair = mask & finite & ~plausible
    repaired = np.full(s0.shape, np.nan)
    for width in NEIGHBOURHOODS:
        open_voxels = to_repair & np.isnan(repaired)
        if not open_voxels.any():
            break
        size = width**3
        count = np.rint(uniform_filter(plausible.astype(np.float64), width, mode="constant") * size)
        total = uniform_filter(np.where(plausible, s0, 0.0), width, mode="constant")
        found = open_voxels & (count > 0)
        repaired[found] = total[found] * size / count[found]
    s0[to_repair] = repaired[to_repair]
    return s0


def largest_finite(signals: np.ndarray) -> float:
    """The largest finite signal, or 1 when none is positive (src/larmor/dwi/inputs.py:212-224)."""
    finite = signals[np.isfinite(signals)]
    largest = float(finite.max()) if finite.size else -np.inf
    return largest if largest > 0 else 1.0


def floors(s0: np.ndarray | None, largest: float, v: int) -> np.ndarray:
    """Each voxel's replacement for samples that are not finite and positive: 1e-3 S0 where S0 is
    finite and positive, else 1e-3 times the largest finite signal
    (src/larmor/dwi/inputs.py:227-252)."""
    out = np.full(v, SIGNAL_FLOOR * largest)
    if s0 is not None:
        usable = np.isfinite(s0) & (s0 > 0)
        out[usable] = SIGNAL_FLOOR * s0[usable]
    return out


def stage(data, slope, intercept, is_b0, mask):
    """Everything the device staging writes for the mask voxels (np.nonzero order): the float32
    signals (v, N), S0 (v) or None without a b0, whether each row is finite, the floors (v) and
    the largest finite signal."""
    voxels = np.nonzero(mask)
    signals = scaled(data[voxels], slope, intercept, always=False)
    s0 = estimate_s0(data, slope, intercept, is_b0, mask)[mask] if np.any(is_b0) else None
    largest = largest_finite(signals)
    return dict(signals=signals, s0=s0, finite=np.isfinite(signals).all(axis=1),
                floor=floors(s0, largest, len(signals)), largest=largest)
