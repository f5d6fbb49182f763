"""Putting masked values back on the image grid (src/larmor/dwi/mask.py:415)."""

from __future__ import annotations

import numpy as np


def unmask(values: np.ndarray, mask: np.ndarray, fill_value: float = 0.0,
           dtype=np.float32) -> np.ndarray:
    """Returns values (K,) or (K, D), one per True voxel of mask in C order, on the grid."""
    values = np.asarray(values)
    dtype = values.dtype if dtype is None else dtype
    out = np.full(mask.shape + values.shape[1:], fill_value, dtype=dtype)
    out[mask] = values
    return out
