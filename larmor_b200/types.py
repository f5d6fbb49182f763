"""The inputs of the fits: a DWI volume and its gradient table.

These keep the parts of Larmor's `Volume` and `GradientTable` (src/larmor/types/volume.py,
src/larmor/types/gradient_table.py) that the fitting hot path reads: the scaled float32 data,
the b-values and unit b-vectors, the b0 mask, the b-matrix and the shells.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# A volume whose b-vector is shorter than this and whose b-value is above the b0 threshold has
# no usable direction (src/larmor/types/gradient_table.py).
_MIN_LENGTH = 0.1


class Volume:
    """A 3D or 4D image with its affine and the value scaling data * slope + intercept."""

    def __init__(self, data: np.ndarray, affine: np.ndarray, *, slope: float = 1.0,
                 intercept: float = 0.0) -> None:
        data = np.asarray(data)
        if data.ndim not in (3, 4):
            raise ValueError(f"A volume is 3D or 4D; got shape {data.shape}.")
        affine = np.array(affine, dtype=np.float64)
        if affine.shape != (4, 4) or not np.isfinite(affine).all():
            raise ValueError("The affine must be a finite 4x4 matrix.")
        if not np.isfinite(slope) or slope == 0:
            slope, intercept = 1.0, 0.0
        self.data = data
        self.affine = affine
        self.slope = float(slope)
        self.intercept = float(intercept)

    def as_float(self, *, dtype=np.float32) -> np.ndarray:
        """The scaled values, data * slope + intercept, computed in `dtype`."""
        dtype = np.dtype(dtype)
        if not np.issubdtype(dtype, np.floating):
            raise ValueError(f"as_float needs a floating-point type, got {dtype}.")
        if np.iscomplexobj(self.data):
            raise ValueError("The volume holds complex data; pass its magnitude.")
        if self.data.dtype == dtype and self.slope == 1.0 and self.intercept == 0.0:
            return self.data
        out = self.data.astype(dtype)
        if self.slope != 1.0 or self.intercept != 0.0:
            out *= dtype.type(self.slope)
            out += dtype.type(self.intercept)
        return out


@dataclass
class GradientTable:
    """The b-value (s/mm^2) and unit gradient direction of each volume of a DWI.

    As in the reference, each b-value is scaled by the squared length of its vector and each
    vector is scaled to unit length; volumes at or below b0_threshold are b0s.
    """

    bvals: np.ndarray
    bvecs: np.ndarray
    b0_threshold: float = 50.0
    shell_epsilon: float = 80.0

    def __post_init__(self) -> None:
        self.bvals = np.array(self.bvals, dtype=np.float64)
        self.bvecs = np.array(self.bvecs, dtype=np.float64)
        if self.bvals.ndim != 1 or len(self.bvals) == 0:
            raise ValueError(f"bvals must be a non-empty (N,) array, got {self.bvals.shape}")
        if self.bvecs.shape != (len(self.bvals), 3):
            raise ValueError(f"bvecs must be (N, 3) = ({len(self.bvals)}, 3), got {self.bvecs.shape}")
        if not np.isfinite(self.bvals).all() or (self.bvals < 0).any():
            raise ValueError("b-values must be finite and non-negative")
        vecs = np.nan_to_num(self.bvecs, nan=0.0)
        if not np.isfinite(vecs).all():
            raise ValueError("b-vectors must not have infinite components")
        length = np.linalg.norm(vecs, axis=1)
        weighted = self.bvals > self.b0_threshold
        if (weighted & (length < _MIN_LENGTH)).any():
            raise ValueError(
                f"a volume has a b-value above {self.b0_threshold} but no direction"
            )
        has = length > 0
        scaled = self.bvals.copy()
        scaled[has] = self.bvals[has] * length[has] ** 2
        vecs[has] = vecs[has] / length[has, None]
        self.bvals = scaled
        self.bvecs = vecs

    @property
    def b0_mask(self) -> np.ndarray:
        return np.asarray(self.bvals <= self.b0_threshold, dtype=bool)

    @property
    def b_matrix(self) -> np.ndarray:
        """(N, 6): b (gx^2, 2 gx gy, 2 gx gz, gy^2, 2 gy gz, gz^2)."""
        b = self.bvals
        gx, gy, gz = self.bvecs.T
        return np.stack([b * gx**2, 2 * b * gx * gy, 2 * b * gx * gz, b * gy**2,
                         2 * b * gy * gz, b * gz**2], axis=1).astype(np.float64)

    @property
    def shell_index(self) -> np.ndarray:
        weighted = np.flatnonzero(~self.b0_mask)
        order = np.argsort(self.bvals[weighted], kind="stable")
        sorted_b = self.bvals[weighted][order]
        labels = np.concatenate([[0], np.cumsum(np.diff(sorted_b) > self.shell_epsilon)])
        index = np.full(len(self.bvals), -1)
        index[weighted[order]] = labels[: len(weighted)]
        return index

    @property
    def shells(self) -> np.ndarray:
        index = self.shell_index
        if index.max() < 0:
            return np.zeros(0)
        return np.array([self.bvals[index == k].mean() for k in range(index.max() + 1)])

    def count_shells(self, *, above: float = 0.0) -> int:
        return int(np.count_nonzero(self.shells > above))
