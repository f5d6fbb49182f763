"""Deconvolution kernels built from response functions (src/larmor/sd/kernel.py)."""

from __future__ import annotations

from collections.abc import Sequence

import numpy as np

from larmor_b200.sd.rf import IsotropicRF, ResponseFunction


def order_rfs(rfs: list[ResponseFunction]) -> list[ResponseFunction]:
    """The responses with the anisotropic ones first."""
    return [rf for rf in rfs if not isinstance(rf, IsotropicRF)] + [rf for rf in rfs if isinstance(rf, IsotropicRF)]


class Kernel:
    """The signal of each response along each direction (n_meas, n_cols), with per-response
    column blocks (anisotropic ones first) and the copy `w_k` weighted per measurement."""

    def __init__(self, rfs, bvals, bvecs, dirs: np.ndarray | Sequence[np.ndarray] | None = None,
                 weights: np.ndarray | None = None) -> None:
        if dirs is None and any(not isinstance(rf, IsotropicRF) for rf in rfs):
            raise ValueError("dirs is required for an anisotropic response function.")
        self.weights = np.ones(len(bvals)) if weights is None else weights
        self.rfs = order_rfs(rfs)
        self.num_iso = sum(1 for rf in self.rfs if isinstance(rf, IsotropicRF))
        n_aniso = len(self.rfs) - self.num_iso
        if dirs is None:
            per_rf = [np.empty((0, 3))] * len(self.rfs)
        elif isinstance(dirs, np.ndarray):
            per_rf = [dirs] * len(self.rfs)
        else:
            if len(dirs) != n_aniso:
                raise ValueError(f"dirs has {len(dirs)} direction sets for {n_aniso} anisotropic response functions.")
            per_rf = [*dirs, *([np.empty((0, 3))] * self.num_iso)]
        blocks, self.blocks, start = [], [], 0
        for rf, rf_dirs in zip(self.rfs, per_rf, strict=True):
            block = rf.signal(bvals, bvecs, rf_dirs)
            blocks.append(block)
            self.blocks.append(slice(start, start + block.shape[1]))
            start += block.shape[1]
        self.k = np.hstack(blocks)
        self.w_k = self.k * self.weights[:, np.newaxis]
        self.aniso_blocks = self.blocks[: len(self.rfs) - self.num_iso]
        self.k_aniso, self.k_iso = self._split(self.k)
        self.w_k_aniso, self.w_k_iso = self._split(self.w_k)

    def _split(self, k: np.ndarray):
        if self.num_iso == 0:
            return k, None
        return k[:, : -self.num_iso], k[:, -self.num_iso:]
