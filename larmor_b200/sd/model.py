"""Spherical deconvolution results (src/larmor/sd/model.py:48-81)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class SDFit:
    """FODs (one per anisotropic response, SH coefficients (X, Y, Z, C) in `basis`), tissue
    fractions (X, Y, Z, N) or None for a single-tissue fit, the lmax used, and the relative
    threshold to give peak finding."""

    fods: list[np.ndarray]
    tissue_fractions: np.ndarray | None
    basis: str
    lmax: int
    peak_relative_threshold: float = 0.1
