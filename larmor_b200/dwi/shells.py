"""The volumes of a b-value shell (src/larmor/dwi/shells.py)."""

from __future__ import annotations

import numpy as np

# How far, in s/mm^2, a b-value may lie from a shell's to belong to it.
SHELL_TOLERANCE = 100.0


def shell_mask(bvals: np.ndarray, shell: float, *, tol: float = SHELL_TOLERANCE) -> np.ndarray:
    """True for the volumes whose b-value is within tol of shell, strictly (shape (N,))."""
    return np.abs(bvals - shell) < tol
