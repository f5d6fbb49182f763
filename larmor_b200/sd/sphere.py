"""Direction sets on the sphere (src/larmor/sd/sphere.py)."""

from __future__ import annotations

from pathlib import Path

import numpy as np

# The 300 unit directions FODs are evaluated on (the reference's src/larmor/data/dir300.txt).
DIRS_300 = np.load(Path(__file__).resolve().parents[1] / "data" / "dirs300.npy")


def get_theta_phi(dirs: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Polar angle from +z and azimuth from +x of unit vectors (n, 3)."""
    return np.arccos(dirs[:, 2]), np.arctan2(dirs[:, 1], dirs[:, 0])


def get_dirs(n_dirs: int = 45) -> np.ndarray:
    """n_dirs roughly uniform unit vectors on a Saff-Kuijlaars spiral, flipped to z >= 0; the
    first and the last are the poles, both +z (src/larmor/sd/sphere.py:get_dirs)."""
    phis: list[float] = []
    dirs = []
    for k in range(1, n_dirs + 1):
        h = -1 + 2 * (k - 1) / (n_dirs - 1)
        theta = np.arccos(h)
        if k == 1 or k == n_dirs:
            phi = 0
        else:
            phi = (phis[-1] + 3.6 / np.sqrt(n_dirs * (1 - h**2))) % (2 * np.pi)
        phis.append(phi)
        x, y, z = np.cos(phi) * np.sin(theta), np.sin(phi) * np.sin(theta), np.cos(theta)
        sz = np.sign(z)
        dirs.append([x * sz, y * sz, z * sz])
    return np.asarray(dirs)
