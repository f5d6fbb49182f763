"""Extraction of the peaks of FODs on the GPU, with the API of larmor.sd.peaks
(src/larmor/sd/peaks.py).

find_peaks keeps the reference's arguments, checks, thresholds and output layout. Underneath,
the selected voxels' series go to the device once per chunk; their amplitudes on the
642-vertex icosphere are one FP64 product with the basis matrix there (project_sh_kernel, the
reference's _get_amplitudes), and the peak search of every voxel is one launch of peaks_kernel
(the reference's _core.peaks_chunk). Only the directions and amplitudes come back.
"""

from __future__ import annotations

import functools
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from larmor_b200 import _core
from larmor_b200._threads import n_threads
from larmor_b200.sd.sh import build_basis_matrix, convert_sh_basis, sh_layout
from larmor_b200.sd.sphere import get_theta_phi

# The largest lmax the search handles.
MAX_LMAX = _core.MAX_LMAX
#: The default relative peak threshold, for FODs fitted as SH coefficients (CSD, MSMT-CSD) and
#: FODs from other software.
PEAK_RELATIVE_THRESHOLD = 0.1
#: The relative peak threshold for the FODs of SDModel (GRL and mFOD), whose truncation to SH
#: leaves side lobes where fibres cross.
SD_MODEL_PEAK_RELATIVE_THRESHOLD = 0.2

# Voxels per device chunk: their icosphere amplitudes take 5 KiB each on the device.
DEVICE_CHUNK = 1 << 17

_ICOSPHERE = Path(__file__).resolve().parents[1] / "data" / "icosphere642.npz"


@functools.cache
def _build_icosphere() -> tuple[np.ndarray, np.ndarray]:
    """The 642 unit vectors of an icosahedron subdivided three times, and the 6 neighbours of
    each (a vertex with 5 lists itself as the sixth): the reference's table
    (src/larmor/sd/peaks.py:_build_icosphere), in its vertex order, which is the order the
    search merges its climbs in."""
    with np.load(_ICOSPHERE) as z:
        return z["vertices"], z["neighbours"]


@functools.cache
def _basis(lmax: int, full: bool) -> np.ndarray:
    vertices, _ = _build_icosphere()
    theta, phi = get_theta_phi(vertices)
    return np.ascontiguousarray(build_basis_matrix(theta, phi, lmax, full=full))


def _get_amplitudes(coeffs: np.ndarray, lmax: int, full: bool) -> np.ndarray:
    """The amplitude of each FOD on each vertex of the icosphere (host, for callers of
    peaks_chunk)."""
    return coeffs @ _basis(lmax, full).T


@functools.lru_cache(maxsize=8)
def _amplitude_projector(lmax: int, full: bool) -> _core.ShProjector:
    return _core.ShProjector(_basis(lmax, full))


@dataclass(frozen=True)
class Peaks:
    """Holds the directions and amplitudes of FOD peaks that `find_peaks` returns.

    Attributes:
        directions: Unit vectors along the peaks, shape (..., P, 3) where P is the number of
            peaks asked for. Sorted by amplitude, largest first. If fewer than P peaks are
            found, the remaining ones are NaN. A symmetric FOD's peaks have z >= 0; an
            asymmetric FOD's keep their sign, since a peak and its opposite are two lobes.
        amplitudes: Amplitude of each peak, shape (..., P), NaN where directions is NaN.
    """

    directions: np.ndarray
    amplitudes: np.ndarray


def find_peaks(
    coeffs: np.ndarray,
    mask: np.ndarray | None = None,
    *,
    basis: str = "tournier",
    num_peaks: int | None = None,
    relative_threshold: float = PEAK_RELATIVE_THRESHOLD,
    threshold: float = 0.0,
    chunk_size: int = 10_000,
    n_jobs: int = -1,
) -> Peaks:
    """Extracts the peaks of FODs (src/larmor/sd/peaks.py:find_peaks).

    The maxima of the FOD's amplitude are found by climbing from the vertices of an
    icosphere, and peaks closer than 0.99 in |cos| are merged. Maxima with an amplitude of 0
    or below are dropped, as are those under `threshold` and those under `relative_threshold`
    times the largest peak. An asymmetric FOD (all SH degrees) is searched the same way, but a
    peak and its opposite are two peaks, merged only when closer than 0.99 in signed cos, and
    peaks keep their sign.

    Args:
        coeffs: FOD coefficients, shape (..., C), the even degrees of a symmetric FOD or all
            degrees of an asymmetric one.
        mask: Voxels to search, shape (...); the other voxels are NaN. Defaults to every voxel.
        basis: SH basis of the FODs. Defaults to "tournier".
        num_peaks: Number of peaks to extract. Defaults to 3 for a symmetric FOD and 6 for an
            asymmetric one.
        relative_threshold: Fraction of the largest peak below which a peak is dropped.
        threshold: Amplitude below which a peak is dropped.
        chunk_size: Accepted for compatibility and checked; the device works in chunks of
            DEVICE_CHUNK voxels, and the results do not depend on either.
        n_jobs: Accepted for compatibility and checked; the results do not depend on it.

    Returns:
        Peaks: The peaks extracted.

    Raises:
        ValueError: If num_peaks or chunk_size is below 1, if n_jobs is 0 or below -1, if
            relative_threshold is not between 0 and 1, if mask does not have the shape of
            coeffs without its last axis, if the coefficient count fits no SH layout or
            convert_sh_basis refuses the basis, or if lmax is above 20.
    """
    if num_peaks is not None and num_peaks < 1:
        raise ValueError(f"num_peaks must be at least 1, got {num_peaks}")
    if chunk_size < 1:
        raise ValueError(f"chunk_size must be at least 1, got {chunk_size}")
    n_threads(n_jobs)
    if not 0 <= relative_threshold <= 1:
        raise ValueError(f"relative_threshold must be between 0 and 1, got {relative_threshold}")

    coeffs = np.asarray(coeffs)
    num_coeffs = coeffs.shape[-1]
    leading = coeffs.shape[:-1]
    if mask is None:
        selected = np.ones(leading, dtype=bool)
    else:
        mask = np.asarray(mask)
        if mask.shape != leading:
            raise ValueError(f"mask has shape {mask.shape}, but the coefficients have {leading} voxels")
        selected = mask.astype(bool)

    lmax, full = sh_layout(num_coeffs)
    if num_peaks is None:
        num_peaks = 6 if full else 3
    if lmax > MAX_LMAX:
        raise ValueError(f"lmax must be at most {MAX_LMAX}, got {lmax}")
    voxels = np.ascontiguousarray(convert_sh_basis(coeffs[selected], basis, "tournier"), dtype=np.float64)
    found_dirs, found_amps = find_peaks_of_series(voxels, lmax, full, num_peaks, relative_threshold, threshold)

    directions = np.full((*leading, num_peaks, 3), np.nan)
    amplitudes = np.full((*leading, num_peaks), np.nan)
    directions[selected] = found_dirs
    amplitudes[selected] = found_amps
    return Peaks(directions, amplitudes)


def find_peaks_of_series(voxels: np.ndarray, lmax: int, full: bool, num_peaks: int, relative_threshold: float,
                         threshold: float) -> tuple[np.ndarray, np.ndarray]:
    """The peaks of (n, C) tournier series on the device: directions (n, num_peaks, 3) and
    amplitudes (n, num_peaks) as host arrays."""
    torch = _core._torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    vertices, neighbours = _build_icosphere()
    sphere = _core.PeakSphere.cached(vertices, neighbours)
    projector = _amplitude_projector(lmax, full)
    n = voxels.shape[0]
    out_dirs = np.empty((n, num_peaks, 3))
    out_amps = np.empty((n, num_peaks))
    for start in range(0, n, DEVICE_CHUNK):
        stop = min(n, start + DEVICE_CHUNK)
        block = torch.from_numpy(voxels[start:stop]).to(dev)
        on_sphere = _core.project_sh_device(projector, block, exact_integral=False)
        dirs, amps = _core.find_peaks_device(sphere, block, lmax, full, on_sphere, num_peaks, relative_threshold,
                                             threshold)
        out_dirs[start:stop] = dirs.cpu().numpy()
        out_amps[start:stop] = amps.cpu().numpy()
    return out_dirs, out_amps
