"""Input checks and signal preparation of the DWI fits (src/larmor/dwi/inputs.py).

These host steps run once per volume, before the device fit: the mask check, the S0 estimate
with its neighbourhood repair, the per-voxel floor of samples that are not finite and positive,
and the gather of the masked voxels' float32 signals.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.ndimage import uniform_filter

from larmor_b200.types import GradientTable, Volume

# Neighbourhood widths searched, in order, for the S0 of a voxel whose b0s are implausible.
S0_NEIGHBOURHOODS = (3, 5)
# Fraction of S0 that replaces a measurement that is not finite and positive.
SIGNAL_FLOOR = 1e-3


def check_dwi(volume: Volume, gtab: GradientTable) -> None:
    """Raises ValueError unless volume is 4D with one table entry per volume."""
    if volume.data.ndim != 4:
        raise ValueError(f"A DWI is 4D, (X, Y, Z, N); got a volume of shape {volume.data.shape}.")
    if len(gtab.bvals) != volume.data.shape[3]:
        raise ValueError(
            f"The gradient table has {len(gtab.bvals)} entries, the volume has "
            f"{volume.data.shape[3]} volumes."
        )


def as_mask(volume: Volume, mask) -> np.ndarray:
    """The mask as booleans on the volume's grid (nonzero inside)."""
    data = mask.data if isinstance(mask, Volume) else np.asarray(mask)
    shape = volume.data.shape[:3]
    if data.shape != shape:
        raise ValueError(f"The mask has shape {data.shape}, the volume's grid is {shape}.")
    return data != 0


def estimate_s0(volume: Volume, gtab: GradientTable, mask: np.ndarray) -> np.ndarray:
    """S0 of every voxel: the mean b0, repaired from plausible neighbours where the voxel's own
    b0s are at or below its mean diffusion-weighted signal (src/larmor/dwi/inputs.py:78-134)."""
    check_dwi(volume, gtab)
    is_b0 = gtab.b0_mask
    if not np.any(is_b0):
        raise ValueError(f"No b0 volume: no b-value is at or below {gtab.b0_threshold} s/mm^2.")
    data = volume.as_float()
    b0_sum = data[..., is_b0].sum(axis=-1, dtype=np.float64)
    s0 = b0_sum / is_b0.sum()
    n_dw = int((~is_b0).sum())
    if n_dw == 0:
        return s0
    mean_dw = (data.sum(axis=-1, dtype=np.float64) - b0_sum) / n_dw
    finite = np.isfinite(s0) & np.isfinite(mean_dw)
    plausible = mask & finite & (s0 > mean_dw)
    to_repair = mask & finite & ~plausible
    repaired = np.full(s0.shape, np.nan)
    for width in S0_NEIGHBOURHOODS:
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


def masked_signals(volume: Volume, voxels: tuple[np.ndarray, ...]) -> np.ndarray:
    """The scaled float32 signals (v, N) of the given voxels, scaled as Volume.as_float does."""
    signal = volume.data[voxels]
    scaled = signal.astype(np.float32)
    if volume.slope != 1.0 or volume.intercept != 0.0:
        scaled *= np.float32(volume.slope)
        scaled += np.float32(volume.intercept)
    return np.ascontiguousarray(scaled)


def largest_finite_signal(signals: np.ndarray) -> float:
    """The largest finite value of the signals, or 1 when none is positive."""
    finite = signals[np.isfinite(signals)]
    largest = float(finite.max()) if finite.size else -np.inf
    return largest if largest > 0 else 1.0


def sample_floors(s0: np.ndarray | None, largest: float | None, v: int) -> np.ndarray:
    """The value (v,) that replaces each voxel's samples that are not finite and positive:
    1e-3 S0 where S0 is finite and positive, else 1e-3 times the largest finite signal
    (src/larmor/dwi/inputs.py:227-252)."""
    floor = np.full(v, SIGNAL_FLOOR * (1.0 if largest is None else largest))
    if s0 is not None:
        usable = np.isfinite(s0) & (s0 > 0)
        floor[usable] = SIGNAL_FLOOR * s0[usable]
    return floor


@dataclass
class StagedDwi:
    """The inputs of a fit, staged on the device from the raw volume (lar_stage_dwi).

    mask is the voxels' mask (their order is np.nonzero's); signals (v, N) float32, s0 (v)
    float64 or None for a table without b0, finite (v) uint8 (every sample finite) and floor (v)
    float64 are device tensors; largest is a (1,) device tensor."""

    mask: np.ndarray
    signals: object
    s0: object
    finite: object
    floor: object
    largest: object

    @property
    def voxels(self) -> tuple[np.ndarray, ...]:
        """The mask voxels' indices, np.nonzero of the mask."""
        return np.nonzero(self.mask)


def upload_volume(volume: Volume):
    """The raw samples of a 4D volume on the device as bytes, with their lar_stage_dwi type code.

    Raises:
        ValueError: If the sample type is not one of the integer or float types the staging reads.
    """
    from larmor_b200 import _core, _lib

    data = np.ascontiguousarray(volume.data)
    code = _lib.LAR_DTYPES.get(str(data.dtype))
    if code is None:
        raise ValueError(f"The volume's samples are {data.dtype}; the device staging reads "
                         f"{', '.join(_lib.LAR_DTYPES)}.")
    torch = _core._torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    raw = torch.empty(data.nbytes, dtype=torch.uint8, device=dev)
    raw.copy_(torch.from_numpy(data.reshape(-1).view(np.uint8)))
    return raw, code


def stage_dwi(volume: Volume, gtab: GradientTable, mask: np.ndarray, *, raw=None, flat=None) -> StagedDwi:
    """Stages the mask voxels' samples on the device: the raw volume is copied to the device once
    and the reference's host preparation -- the float32 scaling, estimate_s0 with its
    neighbourhood repair, largest_finite_signal and the per-voxel floor -- runs there
    (lar_stage_dwi; src/larmor/dwi/inputs.py:78-252). raw: the volume already on the device, as
    upload_volume returns it; flat: the mask voxels' flat grid indices already on the device
    (int64, np.flatnonzero of the mask).

    Raises:
        ValueError: If the volume and table do not match, or the volume's sample type is not
            one of the integer or float types the staging reads.
    """
    from larmor_b200 import _core, _lib

    check_dwi(volume, gtab)
    if raw is None:
        raw = upload_volume(volume)
    data, code = raw
    torch = _core._torch()
    dev = data.device
    nx, ny, nz, n = volume.data.shape
    d_voxels = torch.from_numpy(np.flatnonzero(mask).astype(np.int64)).to(dev) if flat is None else flat
    v = d_voxels.shape[0]
    is_b0 = np.ascontiguousarray(gtab.b0_mask, dtype=np.uint8)
    signals = torch.empty((v, n), dtype=torch.float32, device=dev)
    s0 = torch.empty((v,), dtype=torch.float64, device=dev) if is_b0.any() else None
    finite = torch.empty((v,), dtype=torch.uint8, device=dev)
    floor = torch.empty((v,), dtype=torch.float64, device=dev)
    largest = torch.empty((1,), dtype=torch.float64, device=dev)
    _lib.check(_lib.lib().lar_stage_dwi(
        _lib.ptr(data), code, nx, ny, nz, n, float(volume.slope), float(volume.intercept), _lib.ptr(d_voxels), v,
        is_b0.ctypes.data, _lib.ptr(signals), _lib.ptr(s0), _lib.ptr(finite), _lib.ptr(floor), _lib.ptr(largest),
        _core._stream(torch)))
    return StagedDwi(mask, signals, s0, finite, floor, largest)


def normalise_signals(signals, s0):
    """min(signals / s0, 1) in FP64 on the device and whether each row is finite
    (lar_normalise_signals; the SD models' normalisation, src/larmor/sd/model.py:184-200)."""
    from larmor_b200 import _core, _lib

    torch = _core._torch()
    v, n = signals.shape
    out = torch.empty((v, n), dtype=torch.float64, device=signals.device)
    finite = torch.empty((v,), dtype=torch.uint8, device=signals.device)
    _lib.check(_lib.lib().lar_normalise_signals(_lib.ptr(signals), _lib.ptr(s0), v, n, _lib.ptr(out),
                                                _lib.ptr(finite), _core._stream(torch)))
    return out, finite


def mean_b0(volume: Volume, gtab: GradientTable) -> np.ndarray:
    check_dwi(volume, gtab)
    is_b0 = gtab.b0_mask
    if not np.any(is_b0):
        raise ValueError(f"No b0 volume: no b-value is at or below {gtab.b0_threshold} s/mm^2.")
    return np.mean(volume.as_float()[..., is_b0], axis=-1)
