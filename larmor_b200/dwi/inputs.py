"""Input checks and signal preparation of the DWI fits (src/larmor/dwi/inputs.py).

The host checks the volume, table and mask; the preparation of the fit's inputs -- the gather of
the mask voxels' float32 signals, the S0 estimate with its neighbourhood repair and the per-voxel
floor of samples that are not finite and positive -- runs on the device (lar_stage_dwi).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from larmor_b200.types import GradientTable, Volume


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
    """S0 on the volume's grid (float64): each voxel's mean b0; inside the mask, a voxel whose
    mean b0 is not above its mean diffusion-weighted sample takes the mean S0 of the plausible
    mask voxels in its 3x3x3, else 5x5x5, neighbourhood, NaN when there is none
    (src/larmor/dwi/inputs.py:78-134). The mask voxels' S0 and its repair come from the device
    staging (lar_stage_dwi); outside the mask S0 is the plain b0 mean.

    Raises:
        ValueError: If the volume and table do not match or the table has no b0.
    """
    check_dwi(volume, gtab)
    is_b0 = gtab.b0_mask
    if not np.any(is_b0):
        raise ValueError(f"No b0 volume: no b-value is at or below {gtab.b0_threshold} s/mm^2.")
    mask = as_mask(volume, mask)
    s0 = volume.as_float()[..., is_b0].sum(axis=-1, dtype=np.float64) / int(is_b0.sum())
    if mask.any():
        s0[mask] = stage_dwi(volume, gtab, mask).s0.cpu().numpy()
    return s0


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
    flat: object = None  # the mask voxels' flat grid indices, an int64 device tensor

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
    raw = _core._on_device(torch, data.reshape(-1).view(np.uint8), dev)
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
    return StagedDwi(mask, signals, s0, finite, floor, largest, d_voxels)


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
