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


def unmask_maps(maps, groups, flat, shape, flags=None) -> dict:
    """The model maps on the grid, put back there on the device: maps is a map-major (rows, v)
    float32 device tensor of the mask voxels, flat their flat grid indices (an int64 device
    tensor), groups (name, first row, rows) the outputs. Each output becomes a float32 grid array
    (shape, or shape + (rows,) for rows > 1), zero outside the mask; flags (v,), a uint8 device
    tensor, becomes the boolean grid array "flags". One scatter per output into one device
    buffer (lar_unmask_rows), then one copy to the host: the arrays are views of that copy."""
    from larmor_b200 import _core, _lib

    torch = _core._torch()
    grid = int(np.prod(shape))
    v = int(maps.shape[1])
    rows_total = sum(rows for _, _, rows in groups) + (1 if flags is not None else 0)
    out = torch.zeros(grid * rows_total, dtype=torch.float32, device=maps.device)
    stream = _core._stream(torch)
    pieces, offset = [], 0
    sources = [(name, maps[first:first + rows], rows) for name, first, rows in groups]
    if flags is not None:
        sources.append(("flags", flags.to(torch.float32)[None], 1))
    for name, values, rows in sources:
        if v:
            _lib.check(_lib.lib().lar_unmask_rows(_lib.ptr(values.contiguous()), rows, v, _lib.ptr(flat), grid,
                                                  _lib.ptr(out[offset:]), stream))
        pieces.append((name, offset, rows))
        offset += grid * rows
    host = _core._to_host(out)
    result = {}
    for name, start, rows in pieces:
        piece = host[start:start + grid * rows].reshape(tuple(shape) + ((rows,) if rows > 1 else ()))
        result[name] = piece > 0.5 if name == "flags" else piece
    return result
