"""The per-tile bicubic R-D swap of the adaptive fit on the GPU.

The reference computes, at the end of ``_fit_adaptive_state`` (src/weft/encoder.py:2841-2873),
an alternative stack list ``bicubic_replaced_per_tile``: each tile keeps its selected stack or
becomes one bicubic primitive (kind 5, a 4x4x3 Bezier control grid rounded to u8 steps),
whichever scores lower by ``mse + lambda * bits``.  ``swap`` runs that decision for every tile
at once through ``weftk_bicubic_swap``; ``replaced_stacks`` builds the reference's list from it.
"""

from __future__ import annotations

import ctypes
from functools import lru_cache

import numpy as np
import torch

from . import _lib, rate
from .candidates import Cand
from .fit import pack_cands

SIDES = (8, 16, 32, 64)
BASIS_DOUBLES = 1440  # WEFTK_BICUBIC_BASIS_DOUBLES


@lru_cache(maxsize=1)
def basis_table() -> np.ndarray:
    """pinv(B), pinv(B^T) and B for each tile side, float64, in the layout of
    WEFTK_BICUBIC_BASIS_DOUBLES; the pseudo-inverses come from numpy.linalg.pinv as in the
    reference (src/weft/bicubic.py:31-57)."""
    parts = []
    for n in SIDES:
        t = np.linspace(0.0, 1.0, n, dtype=np.float64)
        B = np.stack([(1.0 - t) ** 3, 3.0 * (1.0 - t) ** 2 * t, 3.0 * (1.0 - t) * t ** 2, t ** 3], axis=-1)
        parts += [np.linalg.pinv(B).reshape(-1), np.linalg.pinv(B.T).reshape(-1), B.reshape(-1)]
    out = np.ascontiguousarray(np.concatenate(parts), np.float64)
    assert out.size == BASIS_DOUBLES
    return out


def swap(src4: torch.Tensor, px_off: torch.Tensor, sizes: torch.Tensor, stacks, quality: int,
         device: int | None = None) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Run the swap decision for every tile.

    ``src4``: float32 CUDA tensor (n_pixels, 4), tile t's side x side pixels row-major from
    ``px_off[t]`` (int32 CUDA tensor); ``sizes``: int32 CUDA tensor of tile sides; ``stacks``:
    the selected stack of every tile (lists of primitives with ``kind``, ``geom``, ``color0``,
    ``color1``, ``alpha``).  Returns (replace flags (n,) bool, u8-rounded control grids (n, 48)
    float32, scores (n, 2) float64: bicubic, stack)."""
    dev = src4.device
    idx = dev.index if device is None else device
    lib = _lib.lib_for_device(idx)
    n = int(sizes.numel())
    recs = pack_cands([p for s in stacks for p in s])
    counts = np.array([len(s) for s in stacks], np.int64)
    prim_off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    t_prims = torch.from_numpy(recs.view(np.uint8)).to(dev) if len(recs) else None
    t_off = torch.from_numpy(prim_off).to(dev)
    t_basis = torch.from_numpy(basis_table()).to(dev)
    grid = torch.empty((n, 48), dtype=torch.float32, device=dev)
    flags = torch.empty(n, dtype=torch.int32, device=dev)
    scores = torch.empty((n, 2), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    _lib.check(lib.weftk_bicubic_swap(_lib.ptr(src4), _lib.ptr(px_off), _lib.ptr(sizes), n, _lib.ptr(t_prims),
                                      len(recs), _lib.ptr(t_off), _lib.ptr(t_basis), float(rate.tile_lambda(quality)),
                                      _lib.ptr(grid), _lib.ptr(flags), _lib.ptr(scores), stream.cuda_stream),
               "weftk_bicubic_swap")
    torch.cuda.synchronize(dev)
    st = ctypes.c_int(0)
    _lib.check(lib.weftk_device_status(ctypes.addressof(st)), "weftk_device_status")
    if st.value:
        raise _lib.WeftkError(f"weftk_bicubic_swap reported status {st.value} (tile side or stack length)")
    return flags.cpu().numpy().astype(bool), grid.cpu().numpy(), scores.cpu().numpy()


def replaced_stacks(stacks, flags: np.ndarray, grids: np.ndarray) -> list[list]:
    """The reference's ``bicubic_replaced_per_tile``: a tile marked for replacement becomes one
    kind-5 primitive whose geometry is the 48 control values (src/weft/encoder.py:2866-2873)."""
    out = []
    for s, f, g in zip(stacks, flags, grids):
        out.append([Cand(5, tuple(float(v) for v in g), (0.0, 0.0, 0.0), None, 1.0)] if f else list(s))
    return out
