"""Drop-in replacement for the reference's GPU render/score launchers.

Same names, signatures and argument meaning as ``src/weft/gpu_render.py``:

* ``gpu_batch_score_prepacked`` (:455-566) — MSE of every (tile, stack) eval;
* ``gpu_batch_objectives`` (:737-845) — MSE of several stacks on one tile;
* ``gpu_render_tiles_to_image`` (:594-690) — the decoder's primitive walk;
* ``_PRIM_DTYPE`` / ``_TILE_DECODE_DTYPE`` / ``_pack_prims`` / ``_pack_one``.

Installing this module's functions as attributes of the reference module
(``weft_b200.install_into(weft.gpu_render)``) makes the reference encoder and
decoder run on libweftk, because the reference imports the launcher inside the
calling function (src/weft/encoder.py:2655).

Differences from the reference, on purpose:

* errors raise ``WeftkError`` instead of returning ``None`` — a ``None``
  makes the reference fit silently degrade to one candidate per tile, which
  is a CPU fallback in disguise;
* samples are taken at pixel centres (the reference CPU renderer's
  convention, src/weft/render.py:29-49) rather than the reference GPU
  scorer's integer corners; ``sample_corner=True`` reproduces the latter;
* alpha is clamped to [0, 1] and the render is clipped before the error, as
  in the reference CPU objective (src/weft/encoder.py:271-285);
* the decode walk renders a square max(w, h) grid and crops, as the CPU walk
  does (src/weft/render.py:326-346); ``_TILE_DECODE_DTYPE``'s ``_pad`` field
  is read as a RES1 grid index only by ``weft_b200.render``.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from ._lib import PRIM_DTYPE as _PRIM_DTYPE
from ._lib import EVAL_DTYPE
from ._lib import TILE_DECODE_DTYPE as _TILE_DECODE_DTYPE

__all__ = ["gpu_batch_score_prepacked", "gpu_batch_objectives", "gpu_render_tiles_to_image", "_PRIM_DTYPE",
           "_TILE_DECODE_DTYPE", "_pack_prims", "_pack_one"]

_FLAG_CORNER = 1


def _pack_one(p, out: np.ndarray, idx: int) -> None:
    """Pack one primitive into ``out[idx]`` (reference _pack_one, src/weft/gpu_render.py:250-269)."""
    out[idx]["kind"] = p.kind
    g = tuple(p.geom)[:7]
    out[idx]["geom"] = g + (0.0,) * (7 - len(g))
    out[idx]["color0"] = p.color0
    out[idx]["color1"] = p.color1 if p.color1 is not None else (0.0, 0.0, 0.0)
    out[idx]["alpha"] = p.alpha


def _pack_prims(prims) -> np.ndarray:
    """Pack primitives into 60-byte records; at least one (zero) record (src/weft/gpu_render.py:272-308)."""
    n = len(prims)
    arr = np.zeros(max(1, n), dtype=_PRIM_DTYPE)
    if n == 0:
        return arr
    arr["kind"][:n] = [p.kind for p in prims]
    arr["alpha"][:n] = [p.alpha for p in prims]
    arr["color0"][:n] = [tuple(p.color0) for p in prims]
    arr["color1"][:n] = [tuple(p.color1) if p.color1 is not None else (0.0, 0.0, 0.0) for p in prims]
    arr["geom"][:n] = [tuple(p.geom)[:7] + (0.0,) * (7 - min(7, len(p.geom))) for p in prims]
    return arr


def _score(evals: np.ndarray, prims: np.ndarray, pixels: np.ndarray, sample_corner: bool) -> np.ndarray:
    lib = _lib.lib_for_device(0)
    evals = np.ascontiguousarray(evals, dtype=EVAL_DTYPE)
    prims = np.ascontiguousarray(prims, dtype=_PRIM_DTYPE)
    pixels = np.ascontiguousarray(pixels, dtype=np.float32)
    out = np.empty(len(evals), dtype=np.float32)
    rc = lib.weftk_score_evals_host(_lib.ptr(evals), len(evals), _lib.ptr(prims), len(prims), _lib.ptr(pixels),
                                    pixels.size, _lib.ptr(out), _FLAG_CORNER if sample_corner else 0)
    _lib.check(rc, "weftk_score_evals_host")
    return out


def gpu_batch_score_prepacked(tile_pixels_flat, tile_pixel_offsets, tile_indices, tile_sizes, eval_prim_arrays,
                              eval_prim_counts, *, sample_corner: bool = False) -> list[np.ndarray]:
    """Score pre-packed candidate stacks for many tiles in one launch.

    Args mirror the reference: all tile pixels concatenated (float32, HWC per
    tile); ``{tile_index: float offset}``; the tiles to score; their sizes;
    per tile a flat record array holding the stacks back to back; per tile the
    stack length of each eval.  Returns one float32 MSE array per tile.
    """
    counts = [np.asarray(c, dtype=np.int64) for c in eval_prim_counts]
    total = int(sum(len(c) for c in counts))
    if total == 0:
        return [np.empty(0, dtype=np.float32) for _ in tile_indices]
    evals = np.empty(total, dtype=EVAL_DTYPE)
    ranges = []
    e0 = 0
    p0 = 0
    for j, ti in enumerate(tile_indices):
        c = counts[j]
        n = len(c)
        offs = np.zeros(n, np.int64)
        if n > 1:
            np.cumsum(c[:-1], out=offs[1:])
        evals["prim_offset"][e0:e0 + n] = p0 + offs
        evals["prim_count"][e0:e0 + n] = c
        evals["tile_offset"][e0:e0 + n] = int(tile_pixel_offsets[ti])
        evals["tile_size"][e0:e0 + n] = int(tile_sizes[j])
        ranges.append((e0, n))
        e0 += n
        p0 += len(eval_prim_arrays[j])
    prims = np.concatenate([np.asarray(a, dtype=_PRIM_DTYPE) for a in eval_prim_arrays]) if eval_prim_arrays \
        else np.zeros(1, _PRIM_DTYPE)
    mse = _score(evals, prims, tile_pixels_flat, sample_corner)
    return [mse[a:a + n].copy() for a, n in ranges]


def gpu_batch_objectives(tile: np.ndarray, prim_sets, *, sample_corner: bool = False) -> np.ndarray:
    """MSE of each primitive set rendered over ``tile`` (float32, shape (len(prim_sets),))."""
    n = len(prim_sets)
    if n == 0:
        return np.empty(0, dtype=np.float32)
    ts = int(tile.shape[0])
    packed = [_pack_prims(s) for s in prim_sets]
    counts = np.array([len(s) for s in prim_sets], np.int64)
    sizes = np.array([len(p) for p in packed], np.int64)
    evals = np.empty(n, dtype=EVAL_DTYPE)
    evals["prim_offset"] = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    evals["prim_count"] = counts
    evals["tile_offset"] = 0
    evals["tile_size"] = ts
    return _score(evals, np.concatenate(packed), np.asarray(tile, np.float32).reshape(-1), sample_corner)


def gpu_render_tiles_to_image(tile_descs, all_prims, output_height, output_width) -> np.ndarray:
    """Render packed tiles into a zero-initialised (H, W, 3) float32 image."""
    lib = _lib.lib_for_device(0)
    descs = np.ascontiguousarray(tile_descs, dtype=_TILE_DECODE_DTYPE)
    prims = np.ascontiguousarray(all_prims, dtype=_PRIM_DTYPE)
    out = np.empty((int(output_height), int(output_width), 3), dtype=np.float32)
    rc = lib.weftk_render_tiles_host(_lib.ptr(descs), len(descs), _lib.ptr(prims), len(prims), 0, 0, 0, 0,
                                     _lib.ptr(out), int(output_height), int(output_width), 0)
    _lib.check(rc, "weftk_render_tiles_host")
    return out
