"""Decoder primitive walk on the GPU (host side).

``render_scene_adaptive`` keeps the reference's signature and semantics
(src/weft/render.py:270-358): each quadtree tile's stack is rendered into its
integer target rect (edges ``round(x * scale)``), sampling the tile's
``[0, size]`` primitive space at pixel centres of a square ``max(w, h)`` grid
that is cropped for anisotropic targets; RES0 is added and clipped, then the
bilinear RES1 grid, then clipped again.  All pixels are produced by
``weftk_render_tiles`` (one launch for the whole image); the host only packs
descriptors.

``render_tile`` renders one stack as a single tile (the reference's
``render_tile``, src/weft/render.py:127-234) through the same kernel.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from ._lib import PRIM_DTYPE, TILE_DECODE_DTYPE

MAX_TILE_PRIMS = 48
DECODE_ITEM_GROUPS = 256   # WEFTK_DECODE_ITEM_GROUPS
ITEM_PIXEL_WORK = 4        # cost of a pixel evaluated per pixel, in pixels of a constant fill


def decode_items(descs: np.ndarray, out_h: int, out_w: int, prims: np.ndarray | None = None) -> np.ndarray:
    """Work items (tile, first row) of weftk_render_tiles, int32 (n, 2), in descending cost order.

    A rect row touches G 4-pixel groups aligned to output x multiples of 4; an item covers
    max(1, DECODE_ITEM_GROUPS // G) rows of its tile.  Only the rows inside the out_h x out_w
    image get items.  The cost of an item is its pixel count, times ITEM_PIXEL_WORK for a tile
    that is evaluated per pixel (anything but a lone constant layer without a RES1 grid; with
    ``prims`` None every tile without a RES1 grid counts as a lone constant layer).
    """
    x0 = descs["target_x0"].astype(np.int64)
    y0 = descs["target_y0"].astype(np.int64)
    w = descs["target_w"].astype(np.int64)
    h = descs["target_h"].astype(np.int64)
    g = np.floor_divide(x0 + w + 3, 4) - np.floor_divide(x0, 4)
    rows = np.maximum(1, DECODE_ITEM_GROUPS // np.maximum(g, 1))
    r0 = np.maximum(0, -y0)
    r1 = np.minimum(h, out_h - y0)
    visible = (w > 0) & (h > 0) & (x0 < out_w) & (x0 + w > 0) & (r1 > r0)
    per = np.where(visible, (r1 - r0 + rows - 1) // rows, 0)
    tile = np.repeat(np.arange(len(descs)), per)
    k = np.arange(int(per.sum())) - np.repeat(np.concatenate([[0], np.cumsum(per)[:-1]]), per)
    first = np.repeat(r0, per) + k * np.repeat(rows, per)
    per_pixel = descs["res1_index"] >= 0
    if prims is not None and len(prims):
        off = np.clip(descs["prim_offset"], 0, len(prims) - 1)
        per_pixel = per_pixel | (descs["prim_count"] != 1) | (prims["kind"][off] != 0)
    n_rows = np.minimum(first + np.repeat(rows, per), np.repeat(r1, per)) - first
    cost = n_rows * np.repeat(w, per) * np.where(np.repeat(per_pixel, per), ITEM_PIXEL_WORK, 1)
    order = np.argsort(-cost, kind="stable")
    return np.stack([tile[order], first[order]], axis=1).astype(np.int32)


def pack_records(stacks) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """Pack per-tile primitive lists.

    Returns (prims, offsets[n+1], cp48 table (m, 48), counts).  A kind-5
    (bicubic) primitive carries its 48 control values in the cp48 table and
    the table index in ``geom[0]``.
    """
    n_tot = sum(len(s) for s in stacks)
    prims = np.zeros(max(1, n_tot), PRIM_DTYPE)
    counts = np.array([len(s) for s in stacks], np.int64)
    offsets = np.zeros(len(stacks) + 1, np.int64)
    np.cumsum(counts, out=offsets[1:])
    cps = []
    k = 0
    for s in stacks:
        for p in s:
            rec = prims[k]
            rec["kind"] = p.kind
            if p.kind == 5:
                rec["geom"][0] = float(len(cps))
                cps.append(np.asarray(p.geom, np.float32).reshape(48))
            else:
                g = tuple(p.geom)[:7]
                rec["geom"][: len(g)] = g
            rec["color0"] = p.color0
            if p.color1 is not None:
                rec["color1"] = p.color1
            rec["alpha"] = p.alpha
            k += 1
    cp48 = np.stack(cps).astype(np.float32) if cps else np.zeros((0, 48), np.float32)
    return prims, offsets, cp48, counts


def res0_float(residual_rgb) -> tuple[float, float, float]:
    """RES0 int8 bias -> float32 ``r / 255`` as the reference adds it (src/weft/render.py:231-232)."""
    r = np.asarray(residual_rgb, np.float32) / np.float32(255.0)
    return float(r[0]), float(r[1]), float(r[2])


def tile_rect(qx: int, qy: int, size: int, sx: float, sy: float, scaled: bool) -> tuple[int, int, int, int]:
    """Target rect of a quad tile (src/weft/render.py:321-334)."""
    if not scaled:
        return qx, qy, size, size
    x0, y0 = int(round(qx * sx)), int(round(qy * sy))
    x1, y1 = int(round((qx + size) * sx)), int(round((qy + size) * sy))
    return x0, y0, max(1, x1 - x0), max(1, y1 - y0)


def _launch(descs, prims, cp48, res1, out_h, out_w) -> np.ndarray:
    lib = _lib.lib_for_device(0)
    descs = np.ascontiguousarray(descs, TILE_DECODE_DTYPE)
    prims = np.ascontiguousarray(prims, PRIM_DTYPE)
    cp48 = np.ascontiguousarray(cp48, np.float32)
    res1 = np.ascontiguousarray(res1, np.float32) if res1 is not None else np.zeros((0, 48), np.float32)
    out = np.empty((out_h, out_w, 3), np.float32)
    rc = lib.weftk_render_tiles_host(_lib.ptr(descs), len(descs), _lib.ptr(prims), len(prims), _lib.ptr(cp48),
                                     len(cp48), _lib.ptr(res1), len(res1), _lib.ptr(out), out_h, out_w, 0)
    _lib.check(rc, "weftk_render_tiles_host")
    return out


def build_scene(records, quad_tiles, width, height, residual_maps=None, target_width=None, target_height=None):
    """Descriptor arrays for a scene; returns (descs, prims, cp48, res1, out_h, out_w)."""
    tw = int(target_width) if target_width is not None else int(width)
    th = int(target_height) if target_height is not None else int(height)
    if tw <= 0 or th <= 0:
        raise ValueError("target dimensions must be > 0")
    sx, sy = tw / float(width), th / float(height)
    scaled = not (tw == width and th == height)
    prims, offsets, cp48, counts = pack_records([r.primitives for r in records])
    if counts.size and counts.max() > MAX_TILE_PRIMS:
        raise ValueError(f"a tile has more than {MAX_TILE_PRIMS} primitives")
    n = len(records)
    descs = np.zeros(n, TILE_DECODE_DTYPE)
    rects = np.array([tile_rect(q.x, q.y, q.size, sx, sy, scaled) for q in quad_tiles[:n]], np.int64).reshape(-1, 4)
    descs["prim_offset"] = offsets[:-1]
    descs["prim_count"] = counts
    descs["target_x0"], descs["target_y0"] = rects[:, 0], rects[:, 1]
    descs["target_w"], descs["target_h"] = rects[:, 2], rects[:, 3]
    descs["source_size"] = [q.size for q in quad_tiles[:n]]
    res0 = np.array([r.residual_rgb for r in records], np.float32).reshape(-1, 3) / np.float32(255.0)
    descs["res0_r"], descs["res0_g"], descs["res0_b"] = res0[:, 0], res0[:, 1], res0[:, 2]
    res1 = None
    if residual_maps is not None:
        m = min(len(residual_maps), n)
        res1 = np.stack([np.asarray(residual_maps[i], np.float32).reshape(48) for i in range(m)]) if m else None
        descs["res1_index"] = [i if i < m else -1 for i in range(n)]
    else:
        descs["res1_index"] = -1
    return descs, prims, cp48, res1, th, tw


def render_scene_adaptive(records, quad_tiles, width: int, height: int, residual_maps=None,
                          res1_grid_size: int = 4, target_width: int | None = None,
                          target_height: int | None = None) -> np.ndarray:
    """GPU render of a quadtree scene; returns (target_h, target_w, 3) float32 in [0, 1]."""
    if residual_maps is not None and res1_grid_size != 4:
        raise ValueError("only 4x4 RES1 grids are supported")
    descs, prims, cp48, res1, th, tw = build_scene(records, quad_tiles, width, height, residual_maps,
                                                   target_width, target_height)
    return _launch(descs, prims, cp48, res1, th, tw)


def render_scene_device(records, quad_tiles, width: int, height: int, residual_maps=None, device: int = 0):
    """``render_scene_adaptive`` at the encoded size into a float32 CUDA tensor (h, w, 3), for the
    raster branch that keeps working on the image on the device."""
    import torch

    descs, prims, cp48, res1, th, tw = build_scene(records, quad_tiles, width, height, residual_maps)
    dev = torch.device("cuda", device)
    out = torch.zeros((th, tw, 3), dtype=torch.float32, device=dev)
    if len(descs) == 0:
        return out
    items = decode_items(descs, th, tw, prims)
    t_d = torch.from_numpy(np.ascontiguousarray(descs, TILE_DECODE_DTYPE).view(np.uint8)).to(dev)
    t_i = torch.from_numpy(items).to(dev)
    t_p = torch.from_numpy(np.ascontiguousarray(prims, PRIM_DTYPE).view(np.uint8)).to(dev)
    t_c = torch.from_numpy(np.ascontiguousarray(cp48, np.float32)).to(dev) if len(cp48) else None
    n_res1 = 0 if res1 is None else len(res1)
    t_r = torch.from_numpy(np.ascontiguousarray(res1, np.float32)).to(dev) if n_res1 else None
    lib = _lib.lib_for_device(device)
    _lib.check(lib.weftk_render_tiles(_lib.ptr(t_d), len(descs), _lib.ptr(t_i), len(items), _lib.ptr(t_p),
                                      _lib.ptr(t_c), len(cp48), _lib.ptr(t_r), n_res1, _lib.ptr(out), th, tw, 0,
                                      torch.cuda.current_stream(dev).cuda_stream), "weftk_render_tiles")
    return out


def render_tile(prims, tile_size: int, residual_rgb=None, source_size: int | None = None) -> np.ndarray:
    """GPU render of one stack as a single tile (clipped, with optional RES0)."""
    ts = int(tile_size)
    src = int(source_size) if source_size is not None else ts
    p, offs, cp48, counts = pack_records([list(prims)])
    d = np.zeros(1, TILE_DECODE_DTYPE)
    d["prim_count"] = counts[0]
    d["target_w"] = d["target_h"] = ts
    d["source_size"] = src
    d["res1_index"] = -1
    if residual_rgb is not None:
        d["res0_r"], d["res0_g"], d["res0_b"] = res0_float(residual_rgb)
    return _launch(d, p, cp48, None, ts, ts)
