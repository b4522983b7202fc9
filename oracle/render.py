"""Numpy restatement of the reference's CPU primitive renderer (test oracle).

Follows ``src/weft/render.py`` and ``src/weft/bicubic.py`` of the reference.
The dtype semantics matter for parity and are kept: sample grids and the
frame buffer are float32; per-primitive scalars computed from the (float64)
primitive fields enter the float32 array arithmetic as weak Python floats,
exactly as numpy >= 2 evaluates the reference code.

Primitives are duck-typed: any object with ``kind``, ``geom``, ``color0``,
``color1`` and ``alpha`` attributes (``oracle.primitives.Prim`` here).
"""

from __future__ import annotations

import numpy as np


def sample_grid(out_size: int, source_size: int | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Pixel-centre sample positions (xs, ys), float32.

    Native: (i + 0.5).  Scaled: (i + 0.5) * (source/out) with the step in
    float64 rounded to float32 by the array multiply.
    Reference: ``_grid`` / ``_scaled_grid`` (src/weft/render.py:29-78).
    """
    if source_size is None or source_size == out_size:
        base = np.arange(out_size, dtype=np.float32) + 0.5
    else:
        step = float(source_size) / float(out_size)
        base = (np.arange(out_size, dtype=np.float32) + 0.5) * step
    ys, xs = np.meshgrid(base, base, indexing="ij")
    return xs, ys


def segment_distance(px, py, x0, y0, x1, y1):
    """Distance from sample points to segment p0-p1 (src/weft/render.py:85-95)."""
    vx = x1 - x0
    vy = y1 - y0
    den = vx * vx + vy * vy + 1e-8
    t = np.clip(((px - x0) * vx + (py - y0) * vy) / den, 0.0, 1.0)
    dx = px - (x0 + t * vx)
    dy = py - (y0 + t * vy)
    return np.sqrt(dx * dx + dy * dy)


def bezier_polyline(g) -> list[tuple[np.float32, np.float32]]:
    """32 float32 points of the quadratic Bezier at linspace(0, 1, 32).

    Reference: ``_eval_curve_distance`` (src/weft/render.py:98-105).
    """
    pts = []
    for t in np.linspace(0.0, 1.0, 32, dtype=np.float32):
        u = np.float32(1.0) - t
        x = u * u * g[0] + 2.0 * u * t * g[2] + t * t * g[4]
        y = u * u * g[1] + 2.0 * u * t * g[3] + t * t * g[5]
        pts.append((x, y))
    return pts


def curve_distance(px, py, g):
    """Min distance to the 31-segment polyline (src/weft/render.py:98-111)."""
    pts = bezier_polyline(g)
    best = np.full_like(px, 1e9, dtype=np.float32)
    for (ax, ay), (bx, by) in zip(pts[:-1], pts[1:]):
        best = np.minimum(best, segment_distance(px, py, ax, ay, bx, by))
    return best


def triangle_mask(px, py, g):
    """Barycentric inside test, 0 for |den| < 1e-6 (src/weft/render.py:114-124)."""
    x0, y0, x1, y1, x2, y2 = g
    den = (y1 - y2) * (x0 - x2) + (x2 - x1) * (y0 - y2)
    if abs(den) < 1e-6:
        return np.zeros_like(px, dtype=np.float32)
    a = ((y1 - y2) * (px - x2) + (x2 - x1) * (py - y2)) / den
    b = ((y2 - y0) * (px - x2) + (x0 - x2) * (py - y2)) / den
    c = 1.0 - a - b
    return ((a >= 0.0) & (b >= 0.0) & (c >= 0.0)).astype(np.float32)


def bernstein_basis(n: int) -> np.ndarray:
    """Cubic Bernstein basis at n points of linspace(0, 1, n), float64 (src/weft/bicubic.py:31-43)."""
    t = np.linspace(0.0, 1.0, n, dtype=np.float64)
    return np.stack([(1.0 - t) ** 3, 3.0 * (1.0 - t) ** 2 * t, 3.0 * (1.0 - t) * t ** 2, t ** 3], axis=-1)


def bicubic_tile(cp: np.ndarray, size: int) -> np.ndarray:
    """Evaluate a (4, 4, 3) control grid on size x size (src/weft/bicubic.py:106-115)."""
    B = bernstein_basis(size)
    out = np.empty((size, size, 3), dtype=np.float32)
    for ch in range(3):
        out[:, :, ch] = (B @ cp[:, :, ch].astype(np.float64) @ B.T).astype(np.float32)
    return np.clip(out, 0.0, 1.0)


def _add_residual(tile: np.ndarray, residual_rgb) -> np.ndarray:
    if residual_rgb is not None:
        tile = tile + np.array(residual_rgb, dtype=np.float32)[None, None, :] / 255.0
    return tile


def render_tile(prims, tile_size: int, residual_rgb=None, source_size: int | None = None) -> np.ndarray:
    """Back-to-front 'over' composite of a primitive stack, clipped to [0, 1].

    Reference: ``render_tile`` (src/weft/render.py:127-234), including the
    sole-bicubic path (:166-172), the all-constant path (:175-182) and the
    rule that kind 5 inside a longer stack is skipped (:225-226).
    """
    xs, ys = sample_grid(tile_size, source_size)
    tile = np.zeros((tile_size, tile_size, 3), dtype=np.float32)
    prims = list(prims)
    if not prims:
        return np.clip(_add_residual(tile, residual_rgb), 0.0, 1.0)

    if len(prims) == 1 and prims[0].kind == 5:
        cp = np.asarray(prims[0].geom, dtype=np.float32).reshape(4, 4, 3)
        return np.clip(_add_residual(bicubic_tile(cp, tile_size), residual_rgb), 0.0, 1.0)

    if all(p.kind == 0 for p in prims):
        for p in prims:
            a = max(0.0, min(1.0, p.alpha))
            tile = np.array(p.color0, dtype=np.float32)[None, None, :] * a + tile * (1.0 - a)
        return np.clip(_add_residual(tile, residual_rgb), 0.0, 1.0)

    for p in prims:
        a = np.float32(max(0.0, min(1.0, p.alpha)))
        r0, g0, b0 = p.color0
        k = p.kind
        if k == 0:
            for ch, cval in enumerate((r0, g0, b0)):
                tile[:, :, ch] = cval * a + tile[:, :, ch] * (1.0 - a)
            continue
        if k == 1:
            x0, y0, x1, y1 = p.geom
            vx, vy = x1 - x0, y1 - y0
            den = vx * vx + vy * vy + 1e-8
            t = np.clip(((xs - x0) * vx + (ys - y0) * vy) / den, 0.0, 1.0)[..., None]
            c0 = np.array(p.color0, dtype=np.float32)
            c1 = np.array(p.color1 if p.color1 is not None else p.color0, dtype=np.float32)
            src = c0 * (1.0 - t) + c1 * t
            alpha = np.full((tile_size, tile_size), a, dtype=np.float32)
        elif k in (2, 3, 4):
            if k == 2:
                x0, y0, x1, y1, thick = p.geom
                dist = segment_distance(xs, ys, x0, y0, x1, y1)
            elif k == 3:
                thick = p.geom[6]
                dist = curve_distance(xs, ys, p.geom)
            if k == 4:
                alpha = triangle_mask(xs, ys, p.geom) * a
            else:
                sigma = max(0.5, float(thick))
                inv = 1.0 / (2.0 * sigma * sigma)
                alpha = np.exp(-(dist * dist) * inv, dtype=np.float32) * a
            src = np.empty_like(tile)
            src[:, :, 0] = r0
            src[:, :, 1] = g0
            src[:, :, 2] = b0
        else:
            continue
        a3 = alpha[..., None]
        tile = src * a3 + tile * (1.0 - a3)

    return np.clip(_add_residual(tile, residual_rgb), 0.0, 1.0)


def upsample_residual_map(residual_map: np.ndarray, tile_size: int, grid_size: int = 4) -> np.ndarray:
    """Bilinear RES1 grid -> tile, sampled at pixel centres, edge-clamped.

    Reference: ``upsample_residual_map`` (src/weft/render.py:474-515).
    """
    if residual_map.shape != (grid_size, grid_size, 3):
        raise ValueError("invalid residual map shape")
    centres = np.arange(tile_size, dtype=np.float32) + 0.5
    g = np.clip(centres * (float(grid_size) / float(tile_size)) - 0.5, 0.0, grid_size - 1)
    i0 = np.floor(g).astype(np.int32)
    f = g - i0
    i1 = np.clip(i0 + 1, 0, grid_size - 1)
    c00 = residual_map[i0[:, None], i0[None, :]]
    c01 = residual_map[i0[:, None], i1[None, :]]
    c10 = residual_map[i1[:, None], i0[None, :]]
    c11 = residual_map[i1[:, None], i1[None, :]]
    wx = f[None, :, None]
    wy = f[:, None, None]
    top = c00 * (1.0 - wx) + c01 * wx
    bot = c10 * (1.0 - wx) + c11 * wx
    return top * (1.0 - wy) + bot * wy


def scene_tile_rect(qx: int, qy: int, qsize: int, sx: float, sy: float) -> tuple[int, int, int, int]:
    """Target rect (x0, y0, w, h) of a quad tile under scale (sx, sy).

    Python round() (half to even) on the scaled edges, width/height >= 1.
    Reference: src/weft/render.py:329-334.
    """
    tx0 = int(round(qx * sx))
    ty0 = int(round(qy * sy))
    tx1 = int(round((qx + qsize) * sx))
    ty1 = int(round((qy + qsize) * sy))
    return tx0, ty0, max(1, tx1 - tx0), max(1, ty1 - ty0)


def render_scene_adaptive(records, quad_tiles, width: int, height: int, residual_maps=None,
                          res1_grid_size: int = 4, target_width: int | None = None,
                          target_height: int | None = None) -> np.ndarray:
    """Decoder primitive walk over quadtree tiles (src/weft/render.py:270-358).

    ``records`` have ``.primitives`` and ``.residual_rgb``; ``quad_tiles``
    have ``.x``, ``.y``, ``.size``.  Scaled targets render a square
    max(w, h) tile with the source coordinate space and crop.
    """
    tw = int(target_width) if target_width is not None else width
    th = int(target_height) if target_height is not None else height
    if tw <= 0 or th <= 0:
        raise ValueError("target dimensions must be > 0")
    sx, sy = tw / float(width), th / float(height)
    scaled = not (tw == width and th == height)
    out = np.zeros((th + (32 - th % 32) % 32, tw + (32 - tw % 32) % 32, 3), dtype=np.float32)
    for i, (rec, qt) in enumerate(zip(records, quad_tiles)):
        if not scaled:
            img = render_tile(rec.primitives, qt.size, residual_rgb=rec.residual_rgb)
            x0, y0 = qt.x, qt.y
        else:
            x0, y0, w, h = scene_tile_rect(qt.x, qt.y, qt.size, sx, sy)
            side = max(w, h)
            img = render_tile(rec.primitives, side, residual_rgb=rec.residual_rgb, source_size=qt.size)
            if (w, h) != (side, side):
                img = img[:h, :w, :]
        if residual_maps is not None and i < len(residual_maps):
            img = np.clip(img + upsample_residual_map(residual_maps[i], img.shape[0], res1_grid_size), 0.0, 1.0)
        out[y0:y0 + img.shape[0], x0:x0 + img.shape[1], :] = img
    return np.clip(out[:th, :tw, :], 0.0, 1.0)
