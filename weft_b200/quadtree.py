"""Quadtree tiling of the image for the fit (host side).

Two split rules:

* ``"gradvar"`` — the reference rule: split while
  ``mean|grad lum| + 4 var(lum) >= threshold`` on linear luminance
  (src/weft/quadtree.py:33-91); thresholds 0.12 / 0.08 / 0.03 by quality band
  (src/weft/encoder.py:2536);
* ``"variance"`` — split while the variance of sRGB-u8 luminance
  (0.2126 R + 0.7152 G + 0.0722 B on 0..255 values) exceeds ``threshold``
  (u8^2 units; the 8-64 px batched workload uses 100).

Tiles come out in the reference order: macro tiles row-major, each split
recursively in TL, TR, BL, BR order.  The image is edge-padded to a multiple
of the macro tile.  ``pack_qtree`` writes the QTRE payload
(``<u32 count>`` then ``<u16 x, u16 y, u8 size>`` per tile, src/weft/quadtree.py:111-119).
"""

from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np

MAX_PRIMS_BY_SIZE = {8: 24, 16: 48, 32: 96}


@dataclass(slots=True)
class QuadTile:
    x: int
    y: int
    size: int
    index: int = 0

    @property
    def max_primitives(self) -> int:
        return MAX_PRIMS_BY_SIZE.get(self.size, 48)


def split_threshold_for(quality: int) -> float:
    """Reference split threshold by quality band (src/weft/encoder.py:2536)."""
    return 0.12 if quality < 70 else 0.08 if quality < 90 else 0.03


def pad_image(image: np.ndarray, mult: int) -> np.ndarray:
    h, w = image.shape[:2]
    ph, pw = (mult - h % mult) % mult, (mult - w % mult) % mult
    if ph or pw:
        image = np.pad(image, ((0, ph), (0, pw), (0, 0)), mode="edge")
    return image


def _gradvar(patch: np.ndarray) -> float:
    lum = 0.2126 * patch[..., 0] + 0.7152 * patch[..., 1] + 0.0722 * patch[..., 2]
    gy, gx = np.gradient(lum)
    return float(np.mean(np.sqrt(gx * gx + gy * gy))) + float(np.var(lum)) * 4.0


def decompose(image: np.ndarray, *, rule: str = "gradvar", threshold: float = 0.08, min_tile: int = 8,
              max_tile: int = 32, image_u8: np.ndarray | None = None) -> list[QuadTile]:
    """Split ``image`` (linear float32 HWC) into quad tiles.

    ``rule="variance"`` measures on ``image_u8`` (sRGB u8, same shape).
    """
    if rule == "variance":
        if image_u8 is None:
            raise ValueError("the variance rule needs the sRGB u8 image")
        src = pad_image(np.asarray(image_u8), max_tile).astype(np.float64)
        lum = 0.2126 * src[..., 0] + 0.7152 * src[..., 1] + 0.0722 * src[..., 2]

        def should_split(x, y, s):
            return float(np.var(lum[y:y + s, x:x + s])) > threshold
    elif rule == "gradvar":
        img = pad_image(image, max_tile)

        def should_split(x, y, s):
            return _gradvar(img[y:y + s, x:x + s]) >= threshold
    else:
        raise ValueError(f"unknown split rule {rule!r}")
    h, w = image.shape[:2]
    ph, pw = h + (max_tile - h % max_tile) % max_tile, w + (max_tile - w % max_tile) % max_tile
    tiles: list[QuadTile] = []

    def visit(x, y, s):
        if s > min_tile and should_split(x, y, s):
            hs = s // 2
            visit(x, y, hs)
            visit(x + hs, y, hs)
            visit(x, y + hs, hs)
            visit(x + hs, y + hs, hs)
        else:
            tiles.append(QuadTile(x, y, s, len(tiles)))

    for my in range(0, ph, max_tile):
        for mx in range(0, pw, max_tile):
            visit(mx, my, max_tile)
    return tiles


def extract_tiles(image: np.ndarray, tiles, pad_mult: int = 32) -> list[np.ndarray]:
    """Per-tile pixel patches from the edge-padded image (src/weft/quadtree.py:94-108)."""
    mult = max(pad_mult, max((t.size for t in tiles), default=pad_mult))
    img = pad_image(image, mult)
    return [img[t.y:t.y + t.size, t.x:t.x + t.size].copy() for t in tiles]


def pack_qtree(tiles) -> bytes:
    return struct.pack("<I", len(tiles)) + b"".join(struct.pack("<HHB", t.x, t.y, t.size) for t in tiles)


def unpack_qtree(blob: bytes) -> list[QuadTile]:
    if len(blob) < 4:
        raise ValueError("truncated QTREE")
    n = struct.unpack_from("<I", blob, 0)[0]
    if len(blob) < 4 + 5 * n:
        raise ValueError("truncated QTREE entries")
    return [QuadTile(*struct.unpack_from("<HHB", blob, 4 + 5 * i), index=i) for i in range(n)]
