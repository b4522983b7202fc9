"""Adaptive quadtree decomposition (test oracle).

Restates ``src/weft/quadtree.py``: the complexity metric
``mean|grad lum| + 4 var(lum)`` (:33-39), the recursive split of edge-padded
macro tiles (:42-91), tile extraction (:94-108) and the QTREE payload
``<u32 count>`` + ``<u16 x, u16 y, u8 size>`` per tile (:111-136).
"""

from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np


@dataclass
class QTile:
    x: int
    y: int
    size: int
    index: int = 0


def complexity(patch: np.ndarray) -> float:
    lum = 0.2126 * patch[..., 0] + 0.7152 * patch[..., 1] + 0.0722 * patch[..., 2]
    gy, gx = np.gradient(lum)
    return float(np.mean(np.sqrt(gx * gx + gy * gy))) + float(np.var(lum)) * 4.0


def pad_to(image: np.ndarray, mult: int) -> np.ndarray:
    h, w = image.shape[:2]
    ph, pw = (mult - h % mult) % mult, (mult - w % mult) % mult
    if ph or pw:
        image = np.pad(image, ((0, ph), (0, pw), (0, 0)), mode="edge")
    return image


def decompose(image: np.ndarray, split_threshold: float = 0.08, min_tile: int = 8, max_tile: int = 32) -> list[QTile]:
    img = pad_to(image, max_tile)
    ph, pw = img.shape[:2]
    tiles: list[QTile] = []

    def split(x, y, s):
        if s <= min_tile or complexity(img[y:y + s, x:x + s]) < split_threshold:
            tiles.append(QTile(x, y, s))
            return
        h = s // 2
        for dx, dy in ((0, 0), (h, 0), (0, h), (h, h)):
            split(x + dx, y + dy, h)

    for my in range(0, ph, max_tile):
        for mx in range(0, pw, max_tile):
            split(mx, my, max_tile)
    for i, t in enumerate(tiles):
        t.index = i
    return tiles


def extract(image: np.ndarray, tiles, pad_mult: int = 32) -> list[np.ndarray]:
    img = pad_to(image, pad_mult)
    return [img[t.y:t.y + t.size, t.x:t.x + t.size].copy() for t in tiles]


def pack_qtree(tiles) -> bytes:
    return struct.pack("<I", len(tiles)) + b"".join(struct.pack("<HHB", t.x, t.y, t.size) for t in tiles)


def unpack_qtree(blob: bytes) -> list[QTile]:
    n = struct.unpack_from("<I", blob, 0)[0]
    return [QTile(*struct.unpack_from("<HHB", blob, 4 + 5 * i), index=i) for i in range(n)]
