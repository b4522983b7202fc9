"""Seeded synthetic test images for the primitive-stack fit.

The generator is the canonical workload definition used by the bench and the
tests: a linear-gradient background plus N alpha-composited axis-aligned
rectangles and ellipses, then Gaussian noise (sigma = 2 in u8 units).  It is
deterministic for a given ``(width, height, n_prims, seed)``.

RNG draw order (``numpy.random.default_rng(seed)``):
  background colour A (3 uniforms in [0, 255)), colour B (3), angle (1 in
  [0, 2*pi)); then per primitive: centre x in [0, W), centre y in [0, H),
  shape switch (rect if < 0.5), full width in [4, 64], full height in [4, 64],
  colour (3 in [0, 255)), opacity in [0.5, 1.0); finally one (H, W, 3) normal
  draw for the noise.

Compositing is float64 in [0, 255] over covered pixel centres
``(x + 0.5, y + 0.5)``: ``dst = dst * (1 - a) + colour * a``.

The linear-light conversion mirrors the reference's image loader
(``src/weft/image_io.py:19-24``, sRGB u8 -> /255 -> piecewise sRGB EOTF, float32).
"""

from __future__ import annotations

import numpy as np


def make_image_u8(width: int, height: int, n_prims: int, seed: int) -> np.ndarray:
    """Return an (H, W, 3) uint8 sRGB image from the canonical generator."""
    rng = np.random.default_rng(seed)
    col_a = rng.uniform(0.0, 255.0, 3)
    col_b = rng.uniform(0.0, 255.0, 3)
    theta = rng.uniform(0.0, 2.0 * np.pi)

    ys = np.arange(height, dtype=np.float64) + 0.5
    xs = np.arange(width, dtype=np.float64) + 0.5
    yy, xx = np.meshgrid(ys, xs, indexing="ij")
    proj = xx * np.cos(theta) + yy * np.sin(theta)
    lo, hi = float(proj.min()), float(proj.max())
    t = (proj - lo) / max(hi - lo, 1e-12)
    canvas = col_a[None, None, :] * (1.0 - t[..., None]) + col_b[None, None, :] * t[..., None]

    for _ in range(n_prims):
        cx = rng.uniform(0.0, width)
        cy = rng.uniform(0.0, height)
        is_rect = rng.random() < 0.5
        w = rng.uniform(4.0, 64.0)
        h = rng.uniform(4.0, 64.0)
        col = rng.uniform(0.0, 255.0, 3)
        a = rng.uniform(0.5, 1.0)
        # Only touch the bounding box of the shape.
        x0 = max(0, int(np.floor(cx - w / 2.0)) - 1)
        x1 = min(width, int(np.ceil(cx + w / 2.0)) + 1)
        y0 = max(0, int(np.floor(cy - h / 2.0)) - 1)
        y1 = min(height, int(np.ceil(cy + h / 2.0)) + 1)
        if x1 <= x0 or y1 <= y0:
            continue
        px = xx[y0:y1, x0:x1]
        py = yy[y0:y1, x0:x1]
        if is_rect:
            mask = (np.abs(px - cx) <= w / 2.0) & (np.abs(py - cy) <= h / 2.0)
        else:
            mask = ((px - cx) / (w / 2.0)) ** 2 + ((py - cy) / (h / 2.0)) ** 2 <= 1.0
        region = canvas[y0:y1, x0:x1]
        region[mask] = region[mask] * (1.0 - a) + col[None, :] * a

    canvas = canvas + rng.normal(0.0, 2.0, canvas.shape)
    return np.clip(np.rint(canvas), 0.0, 255.0).astype(np.uint8)


def srgb_u8_to_linear(img_u8: np.ndarray) -> np.ndarray:
    """sRGB u8 -> linear float32 in [0, 1] (same arithmetic as the reference loader)."""
    x = np.asarray(img_u8, dtype=np.float32) / 255.0
    a = 0.055
    return np.where(x <= 0.04045, x / 12.92, ((x + a) / (1.0 + a)) ** 2.4).astype(np.float32)


def make_image_linear(width: int, height: int, n_prims: int, seed: int) -> np.ndarray:
    """Canonical synthetic image in linear RGB float32, shape (H, W, 3)."""
    return srgb_u8_to_linear(make_image_u8(width, height, n_prims, seed))


def multi_image_specs() -> list[tuple[int, int, int, int]]:
    """The 64-image mixed batch: (width, height, n_prims, seed) per image.

    16 images each of 256^2, 512^2, 1024^2 and 2048^2; seeds 0..63;
    n_prims = 50 + (2450 * i) // 63.
    """
    sizes = [256] * 16 + [512] * 16 + [1024] * 16 + [2048] * 16
    return [(s, s, 50 + (2450 * i) // 63, i) for i, s in enumerate(sizes)]
