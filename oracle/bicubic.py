"""Per-tile bicubic fit and the bicubic R-D swap of the adaptive fit (test oracle).

Restates ``bicubic.fit_tile`` / ``_bernstein4_pinvs`` (src/weft/bicubic.py:45-86) and the
swap loop at the end of ``_fit_adaptive_state`` (src/weft/encoder.py:2841-2873): every
tile's least-squares 4x4 Bezier control grid, rounded to u8 steps, evaluated, scored as
``mse + lambda * 408`` against the selected stack's ``mse + lambda * bits``; the tile is
replaced by the bicubic primitive when that score is lower.
"""

from __future__ import annotations

import numpy as np

from . import rate, render

BICUBIC_BITS = 51 * 8  # prim count + kind + length bytes + 48 control bytes (src/weft/encoder.py:2844-2846)


def pinvs(n: int) -> tuple[np.ndarray, np.ndarray]:
    """(pinv(B), pinv(B.T)) of the n-point Bernstein basis, float64 (src/weft/bicubic.py:45-57)."""
    B = render.bernstein_basis(n)
    return np.linalg.pinv(B), np.linalg.pinv(B.T)


def fit_tile(tile: np.ndarray) -> np.ndarray:
    """Least-squares control grid (4, 4, 3) float32 clipped to [0, 1] of a square tile
    (src/weft/bicubic.py:65-86)."""
    n = tile.shape[0]
    a, c = pinvs(n)
    P = np.empty((4, 4, 3), dtype=np.float32)
    for ch in range(3):
        P[:, :, ch] = (a @ tile[:, :, ch].astype(np.float64) @ c).astype(np.float32)
    return np.clip(P, 0.0, 1.0)


def quantize_grid(cp: np.ndarray) -> np.ndarray:
    """Round to u8 steps as the swap does before scoring (src/weft/encoder.py:2851-2853)."""
    return np.round(np.clip(cp, 0.0, 1.0) * 255.0) / 255.0


def tile_swap(patch: np.ndarray, prims, lam: float) -> tuple[bool, np.ndarray, float, float]:
    """One tile of the swap loop (src/weft/encoder.py:2847-2873): (replace?, quantized grid,
    bicubic score, stack score)."""
    n = patch.shape[0]
    cp_q = quantize_grid(fit_tile(patch))
    bic_mse = float(np.mean((patch - render.bicubic_tile(cp_q, n)) ** 2))
    prim_mse = float(np.mean((patch - render.render_tile(prims, n)) ** 2))
    prim_bits = 8 + sum(rate.PRIM_BYTES.get(p.kind, 20) for p in prims) * 8
    bic_score = bic_mse + lam * BICUBIC_BITS
    prim_score = prim_mse + lam * prim_bits
    return bic_score < prim_score, cp_q, bic_score, prim_score


def swap(patches, stacks, lam: float):
    """The swap over every tile: (replaced flags, quantized grids (n, 48), bicubic scores,
    stack scores)."""
    flags, grids, bs, ps = [], [], [], []
    for patch, prims in zip(patches, stacks):
        f, g, b, p = tile_swap(patch, prims, lam)
        flags.append(f)
        grids.append(g.reshape(-1))
        bs.append(b)
        ps.append(p)
    return np.array(flags, bool), np.array(grids, np.float32).reshape(-1, 48), np.array(bs), np.array(ps)
