"""Rate model and per-tile objective (test oracle).

Restates ``_tile_lambda`` (src/weft/encoder.py:167-174), the byte-size table
``_PRIM_BYTE_SIZES`` / ``_PRIM_BYTE_SIZES_LUT`` (:242-256), ``_estimate_bits``
(:259-268), ``_tile_objective`` (:271-285) and ``_quantize_residual_map``
(:288-301), plus the RD score of the auto-select tournament
(src/weft/encoder.py:3926-3931, :4008-4011) and ``psnr`` (src/weft/metrics.py:15-19).
"""

from __future__ import annotations

import math

import numpy as np

from . import render

PRIM_BYTES = {0: 7, 1: 18, 2: 17, 3: 21, 4: 19}
LUT = np.array([PRIM_BYTES.get(k, 20) for k in range(16)], dtype=np.int32)


def tile_lambda(quality: int) -> float:
    q = max(0, min(100, int(quality)))
    base = ((101 - q) / 100.0) ** 2
    return base * (0.0002 if q >= 90 else 0.001)


def estimate_bits(prims, include_residual: bool, include_res1: bool = False, res1_grid_size: int = 4) -> int:
    bits = 8 + sum(PRIM_BYTES.get(p.kind, 20) * 8 for p in prims)
    if include_residual:
        bits += 24
    if include_res1:
        bits += res1_grid_size * res1_grid_size * 24
    return bits


def tile_objective(src, prims, residual, lam, residual_map=None, res1_grid_size: int = 4):
    pred = render.render_tile(prims, src.shape[0], residual_rgb=residual)
    if residual_map is not None:
        pred = np.clip(pred + render.upsample_residual_map(residual_map, src.shape[0], res1_grid_size), 0.0, 1.0)
    dist = float(np.mean((src - pred) ** 2))
    rate = estimate_bits(prims, tuple(residual) != (0, 0, 0), residual_map is not None, res1_grid_size)
    return dist + lam * rate, pred


def quantize_residual_map(error: np.ndarray, grid_size: int = 4) -> np.ndarray:
    h, w, _ = error.shape
    sh, sw = h // grid_size, w // grid_size
    out = np.empty((grid_size, grid_size, 3), dtype=np.float32)
    for gy in range(grid_size):
        for gx in range(grid_size):
            out[gy, gx] = error[gy * sh:(gy + 1) * sh, gx * sw:(gx + 1) * sw].mean(axis=(0, 1))
    q = np.clip(np.round(out * 255.0), -127.0, 127.0).astype(np.int8)
    return q.astype(np.float32) / 255.0


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    d = np.asarray(a, dtype=np.float32) - np.asarray(b, dtype=np.float32)
    m = float(np.mean(d * d))
    return 100.0 if m <= 1e-12 else float(10.0 * math.log10(1.0 / m))


def rd_lambda(quality: int) -> float:
    """Auto-select RD lambda: 4 * ((100 - q) / 25)^2 above q = 75, else 4."""
    q = int(quality)
    return 4.0 * ((100 - q) / 25.0) ** 2 if q > 75 else 4.0


def rd_score(psnr_db: float, n_bytes: int, width: int, height: int, quality: int) -> float:
    return psnr_db - rd_lambda(quality) * (n_bytes * 8.0 / float(width * height))
