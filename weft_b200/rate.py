"""Rate model and RD score used by the fit (host side).

* ``tile_lambda`` — rate weight of the per-tile objective (src/weft/encoder.py:167-174);
* ``PRIM_BYTES`` — serialized bytes per primitive kind (src/weft/encoder.py:242-256;
  bicubic and unknown kinds count 20);
* ``estimate_bits`` — src/weft/encoder.py:259-268;
* ``rd_score`` — the auto-select tournament score PSNR - lambda_rd * BPP
  (src/weft/encoder.py:3926-3931, :4008-4011) with PSNR over linear RGB capped at
  100 dB (src/weft/metrics.py:15-19).
"""

from __future__ import annotations

import math

import numpy as np

PRIM_BYTES = {0: 7, 1: 18, 2: 17, 3: 21, 4: 19}
BYTES_LUT = np.array([PRIM_BYTES.get(k, 20) for k in range(16)], dtype=np.int32)


def tile_lambda(quality: int) -> float:
    q = max(0, min(100, int(quality)))
    base = ((101 - q) / 100.0) ** 2
    return base * (0.0002 if q >= 90 else 0.001)


def complexity_threshold(quality: int) -> float:
    """Objective above which a tile keeps taking greedy rounds (src/weft/encoder.py:2738)."""
    return 0.00005 if quality >= 90 else 0.0005


def max_rounds(quality: int) -> int:
    """Greedy round budget (src/weft/encoder.py:2745)."""
    return 20 if quality >= 90 else 8 if quality >= 70 else 4


def estimate_bits(kinds, include_residual: bool = False, include_res1: bool = False, res1_grid: int = 4) -> int:
    bits = 8 + sum(8 * PRIM_BYTES.get(int(k), 20) for k in kinds)
    if include_residual:
        bits += 24
    if include_res1:
        bits += res1_grid * res1_grid * 24
    return bits


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    d = np.asarray(a, dtype=np.float32) - np.asarray(b, dtype=np.float32)
    m = float(np.mean(d * d))
    return 100.0 if m <= 1e-12 else float(10.0 * math.log10(1.0 / m))


def rd_lambda(quality: int) -> float:
    q = max(0, min(100, int(quality)))
    return 4.0 * ((100 - q) / 25.0) ** 2 if q > 75 else 4.0


def rd_score(psnr_db: float, n_bytes: int, width: int, height: int, quality: int) -> float:
    return psnr_db - rd_lambda(quality) * (n_bytes * 8.0 / float(width * height))
