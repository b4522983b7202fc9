"""Host-side logic around the kernels (no GPU): decode work items and the refine op count."""

from __future__ import annotations

import os
import sys
import types

import numpy as np
import torch

from weft_b200 import render
from weft_b200._lib import TILE_DECODE_DTYPE


def test_decode_items_cover_every_chunk_once():
    rng = np.random.default_rng(3)
    n = 200
    d = np.zeros(n, TILE_DECODE_DTYPE)
    d["target_x0"] = rng.integers(-5, 3000, n)
    d["target_y0"] = rng.integers(0, 2000, n)
    d["target_w"] = rng.integers(1, 300, n)
    d["target_h"] = rng.integers(1, 300, n)
    items = render.decode_items(d)
    k = render.DECODE_ITEM_CHUNKS
    for t in range(n):
        x0, w, h = int(d["target_x0"][t]), int(d["target_w"][t]), int(d["target_h"][t])
        groups = ((x0 + w + 3) // 4 - x0 // 4) * h  # floor division, as the kernel
        chunks = -(-groups // render.DECODE_CHUNK_GROUPS)
        starts = sorted(int(c) for tt, c in items if tt == t)
        assert starts == list(range(0, chunks, k))


def test_refine_flop_count_follows_the_per_kind_table():
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    ss = types.SimpleNamespace(t_kind=torch.tensor([0, 1, 0, 4], dtype=torch.int32),
                               prim_off_np=np.array([0, 2, 2, 4]), sizes=torch.tensor([8, 16, 32]))
    per = {k: 2 * bench.REFINE_EVAL[k] + 9 + bench.REFINE_CHAIN[k] for k in (0, 1, 4)}
    want = 64 * (per[0] + per[1] + 9) + 256 * 9 + 1024 * (per[0] + per[4] + 9)
    assert bench.refine_flops(ss) == want


def test_kinds_mask():
    from weft_b200.refine import kinds_mask_of

    assert kinds_mask_of(np.array([0, 1, 1, 0], np.int8)) == 3
    assert kinds_mask_of(np.zeros(0, np.int32)) == 0
    assert kinds_mask_of(np.array([4, 2, -1, 7], np.int32)) == (1 << 4) | (1 << 2) | (1 << 7)
