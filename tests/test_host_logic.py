"""Host-side logic around the kernels (no GPU): decode work items and the refine op count."""

from __future__ import annotations

import os
import sys
import types

import numpy as np
import torch

from weft_b200 import render
from weft_b200._lib import TILE_DECODE_DTYPE


def test_decode_items_cover_every_visible_row_once():
    rng = np.random.default_rng(3)
    n = 200
    out_h, out_w = 1500, 2500
    d = np.zeros(n, TILE_DECODE_DTYPE)
    d["target_x0"] = rng.integers(-40, 3000, n)
    d["target_y0"] = rng.integers(-40, 2000, n)
    d["target_w"] = rng.integers(1, 300, n)
    d["target_h"] = rng.integers(1, 300, n)
    items = render.decode_items(d, out_h, out_w)
    for t in range(n):
        x0, y0, w, h = (int(d[k][t]) for k in ("target_x0", "target_y0", "target_w", "target_h"))
        groups = (x0 + w + 3) // 4 - x0 // 4  # floor division, as the kernel
        rows = max(1, render.DECODE_ITEM_GROUPS // groups)
        covered = []
        for tt, r in items:
            if tt == t:
                covered += range(int(r), min(int(r) + rows, h))
        visible = x0 < out_w and x0 + w > 0
        expect = [r for r in range(h) if 0 <= y0 + r < out_h] if visible else []
        assert sorted(c for c in covered if 0 <= y0 + c < out_h) == expect
        assert len(covered) == len(set(covered))
        assert all(0 <= c < h for c in covered)
    # descending cost: rows x width (every tile without a RES1 grid and prims counts as a fill)
    x = d["target_x0"].astype(np.int64)
    g = (x + d["target_w"] + 3) // 4 - x // 4
    rows = np.maximum(1, render.DECODE_ITEM_GROUPS // g)
    t_, r_ = items[:, 0], items[:, 1].astype(np.int64)
    n_rows = np.minimum(r_ + rows[t_], np.minimum(d["target_h"][t_], out_h - d["target_y0"][t_])) - r_
    cost = n_rows * d["target_w"][t_]
    assert np.all(np.diff(cost) <= 0)


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


def test_slot_layout_matches_the_scatter_formula():
    """Slots and kinds of the packed records, with and without reserved slots, against the direct
    formula (pool_off of the tile + index in its pool)."""
    from weft_b200._lib import PRIM_DTYPE
    from weft_b200.fit import slot_layout

    rng = np.random.default_rng(7)
    for reserve in (0, 3, 384):
        cnt = rng.integers(0, 9, 40).astype(np.int64)
        recs = np.zeros(int(cnt.sum()), PRIM_DTYPE)
        recs["kind"] = rng.integers(0, 9, len(recs))
        cap = cnt + reserve
        pool_off = np.concatenate([[0], np.cumsum(cap)[:-1]]).astype(np.int64)
        n_slots = int(cap.sum())
        kinds, slots = slot_layout(recs, cnt, pool_off, n_slots)
        want_slots = np.concatenate([pool_off[t] + np.arange(cnt[t]) for t in range(len(cnt))]).astype(np.int64)
        want_kinds = np.full(n_slots, 7, np.int8)
        want_kinds[want_slots] = np.where(recs["kind"] < 7, recs["kind"], 7)
        np.testing.assert_array_equal(kinds, want_kinds)
        if reserve == 0:
            assert slots is None and np.array_equal(want_slots, np.arange(len(recs)))
        else:
            np.testing.assert_array_equal(slots, want_slots)


def test_init_kinds_mask_matches_kinds_mask_of():
    from weft_b200.fit import BatchedFit
    from weft_b200.refine import kinds_mask_of

    rng = np.random.default_rng(3)
    cases = [rng.integers(0, 8, 5000).astype(np.int8), np.full(10, 7, np.int8), np.zeros(0, np.int8),
             np.array([0, 1, 1, 7, 7], np.int8), np.array([-3, 2, 7, 5], np.int8), np.array([4, 4, 6], np.int8)]
    for k in cases:
        f = BatchedFit.__new__(BatchedFit)
        f._init_kinds = k
        assert f.init_kinds_mask() == kinds_mask_of(f.init_kinds()), k


def test_tile_lambda_branches():
    """The reference's locked-down λ(q) properties (tests/test_rd_scoring.py): base (101 - q)^2 / 1e4
    times 0.0002 from q = 90, times 0.001 below; a cliff at 90 and monotone within each branch."""
    import pytest

    from weft_b200 import rate

    for q in (95, 90):
        assert rate.tile_lambda(q) == pytest.approx(((101 - q) / 100.0) ** 2 * 0.0002, rel=1e-9)
    for q in (89, 75, 50):
        assert rate.tile_lambda(q) == pytest.approx(((101 - q) / 100.0) ** 2 * 0.001, rel=1e-9)
    assert rate.tile_lambda(89) / rate.tile_lambda(90) > 2.0
    assert all(rate.tile_lambda(q) >= rate.tile_lambda(q + 1) for q in range(50, 89))
    assert all(rate.tile_lambda(q) >= rate.tile_lambda(q + 1) for q in range(90, 100))


def test_bicubic_basis_and_exact_fits():
    """The reference's bicubic properties (tests/test_bicubic.py) for the basis table the swap
    kernel reads and for the oracle fit it is checked against: every Bernstein row sums to 1, a
    constant tile and a linear gradient are fitted exactly."""
    from oracle import bicubic as obic
    from oracle import render as orender
    from weft_b200 import bicubic

    tab = bicubic.basis_table()
    for n in bicubic.SIDES:
        B = tab[12 * (n - 8) + 8 * n:12 * (n - 8) + 12 * n].reshape(n, 4)
        assert np.allclose(B.sum(axis=1), 1.0, atol=1e-10)
        assert np.array_equal(B, orender.bernstein_basis(n))
    tile = np.full((16, 16, 3), 0.4, dtype=np.float32)
    assert np.allclose(orender.bicubic_tile(obic.fit_tile(tile), 16), tile, atol=1e-5)
    yy, xx = np.mgrid[0:16, 0:16].astype(np.float32) / 15
    tile = np.stack([xx, yy, np.zeros_like(xx)], axis=-1)
    assert np.max(np.abs(orender.bicubic_tile(obic.fit_tile(tile), 16) - tile)) < 1e-4
