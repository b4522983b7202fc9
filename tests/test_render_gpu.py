"""GPU parity of the render and scoring kernels against the reference goldens and the oracle.

Tolerances (from the path's parity contract): render max-abs <= 1/255 on linear
float32 RGB; per-tile MSE within 1e-5 relative.  Triangle coverage reproduces the
reference's float32 inside test exactly, so in practice renders agree to a few ulp.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import quadtree as oq
from oracle import render as orender
from oracle.primitives import Prim, Record, prims_from_pack
from tests.test_oracle_golden import _pack, golden_src, render_cases

pytestmark = pytest.mark.gpu

RENDER_TOL = 1.0 / 255.0
MSE_RTOL = 1e-5


def _rand_prim(rng, kind, ts):
    f = lambda v: float(np.float32(v))  # noqa: E731
    lo, hi = -2.0, ts + 1.0
    g = {0: (), 1: tuple(f(v) for v in rng.uniform(lo, hi, 4)),
         2: tuple(f(v) for v in rng.uniform(lo, hi, 4)) + (f(rng.uniform(0, 4)),),
         3: tuple(f(v) for v in rng.uniform(lo, hi, 6)) + (f(rng.uniform(0, 4)),),
         4: tuple(f(v) for v in rng.uniform(lo, hi, 6))}[kind]
    c1 = tuple(f(v) for v in rng.uniform(0, 1, 3)) if kind == 1 else None
    return Prim(kind, g, tuple(f(v) for v in rng.uniform(0, 1, 3)), c1, f(rng.uniform(0.05, 1.0)))


def test_render_tile_matches_reference_goldens(golden):
    from weft_b200 import render

    g = golden("render_tiles.npz")
    worst = 0.0
    for i, prims, ts, src_size, res, want, _ in render_cases(g):
        got = render.render_tile(prims, ts, residual_rgb=res, source_size=src_size)
        err = float(np.max(np.abs(got - want)))
        worst = max(worst, err)
        assert err <= RENDER_TOL, f"case {i}: max abs {err}"
    assert worst < 1e-4  # well inside the contract: only rounding-level differences


def test_score_evals_mse_matches_reference_goldens(golden):
    from weft_b200 import gpu_render

    g = golden("render_tiles.npz")
    sel = [(i, prims, ts, want_mse) for i, prims, ts, src_size, res, _, want_mse in render_cases(g)
           if src_size == ts and res is None and not any(p.kind == 5 for p in prims)]
    assert len(sel) > 60
    for i, prims, ts, want in sel:
        got = gpu_render.gpu_batch_objectives(golden_src(i, ts), [prims])[0]
        assert got == pytest.approx(want, rel=MSE_RTOL), f"case {i}"


def test_prepacked_scoring_many_tiles_random_stacks():
    from weft_b200 import gpu_render

    rng = np.random.default_rng(3)
    sizes = [8, 16, 32, 64, 8, 16, 32]
    tiles = [rng.random((s, s, 3), dtype=np.float32) for s in sizes]
    flat = np.concatenate([t.reshape(-1) for t in tiles])
    offs = dict(enumerate(np.concatenate([[0], np.cumsum([t.size for t in tiles])[:-1]]).tolist()))
    arrays, counts, stacks = [], [], []
    for j, s in enumerate(sizes):
        st = [[_rand_prim(rng, int(k), s) for k in rng.integers(0, 5, int(rng.integers(0, 9)))] for _ in range(11)]
        stacks.append(st)
        counts.append(np.array([len(x) for x in st], np.int32))
        arrays.append(np.concatenate([gpu_render._pack_prims(x)[:len(x)] for x in st]) if sum(counts[-1]) else
                      np.zeros(0, gpu_render._PRIM_DTYPE))
    out = gpu_render.gpu_batch_score_prepacked(flat, offs, list(range(len(sizes))), sizes, arrays, counts)
    for j, s in enumerate(sizes):
        want = [float(np.mean((tiles[j] - orender.render_tile(x, s)) ** 2)) for x in stacks[j]]
        np.testing.assert_allclose(out[j], want, rtol=MSE_RTOL, atol=1e-9)


def test_corner_sampling_reproduces_reference_gpu_convention():
    """sample_corner=True samples at integer pixel positions like the reference GPU scorer."""
    from weft_b200 import gpu_render

    rng = np.random.default_rng(8)
    ts = 16
    tile = rng.random((ts, ts, 3), dtype=np.float32)
    stacks = [[_rand_prim(rng, int(k), ts) for k in rng.integers(0, 5, 3)] for _ in range(20)]
    got = gpu_render.gpu_batch_objectives(tile, stacks, sample_corner=True)
    base = np.arange(ts, dtype=np.float32)
    ys, xs = np.meshgrid(base, base, indexing="ij")
    orig = orender.sample_grid
    try:
        orender.sample_grid = lambda n, s=None: (xs, ys)
        want = [float(np.mean((tile - orender.render_tile(s, ts)) ** 2)) for s in stacks]
    finally:
        orender.sample_grid = orig
    np.testing.assert_allclose(got, want, rtol=MSE_RTOL)


def test_render_scene_matches_reference_goldens(golden):
    from weft_b200 import render

    g = golden("render_scene.npz")
    for name in ("a", "b"):
        w, h = (int(v) for v in g[f"{name}_dims"])
        qts = [oq.QTile(int(x), int(y), int(s)) for x, y, s in g[f"{name}_qt"]]
        pk = _pack(g, f"{name}_p_")
        recs = [Record(prims_from_pack(pk, int(pk["offsets"][i]), int(pk["offsets"][i + 1])),
                       tuple(int(v) for v in g[f"{name}_residual"][i])) for i in range(len(qts))]
        res1 = list(g[f"{name}_res1"])
        off = 0
        for tw, th, use_res1 in g[f"{name}_targets"]:
            img = render.render_scene_adaptive(recs, qts, w, h, res1 if use_res1 else None, 4, int(tw), int(th))
            want = g[f"{name}_images"][off:off + img.size].reshape(img.shape)
            off += img.size
            err = float(np.max(np.abs(img - want)))
            assert err <= RENDER_TOL, f"{name} {tw}x{th}: {err}"


def test_render_scene_random_against_oracle_at_scale():
    from weft_b200 import render
    from weft_b200.synth import make_image_linear

    rng = np.random.default_rng(21)
    img = make_image_linear(128, 96, 20, 2)
    qts = oq.decompose(img, 0.08, 8, 32)
    recs = [Record([_rand_prim(rng, int(k), q.size) for k in rng.integers(0, 5, int(rng.integers(0, 6)))],
                   tuple(int(v) for v in rng.integers(-20, 21, 3))) for q in qts]
    maps = [rng.integers(-60, 61, (4, 4, 3)).astype(np.float32) / 255.0 for _ in qts]
    for tw, th in ((128, 96), (256, 192), (64, 48), (320, 240)):
        got = render.render_scene_adaptive(recs, qts, 128, 96, maps, 4, tw, th)
        want = orender.render_scene_adaptive(recs, qts, 128, 96, maps, 4, tw, th)
        assert float(np.max(np.abs(got - want))) <= RENDER_TOL


def test_drop_in_render_tiles_to_image():
    from weft_b200 import gpu_render

    rng = np.random.default_rng(5)
    descs = np.zeros(4, gpu_render._TILE_DECODE_DTYPE)
    stacks = [[_rand_prim(rng, int(k), 16) for k in rng.integers(0, 5, 3)] for _ in range(4)]
    prims = np.concatenate([gpu_render._pack_prims(s) for s in stacks])
    for i in range(4):
        descs[i] = (3 * i, 3, (i % 2) * 16, (i // 2) * 16, 16, 16, 16, 0, 0.0, 0.0, 0.0, 0.0)
    out = gpu_render.gpu_render_tiles_to_image(descs, prims, 32, 32)
    for i in range(4):
        want = orender.render_tile(stacks[i], 16)
        got = out[(i // 2) * 16:(i // 2) * 16 + 16, (i % 2) * 16:(i % 2) * 16 + 16]
        assert float(np.max(np.abs(got - want))) <= RENDER_TOL


def test_bad_descriptor_raises_not_falls_back():
    from weft_b200 import gpu_render
    from weft_b200._lib import WeftkError

    descs = np.zeros(1, gpu_render._TILE_DECODE_DTYPE)
    descs[0] = (0, 99, 0, 0, 16, 16, 16, 0, 0, 0, 0, 0)  # 99 primitives > 48
    with pytest.raises(WeftkError):
        gpu_render.gpu_render_tiles_to_image(descs, np.zeros(99, gpu_render._PRIM_DTYPE), 16, 16)
