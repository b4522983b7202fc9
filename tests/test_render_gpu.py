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


def _const_heavy_scene(rng, qts):
    """Mostly lone constant layers (the decoder's common tile), some longer stacks, RES0 offsets."""
    recs = []
    for q in qts:
        if rng.random() < 0.8:
            c = tuple(float(v) for v in rng.random(3).astype(np.float32))
            stack = [Prim(0, (), c, None, float(np.float32(0.3 + 0.7 * rng.random())))]
        else:
            stack = [_rand_prim(rng, int(k), q.size) for k in rng.integers(0, 5, int(rng.integers(1, 4)))]
        recs.append(Record(stack, tuple(int(v) for v in rng.integers(-20, 21, 3))))
    return recs


@pytest.mark.parametrize("with_res1", [False, True])
def test_walk_constant_fill_paths_against_oracle(with_res1):
    """The walk's whole-slot paths for lone constant tiles (with and without the RES1 grid) and the
    per-group path for the rest, at output widths of every residue mod 4 (the slot paths need rows
    on 16-byte boundaries, so widths not a multiple of 4 take the per-group path) and at scales that
    split 4-pixel groups between tiles."""
    from weft_b200 import render
    from weft_b200.synth import make_image_linear

    rng = np.random.default_rng(33)
    # images of every width mod 4 at their own size, and a square one at scaled targets: every
    # width mod 4 without grids; with grids only scales that keep every tile square (the reference
    # walk refuses a RES1 grid on a non-square rect, and cannot place the edge tiles of a source
    # whose sides are not multiples of 32 at a scaled target)
    scaled = ((256, 256), (64, 64)) if with_res1 else ((129, 129), (130, 130), (131, 131), (200, 200), (91, 91))
    for iw, ih, targets in ((130, 98, ((130, 98),)), (131, 99, ((131, 99),)), (129, 97, ((129, 97),)),
                            (128, 128, ((128, 128),) + scaled)):
        img = make_image_linear(iw, ih, 20, 4)
        qts = oq.decompose(img, 0.08, 8, 32)
        recs = _const_heavy_scene(rng, qts)
        maps = [rng.integers(-60, 61, (4, 4, 3)).astype(np.float32) / 255.0 for _ in qts] if with_res1 else None
        for tw, th in targets:
            got = render.render_scene_adaptive(recs, qts, iw, ih, maps, 4, tw, th)
            want = orender.render_scene_adaptive(recs, qts, iw, ih, maps, 4, tw, th)
            assert float(np.max(np.abs(got - want))) <= RENDER_TOL, (iw, ih, tw, th)


def test_walk_rects_partly_outside_the_image():
    """Lone constant rects (disjoint) that start left of / above the image or end past it, rects
    narrower than a 16-byte slot, and rects wholly outside: only in-image pixels are written, with
    the tile's colour (blend over black + RES0, clipped); the rest of the buffer is left as it was."""
    import torch

    from weft_b200 import _lib
    from weft_b200.gpu_render import _PRIM_DTYPE, _TILE_DECODE_DTYPE
    from weft_b200.render import decode_items

    rng = np.random.default_rng(8)
    H, W = 61, 100
    rects = [(-7, -3, 20, 11), (90, 50, 25, 20), (5, 20, 1, 9), (17, 33, 2, 2), (31, 2, 3, 30), (120, 5, 10, 10),
             (4, -40, 9, 20), (-13, 45, 130, 3), (40, 10, 37, 29), (80, 0, 5, 40)]
    n = len(rects)
    descs = np.zeros(n, _TILE_DECODE_DTYPE)
    prims = np.zeros(n, _PRIM_DTYPE)
    want = np.full((H, W, 3), -1.0, np.float32)
    for i, (x0, y0, w, h) in enumerate(rects):
        col = rng.random(3).astype(np.float32)
        a = np.float32(0.4 + 0.6 * rng.random())
        res0 = (rng.integers(-20, 21, 3).astype(np.float32) / np.float32(255.0))
        prims[i]["kind"], prims[i]["color0"], prims[i]["alpha"] = 0, col, a
        descs[i] = (i, 1, x0, y0, w, h, 16, -1, res0[0], res0[1], res0[2], 0.0)
        # blend over black: fma(c, a, 0 * (1 - a)) = c * a, then + RES0, clipped
        v = np.clip((col * a).astype(np.float32) + res0, 0.0, 1.0).astype(np.float32)
        ya, yb, xa, xb = max(0, y0), min(H, y0 + h), max(0, x0), min(W, x0 + w)
        if ya < yb and xa < xb:
            want[ya:yb, xa:xb] = v
    dev = torch.device("cuda", 0)
    lib = _lib.lib_for_device(0)
    items = decode_items(descs, H, W, prims)
    out = torch.full((H, W, 3), -1.0, dtype=torch.float32, device=dev)
    t_d = torch.from_numpy(descs.view(np.uint8)).to(dev)
    t_p = torch.from_numpy(prims.view(np.uint8)).to(dev)
    t_i = torch.from_numpy(items).to(dev)
    _lib.check(lib.weftk_render_tiles(_lib.ptr(t_d), n, _lib.ptr(t_i), len(items), _lib.ptr(t_p), 0, 0, 0, 0,
                                      _lib.ptr(out), H, W, 0, torch.cuda.current_stream().cuda_stream),
               "weftk_render_tiles")
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), want)
