"""Device generation of the constant + linear candidate pools (``weftk_gen_pools``) against the
host restatement of the reference's generators (``candidates.tile_candidates`` with kinds
(0, 1)) under the same float32 arctan2 rule: identical pools, record for record, on every tile
side, on flat tiles (the histogram's fallback orientations) and on noise."""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _device_pools(patches, quality):
    from weft_b200 import pools
    from weft_b200._lib import PRIM_DTYPE

    dev = torch.device("cuda", 0)
    sizes = np.array([p.shape[0] for p in patches], np.int32)
    px = sizes.astype(np.int64) ** 2
    px_off = np.concatenate([[0], np.cumsum(px)[:-1]]).astype(np.int32)
    src = np.zeros((int(px.sum()), 4), np.float32)
    src[:, :3] = np.concatenate([p.reshape(-1, 3) for p in patches])
    cap = pools.MAX_CONST_LINEAR
    pool_off = (np.arange(len(patches)) * cap).astype(np.int32)
    t_cand = torch.zeros(len(patches) * cap * PRIM_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    t_cnt = torch.full((len(patches),), -1, dtype=torch.int32, device=dev)
    pools.generate_pools(torch.from_numpy(src).to(dev), torch.from_numpy(px_off).to(dev), sizes,
                         torch.from_numpy(pool_off).to(dev), t_cand, t_cnt, quality)
    torch.cuda.synchronize()
    recs = t_cand.cpu().numpy().view(PRIM_DTYPE)
    cnt = t_cnt.cpu().numpy()
    return [recs[i * cap:i * cap + int(cnt[i])] for i in range(len(patches))]


def _host_pool(patch, quality):
    from weft_b200 import candidates
    from weft_b200.fit import pack_cands

    return pack_cands(candidates.tile_candidates(patch, quality, kinds=(0, 1), atan2="rounded"))


def _compare(patches, quality):
    got = _device_pools(patches, quality)
    bad = []
    for i, (p, g) in enumerate(zip(patches, got)):
        want = _host_pool(p, quality)
        if len(g) != len(want) or g.tobytes() != want.tobytes():
            bad.append((i, p.shape[0], len(g), len(want)))
    return bad, sum(len(g) for g in got)


@pytest.mark.parametrize("quality", [75, 92])
def test_device_pools_equal_host_pools_on_quadtree_tiles(quality):
    from weft_b200 import quadtree
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(256, 256, 60, 4)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, qts, 64)
    assert {p.shape[0] for p in patches} == {8, 16, 32, 64}
    bad, n = _compare(patches, quality)
    assert n > 20 * len(patches)
    assert not bad, f"{len(bad)} of {len(patches)} tiles differ, e.g. {bad[:5]}"


def test_device_pools_flat_and_noise_tiles():
    rng = np.random.default_rng(11)
    patches = []
    for s in (8, 16, 32, 64):
        patches.append(np.full((s, s, 3), 0.25, np.float32))                # flat: fallback orientations
        patches.append(rng.random((s, s, 3), dtype=np.float32))             # noise
        t = np.zeros((s, s, 3), np.float32)
        t[:, s // 3:] = (0.9, 0.1, 0.4)                                     # one vertical edge
        patches.append(t)
        patches.append((np.floor(rng.random((s, s, 3)) * 4) / 4).astype(np.float32))  # many exact ties
    bad, _ = _compare(patches, 75)
    assert not bad, bad


def test_fit_over_device_pools_equals_fit_over_host_pools():
    """The greedy (device re-seeds) and the refined fit's init round over device-generated pools
    pick what they pick over the same pools generated on the host."""
    from weft_b200 import candidates, pools, quadtree
    from weft_b200._lib import PRIM_DTYPE
    from weft_b200.fit import RESEED_RESERVE, BatchedFit, pack_cands
    from weft_b200.refine import RefinedFit
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(192, 128, 30, 8)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, qts, 64)
    sizes = np.array([p.shape[0] for p in patches], np.int32)
    host = [pack_cands(candidates.tile_candidates(p, 75, kinds=(0, 1), atan2="rounded")) for p in patches]
    dev = torch.device("cuda", 0)
    stride = pools.MAX_CONST_LINEAR + RESEED_RESERVE
    px = sizes.astype(np.int64) ** 2
    src = torch.zeros((int(px.sum()), 4), dtype=torch.float32, device=dev)
    src[:, :3] = torch.from_numpy(np.concatenate([p.reshape(-1, 3) for p in patches])).to(dev)
    px_off = torch.from_numpy(np.concatenate([[0], np.cumsum(px)[:-1]]).astype(np.int32)).to(dev)
    pool_off = torch.from_numpy((np.arange(len(patches)) * stride).astype(np.int32)).to(dev)
    cand = torch.zeros(len(patches) * stride * PRIM_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    cnt = torch.zeros(len(patches), dtype=torch.int32, device=dev)
    pools.generate_pools(src, px_off, sizes, pool_off, cand, cnt, 75, pool_cap=stride)
    dfit = BatchedFit.from_device_pools(src, sizes, cand, cnt, stride, 75, caps=[16] * len(sizes))
    hfit = BatchedFit(patches, host, 75, caps=[16] * len(sizes))
    for f in (dfit, hfit):
        f.run_device()
    assert dfit.selected_indices() == hfit.selected_indices()
    np.testing.assert_array_equal(dfit.objectives(), hfit.objectives())
    assert dfit.control() == hfit.control()
    dfit.quantize_selected()
    hfit.quantize_selected()
    assert torch.equal(dfit.t_qrows, hfit.t_qrows) and torch.equal(dfit.t_qkind, hfit.t_qkind)

    hfast = BatchedFit(patches, host, 75, caps=[16] * len(sizes), reserve=0)
    rows = []
    for f in (dfit, hfast):
        rf = RefinedFit(f, steps=5, lr=1e-2, use_graph=True)
        rf.run()
        rows.append(rf.q_rows.clone())
    torch.testing.assert_close(rows[0], rows[1], rtol=0, atol=0)


def test_device_refined_fit_graph_replays_and_matches_host_pools():
    """Generation + init round + Adam + snap from one CUDA graph: replays give the same rows, equal
    to the refined fit over the same pools generated on the host."""
    from weft_b200 import candidates, pools, quadtree
    from weft_b200.fit import BatchedFit, pack_cands
    from weft_b200.refine import RefinedFit
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(128, 128, 20, 2)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, qts, 64)
    sizes = np.array([p.shape[0] for p in patches], np.int32)
    dev = torch.device("cuda", 0)
    src = torch.zeros((int((sizes.astype(np.int64) ** 2).sum()), 4), dtype=torch.float32, device=dev)
    src[:, :3] = torch.from_numpy(np.concatenate([p.reshape(-1, 3) for p in patches])).to(dev)
    drf = pools.DeviceRefinedFit(src, sizes, 75, caps=[16] * len(sizes), steps=4)
    a = drf.run().clone()
    b = drf.run().clone()
    assert torch.equal(a, b)
    host = [pack_cands(candidates.tile_candidates(p, 75, kinds=(0, 1), atan2="rounded")) for p in patches]
    got = drf.pool_records()
    assert all(g.tobytes() == h.tobytes() for g, h in zip(got, host))
    hf = BatchedFit(patches, host, 75, caps=[16] * len(sizes), reserve=0)
    rf = RefinedFit(hf, steps=4, lr=1e-2, use_graph=False)
    rf.run()
    assert torch.equal(a, rf.q_rows)


@pytest.mark.parametrize("quality", [75, 92])
def test_side_bit_table_matches_the_host_side_tests(quality):
    """The device's side-bit table against the split tests of ``candidates`` (the orientation
    lines with Python-float endpoints on the float32 grid, the template lines as float32)."""
    from weft_b200 import pools
    from weft_b200.candidates import _int_grid

    tb = pools.PoolTables(quality, 0)
    for s in pools.SIDES:
        got = tb.side_masks(s)
        ys, xs = _int_grid(s, s)
        for oi, th in enumerate(pools.orientation_angles()):
            x0, y0, x1, y1 = pools.orientation_lines(s, th)[0]
            want = (xs - x0) * (y1 - y0) - (ys - y0) * (x1 - x0) >= 0
            assert np.array_equal(got[oi], want), (s, oi)
        specs, _ = pools.template_specs(s, quality)
        lines = np.array([sp[:4] for sp in specs], dtype=np.float32)
        for k, (x0, y0, x1, y1) in enumerate(lines):
            want = (xs - x0) * (y1 - y0) - (ys - y0) * (x1 - x0) >= 0
            assert np.array_equal(got[16 + k], want), (s, k)
        assert not got[16 + len(specs):].any()
