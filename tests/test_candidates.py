"""The product's candidate generators reproduce the reference's pools value for value."""

from __future__ import annotations

import numpy as np

from oracle.primitives import prims_from_pack
from tests.test_oracle_golden import _pack
from weft_b200 import candidates


def _same(got, want):
    assert len(got) == len(want)
    for a, b in zip(got, want):
        assert a.kind == b.kind
        assert tuple(float(v) for v in a.geom) == tuple(b.geom)
        assert tuple(float(v) for v in a.color0) == tuple(b.color0)
        assert (None if a.color1 is None else tuple(float(v) for v in a.color1)) == b.color1
        assert float(a.alpha) == b.alpha


def test_initial_and_residual_pools_match_reference(golden):
    g = golden("candidates.npz")
    c, r = _pack(g, "c_"), _pack(g, "r_")
    for i, ts in enumerate(g["sizes"]):
        a, b = int(g["px_offsets"][i]), int(g["px_offsets"][i + 1])
        patch = g["patch"][a:b].reshape(ts, ts, 3)
        pred = g["pred"][a:b].reshape(ts, ts, 3)
        _same(candidates.tile_candidates(patch, 75), prims_from_pack(c, int(c["offsets"][i]), int(c["offsets"][i + 1])))
        _same(candidates.residual_candidates(patch, pred, 75),
              prims_from_pack(r, int(r["offsets"][i]), int(r["offsets"][i + 1])))


def test_fit_golden_pools_match_reference(golden):
    """Every tile of the recorded reference fit gets the same initial pool."""
    from oracle import quadtree as oq

    for name in ("fit_small.npz", "fit_hq.npz"):
        g = golden(name)
        tiles = [oq.QTile(int(x), int(y), int(s)) for x, y, s in g["qt"]]
        patches = oq.extract(g["image"], tiles)
        pool = _pack(g, "pool_")
        for i, p in enumerate(patches):
            _same(candidates.tile_candidates(p, int(g["quality"])),
                  prims_from_pack(pool, int(pool["offsets"][i]), int(pool["offsets"][i + 1])))


def test_kind_restricted_pools_are_the_filtered_full_pools(golden):
    """``tile_candidates(..., kinds=...)`` generates only those kinds and equals the full pool
    filtered to them, in order (the refined fit's constant + linear pools)."""
    g = golden("candidates.npz")
    for i, ts in enumerate(g["sizes"]):
        a, b = int(g["px_offsets"][i]), int(g["px_offsets"][i + 1])
        patch = g["patch"][a:b].reshape(ts, ts, 3)
        for q in (40, 75, 92):
            full = candidates.tile_candidates(patch, q)
            for kinds in ((0, 1), (0, 1, 2), (1, 4)):
                assert candidates.tile_candidates(patch, q, kinds=kinds) == [c for c in full if c.kind in kinds]


def test_bench_restricted_pools_match_filtered_full_pools():
    """The bench's directly generated constant + linear pools (worker processes) equal the full
    pools filtered to those kinds, under the same float32 arctan2 rule."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    import bench
    from weft_b200 import quadtree
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(128, 128, 25, 9)
    img = srgb_u8_to_linear(u8)
    tiles = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, tiles, 64)
    pools = [bench._pool_cands((p, 75, None, "rounded")) for p in patches]
    with ProcessPoolExecutor(max_workers=2, mp_context=mp.get_context("spawn")) as ex:
        got, gen_s = bench.restricted_pools(patches, (0, 1), ex)
    assert gen_s > 0 and len(got) == len(patches)
    for g, f in zip(got, pools):
        assert np.array_equal(g.view(np.uint8), f[np.isin(f["kind"], (0, 1))].view(np.uint8))


def test_arctan2_rule_only_moves_the_edge_pool_orientations():
    """The two float32 arctan2 rules give pools that differ only in the edge pool's linear
    splits (their orientation is the only value the Sobel angle decides)."""
    from weft_b200 import quadtree
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(128, 128, 25, 9)
    img = srgb_u8_to_linear(u8)
    tiles = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    for p in quadtree.extract_tiles(img, tiles, 64)[::5]:
        a = candidates.tile_candidates(p, 75, atan2="numpy")
        b = candidates.tile_candidates(p, 75, atan2="rounded")
        assert [c for c in a if c.kind != 1] == [c for c in b if c.kind != 1]
