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
