"""The device generator's host-built tables (``pools.build_tables``) against the host
restatement of the reference's generators: the same float64 split geometry, in the same order,
and side tests that select exactly the reference's pixels (CPU, no GPU)."""

from __future__ import annotations

import numpy as np
import pytest

from weft_b200 import candidates, pools


def _side_a(c, size):
    ys, xs = np.meshgrid(np.arange(size, dtype=np.float32), np.arange(size, dtype=np.float32), indexing="ij")
    x0, y0, dy, dx = (np.float32(v) for v in c)
    return (xs - x0) * dy - (ys - y0) * dx >= 0


@pytest.mark.parametrize("quality", [40, 75, 92])
def test_template_split_geometry_and_masks(quality):
    tb = pools.build_tables(quality)
    rng = np.random.default_rng(quality)
    for si, size in enumerate(pools.SIDES):
        tile = rng.random((size, size, 3), dtype=np.float32)
        lin = [c for c in candidates.template_candidates(tile, quality, kinds={1})]
        raw = [c for c in candidates._template_raw(tile, quality, frozenset({1}))]
        n_spec, n_centre = tb["n_spec"], tb["n_centre"]
        want = []
        for i in range(n_spec):
            want += [tuple(tb["spec_geom"][si, i])] * (3 if i < n_centre else 1)
        assert [tuple(c.geom) for c in raw] == want
        assert len(lin) <= len(raw)
        # the float32 side test selects the batched side means' pixels
        specs, _ = pools.template_specs(size, quality)
        lines = np.array([s[:4] for s in specs], dtype=np.float32)
        ys, xs = np.meshgrid(np.arange(size, dtype=np.float32), np.arange(size, dtype=np.float32), indexing="ij")
        for i in range(n_spec):
            x0, y0, x1, y1 = (lines[i, k] for k in range(4))
            ref = (xs - x0) * (y1 - y0) - (ys - y0) * (x1 - x0) >= 0
            assert np.array_equal(_side_a(tb["spec_mask"][si, i], size), ref)


def test_orientation_split_geometry_and_masks(monkeypatch):
    """With every orientation forced dominant, the edge pool's split lines follow the table."""
    tb = pools.build_tables(75)
    angles = pools.orientation_angles()
    monkeypatch.setattr(candidates, "dominant_orientations", lambda angle, mag, n_bins=12: list(angles))
    rng = np.random.default_rng(3)
    for si, size in enumerate(pools.SIDES):
        tile = rng.random((size, size, 3), dtype=np.float32)
        raw = [c for c in candidates._edge_raw(tile, 75, frozenset({1})) if c.kind == 1]
        want = []
        for oi in range(16):
            g = [tuple(v) for v in tb["orient_geom"][si, oi]]
            want += [g[0]] * 3 + [g[1], g[2]]
        assert [tuple(c.geom) for c in raw] == want
        ys, xs = np.meshgrid(np.arange(size, dtype=np.float32), np.arange(size, dtype=np.float32), indexing="ij")
        for oi, th in enumerate(angles):
            x0, y0, x1, y1 = pools.orientation_lines(size, th)[0]
            ref = (xs - x0) * (y1 - y0) - (ys - y0) * (x1 - x0) >= 0
            assert np.array_equal(_side_a(tb["orient_mask"][si, oi], size), ref)


def test_bin_edges_and_palette_cuts():
    tb = pools.build_tables(75)
    np.testing.assert_array_equal(tb["bin_edges"], np.linspace(0, np.pi, 13))
    for si, size in enumerate(pools.SIDES):
        n = size * size
        for ki, k in enumerate((2, 3, 4)):
            c = (np.arange(k + 1, dtype=np.float64) * (n / k)).astype(np.int64)
            assert list(tb["cuts"][si, ki, :k + 1]) == list(c)
