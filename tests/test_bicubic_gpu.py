"""GPU parity of the per-tile bicubic R-D swap (src/weft/encoder.py:2841-2873).

The control grids are float64 products rounded to float32 and then to u8 steps, so they equal
the reference's unless a product lands on a rounding boundary (none does in these cases); the
scores are float32 squared errors summed in float64 (the reference: numpy's float32 mean),
within 1e-6 relative for the bicubic score and within the scorer's 1e-5 for the stack's, which
the device renders from float32 records; the decisions must be the reference's.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import bicubic as obic
from oracle import fit as ofit
from oracle import quadtree as oq
from oracle import rate as orate
from oracle.primitives import Prim
from tests.test_oracle_golden import bicubic_swap_inputs

pytestmark = pytest.mark.gpu


def _device_tiles(patches):
    sizes = np.array([p.shape[0] for p in patches], np.int32)
    px = np.zeros((int((sizes.astype(np.int64) ** 2).sum()), 4), np.float32)
    px[:, :3] = np.concatenate([p.reshape(-1, 3) for p in patches])
    off = np.concatenate([[0], np.cumsum(sizes.astype(np.int64) ** 2)[:-1]]).astype(np.int32)
    dev = torch.device("cuda", 0)
    return torch.from_numpy(px).to(dev), torch.from_numpy(off).to(dev), torch.from_numpy(sizes).to(dev)


@pytest.mark.parametrize("name", ["a", "b", "c"])
def test_swap_matches_reference_fit(golden, name):
    from weft_b200 import bicubic

    g = golden("bicubic.npz")
    patches, stacks, lam = bicubic_swap_inputs(g, name)
    quality = int(g[f"{name}_quality"])
    assert lam == orate.tile_lambda(quality)
    flags, grids, scores = bicubic.swap(*_device_tiles(patches), stacks, quality)
    want = g[f"{name}_swapped"].astype(bool)
    np.testing.assert_array_equal(flags, want)
    np.testing.assert_array_equal(grids[want], g[f"{name}_grids"][want])
    # the device renders the 60-byte float32 records: the oracle on the same rounded values
    o_flags, o_grids, o_bic, o_stack = obic.swap(patches, [[ofit.as_f32(p) for p in s] for s in stacks], lam)
    np.testing.assert_array_equal(grids, o_grids)
    np.testing.assert_allclose(scores[:, 0], o_bic, rtol=1e-6)
    np.testing.assert_allclose(scores[:, 1], o_stack, rtol=1e-5)
    out = bicubic.replaced_stacks(stacks, flags, grids)
    assert all(len(s) == 1 and s[0].kind == 5 for s, f in zip(out, flags) if f)
    assert all(s is not st and s == list(st) for s, st, f in zip(out, stacks, flags) if not f)


def _random_stack(rng, ts):
    out = []
    for _ in range(int(rng.integers(0, 4))):
        k = int(rng.integers(0, 5))
        c0 = tuple(float(v) for v in rng.random(3).astype(np.float32))
        c1 = tuple(float(v) for v in rng.random(3).astype(np.float32)) if k == 1 else None
        g = {0: 0, 1: 4, 2: 5, 3: 7, 4: 6}[k]
        geom = [float(v) for v in (rng.random(g) * ts).astype(np.float32)]
        if k in (2, 3):
            geom[-1] = float(np.float32(0.5 + 2 * rng.random()))
        out.append(Prim(k, tuple(geom), c0, c1, float(np.float32(0.5 + 0.5 * rng.random()))))
    return out


@pytest.mark.parametrize("quality", [75, 95])
def test_swap_matches_oracle_on_random_tiles(quality):
    """Random stacks of every kind (and empty stacks) over noise, smooth and edge tiles of every
    side; decisions equal wherever the two scores are not within 1e-6 of each other."""
    from weft_b200 import bicubic

    rng = np.random.default_rng(9)
    img = rng.random((256, 256, 3), dtype=np.float32)
    yy, xx = np.meshgrid(np.linspace(0, 1, 256), np.linspace(0, 1, 256), indexing="ij")
    img[:128, :, 0] = (0.2 + 0.6 * xx[:128]).astype(np.float32)
    img[:128, :, 1] = (0.3 + 0.4 * yy[:128] * xx[:128]).astype(np.float32)
    img[:128, :, 2] = (0.9 - 0.8 * yy[:128]).astype(np.float32)
    tiles = []
    for s in (8, 16, 32, 64):
        for k in range(12):
            tiles.append(oq.QTile(int(rng.integers(0, 256 - s)), int(rng.integers(0, 256 - s)), s))
    patches = oq.extract(img, tiles)
    stacks = [_random_stack(rng, t.size) for t in tiles]
    for i, (t, patch) in enumerate(zip(tiles, patches)):
        if i % 2 == 0:  # every other tile: one constant patch of the tile's mean colour
            stacks[i] = [Prim(0, (), tuple(float(v) for v in patch.reshape(-1, 3).mean(0)), None, 1.0)]
    lam = orate.tile_lambda(quality)
    flags, grids, scores = bicubic.swap(*_device_tiles(patches), stacks, quality)
    o_flags, o_grids, o_bic, o_stack = obic.swap(patches, stacks, lam)
    np.testing.assert_array_equal(grids, o_grids)
    np.testing.assert_allclose(scores[:, 0], o_bic, rtol=1e-6)
    np.testing.assert_allclose(scores[:, 1], o_stack, rtol=1e-5)
    near = np.abs(o_bic - o_stack) <= 1e-6 * np.maximum(np.abs(o_bic), np.abs(o_stack))
    np.testing.assert_array_equal(flags[~near], o_flags[~near])
    assert 0 < o_flags.sum() < len(o_flags)


def test_fit_bicubic_swap_follows_its_selections(golden):
    """BatchedFit.bicubic_swap on the reference's q=92 fit: the same decisions as the reference."""
    from tests.test_oracle_golden import _fit_inputs
    from weft_b200.fit import BatchedFit

    g = golden("fit_hq.npz")
    tiles, patches, pools, reseeds = _fit_inputs(g)
    queue = {k: list(v) for k, v in reseeds.items()}
    fit = BatchedFit(patches, pools, int(g["quality"]))
    fit.run(reseed=lambda i, patch, pred: queue[i].pop(0))
    flags, grids, stacks = fit.bicubic_swap()
    o_flags, o_grids, o_bic, o_stack = obic.swap(patches, fit.selected(), orate.tile_lambda(int(g["quality"])))
    np.testing.assert_array_equal(flags, o_flags)
    np.testing.assert_array_equal(grids, o_grids)
    assert [s[0].kind for s, f in zip(stacks, flags) if f] == [5] * int(flags.sum())
