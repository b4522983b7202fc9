"""The drop-in launcher under the reference's own calls.

The reference cannot run on the GPU machine, so its fit's first three calls to
``gpu_batch_score_prepacked`` (the init round, the current objective of the selected stacks and the
first greedy round; src/weft/encoder.py:2698-2811) were recorded with their arguments exactly as the
fit passes them (``tests/golden/launcher_calls.npz``).  Here they go through the launcher that
``weft_b200.install_into`` puts in place of the reference's, and the fit's decisions are replayed
from the returned MSEs.
"""

from __future__ import annotations

import types

import numpy as np
import pytest

from oracle import rate as orate

pytestmark = pytest.mark.gpu


def recorded_calls(g):
    from weft_b200.gpu_render import _PRIM_DTYPE

    calls = []
    for i in range(int(g["n_calls"])):
        p = f"c{i}_"
        offsets = dict(zip((int(k) for k in g[p + "offset_keys"]), (int(v) for v in g[p + "offset_vals"])))
        raw = g[p + "prims"]
        ends = np.cumsum(g[p + "prim_len"]) * _PRIM_DTYPE.itemsize
        prim_arrays = [np.frombuffer(raw[a:b].tobytes(), _PRIM_DTYPE) for a, b in zip(np.r_[0, ends[:-1]], ends)]
        cends = np.cumsum(g[p + "count_len"])
        counts = [g[p + "counts"][a:b] for a, b in zip(np.r_[0, cends[:-1]], cends)]
        args = (g[p + "pixels"], offsets, [int(t) for t in g[p + "tile_indices"]],
                [int(s) for s in g[p + "tile_sizes"]], prim_arrays, counts)
        mends = np.cumsum(g[p + "count_len"])
        want = [g[p + "mse"][a:b] for a, b in zip(np.r_[0, mends[:-1]], mends)]
        calls.append((args, want))
    return calls


def objectives(mse, arr, counts, lam):
    """mse + lambda * bits of every eval (8 + 8 * byte size of each of its primitives)."""
    kinds = arr["kind"]
    out, o = [], 0
    for k, nc in enumerate(counts):
        nc = int(nc)
        bits = 8 + 8 * sum(orate.PRIM_BYTES.get(int(kinds[o + m]), 20) for m in range(nc))
        out.append(float(mse[k]) + lam * bits)
        o += nc
    return np.array(out)


def test_installed_launcher_reproduces_the_reference_fit_calls(golden):
    import weft_b200

    g = golden("launcher_calls.npz")
    ns = types.SimpleNamespace()  # stands in for the reference's weft.gpu_render module
    weft_b200.install_into(ns)
    lam = orate.tile_lambda(int(g["quality"]))
    results = []
    for args, want in recorded_calls(g):
        got = ns.gpu_batch_score_prepacked(*args)
        assert len(got) == len(want)
        for a, b in zip(got, want):
            np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-9)
        results.append((args, got))
    # init round: every tile takes its best single candidate, the reference's first selection
    (args0, got0), (args1, got1), (args2, got2) = results
    init_pick = [int(np.argmin(objectives(m, a, c, lam))) for m, a, c in zip(got0, args0[4], args0[5])]
    assert init_pick == [int(row[0]) for row in g["selected"]]
    # first greedy round: no candidate beats a tile's current objective, so the reference's round
    # stalled on every tile (it kept one primitive per tile)
    cur = [objectives(m, a, c, lam)[0] for m, a, c in zip(got1, args1[4], args1[5])]
    best = [objectives(m, a, c, lam).min() for m, a, c in zip(got2, args2[4], args2[5])]
    assert all(b >= c for b, c in zip(best, cur))
    assert all(int((row >= 0).sum()) == 1 for row in g["selected"])
