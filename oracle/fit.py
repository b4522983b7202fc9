"""Greedy candidate-scoring fit (test oracle).

Restates the batched greedy of ``_fit_adaptive_state``
(src/weft/encoder.py:2668-2831) for given per-tile candidate pools:

* init: every candidate alone, objective ``mse + lam*(8 + 8*LUT[kind])`` in
  float32; keep the argmin (first on ties) (:2683-2715);
* current objective ``f64(mse) + lam*bits`` (:2718-2734); tiles with
  objective above 5e-4 (q < 90) or 5e-5 (q >= 90) and a non-empty pool are
  "complex" (:2738-2740);
* up to 20/8/4 rounds (q >= 90 / >= 70 / else) (:2745): each complex tile with
  pool left and room under its cap scores ``selected + [cand]`` for every
  remaining candidate; argmin of ``mse + lam*(base_bits + 8*LUT[kind])`` in
  float32 is accepted if below the current objective (:2788-2811);
* if no tile improved, re-seed the complex tiles that have room with
  residual-targeted candidates, at most 3 times (:2813-2828); otherwise the
  complex set becomes the tiles that improved (:2829-2831).

Scoring renders float32-rounded primitives, as the reference's GPU scorer
does with its packed float32 records.  Selections are returned as indices
into each tile's extended pool (initial candidates, then re-seeds in order).
"""

from __future__ import annotations

import numpy as np

from . import rate, render
from .primitives import PRIM_DTYPE, Prim, pack_prims

MAX_PRIMS_BY_SIZE = {8: 24, 16: 48, 32: 96}


def tile_cap(size: int) -> int:
    """Primitive cap per tile size (src/weft/quadtree.py:28-30, src/weft/constants.py:31)."""
    return MAX_PRIMS_BY_SIZE.get(size, 48)


def as_f32(p: Prim) -> Prim:
    rec = pack_prims([p])[0]
    n = {0: 0, 1: 4, 2: 5, 3: 7, 4: 6}.get(p.kind, 7)
    c1 = tuple(float(v) for v in rec["color1"]) if p.kind == 1 else None
    return Prim(p.kind, tuple(float(v) for v in rec["geom"][:n]), tuple(float(v) for v in rec["color0"]), c1,
                float(rec["alpha"]))


def stack_mse(patch: np.ndarray, prims) -> np.float32:
    return np.float32(np.mean((patch - render.render_tile(prims, patch.shape[0])) ** 2))


def greedy_fit(patches, sizes, pools, quality: int, reseed=None, caps=None, max_rounds=None, schedule=None):
    """Run the greedy; ``reseed(tile_index, patch, pred) -> list[Prim]``.

    The round loop's decisions are global over the tiles it is given: a round in which no tile
    improved is a stall (re-seed, or stop after the fourth in a row), otherwise the complex set
    becomes the tiles that improved.  ``schedule`` replays them from a larger fit these tiles
    belong to: one bool per greedy round that fit ran, True when any of its tiles improved; the
    tiles given here then take exactly the decisions they took there.

    Returns (selected index lists, current objectives (float64), stats dict).
    """
    n = len(patches)
    lam = rate.tile_lambda(quality)
    lut = rate.LUT
    caps = caps if caps is not None else [tile_cap(s) for s in sizes]
    ext = [list(p) for p in pools]
    f32 = [[as_f32(p) for p in pool] for pool in ext]
    alive = [list(range(len(p))) for p in ext]
    selected: list[list[int]] = [[] for _ in range(n)]
    cur = np.zeros(n, np.float64)
    stats = {"rounds": 0, "reseeds": 0, "evals": 0, "schedule": []}

    for i in range(n):
        kinds = np.array([p.kind for p in ext[i]], np.int32)
        mses = np.array([stack_mse(patches[i], [c]) for c in f32[i]], np.float32)
        stats["evals"] += len(mses)
        objs = mses + lam * (8 + lut[kinds] * 8).astype(np.float32)
        b = int(np.argmin(objs))
        selected[i] = [b]
        alive[i].remove(b)
        cur[i] = float(mses[b]) + lam * rate.estimate_bits([ext[i][b]], False)

    thr = 0.00005 if quality >= 90 else 0.0005
    complex_tiles = [i for i in range(n) if cur[i] > thr and alive[i]]
    if max_rounds is None:
        max_rounds = 20 if quality >= 90 else 8 if quality >= 70 else 4
    stalls = 0
    rounds = range(max_rounds) if schedule is None else range(len(schedule))
    for r in rounds:
        active = [i for i in complex_tiles if alive[i] and len(selected[i]) < caps[i]]
        if not active and schedule is None:
            break
        stats["rounds"] += 1
        improved = []
        for i in active:
            base = [f32[i][j] for j in selected[i]]
            mses = np.array([stack_mse(patches[i], base + [f32[i][j]]) for j in alive[i]], np.float32)
            stats["evals"] += len(mses)
            kinds = np.array([ext[i][j].kind for j in alive[i]], np.int32)
            base_bits = rate.estimate_bits([ext[i][j] for j in selected[i]], False)
            objs = mses + lam * (base_bits + (lut[kinds] * 8).astype(np.float32))
            b = int(np.argmin(objs))
            if float(objs[b]) < cur[i]:
                j = alive[i].pop(b)
                selected[i].append(j)
                cur[i] = float(objs[b])
                improved.append(i)
        stalled = not improved if schedule is None else not schedule[r]
        stats["schedule"].append(not stalled)
        if stalled:
            stalls += 1
            if stalls > 3:
                break
            for i in complex_tiles:
                if len(selected[i]) >= caps[i] or reseed is None:
                    continue
                pred = render.render_tile([ext[i][j] for j in selected[i]], sizes[i])
                new = list(reseed(i, patches[i], pred))
                stats["reseeds"] += 1
                base = len(ext[i])
                ext[i].extend(new)
                f32[i].extend(as_f32(p) for p in new)
                alive[i].extend(range(base, base + len(new)))
        else:
            stalls = 0
            complex_tiles = improved
    return selected, cur, stats


__all__ = ["greedy_fit", "stack_mse", "tile_cap", "as_f32", "PRIM_DTYPE"]
