"""The hand-written backward against central finite differences and a float64 autograd restatement.

64 random tiles (seed 1234), stacks of 1-4 primitives of kinds 0-4.  Smooth
kinds are checked in the normal forward; triangles in the soft-edge forward the
backward's surrogate differentiates.
"""

from __future__ import annotations

import functools

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

F64 = torch.float64


def _rand_stack(rng, ts, n):
    from weft_b200.candidates import Cand

    out = []
    for k in rng.integers(0, 5, n):
        k = int(k)
        lo, hi = 1.0, ts - 1.0
        g = {0: (), 1: tuple(rng.uniform(lo, hi, 4)), 2: tuple(rng.uniform(lo, hi, 4)) + (rng.uniform(0.7, 3.5),),
             3: tuple(rng.uniform(lo, hi, 6)) + (rng.uniform(0.7, 3.5),), 4: tuple(rng.uniform(lo, hi, 6))}[k]
        c1 = tuple(rng.uniform(0.05, 0.95, 3)) if k == 1 else None
        out.append(Cand(k, tuple(float(np.float32(v)) for v in g), tuple(rng.uniform(0.05, 0.95, 3)), c1,
                        float(rng.uniform(0.15, 0.9))))
    return out


def _workload(seed=1234, n_tiles=64, sizes=(8, 16, 32)):
    rng = np.random.default_rng(seed)
    sizes = rng.choice(list(sizes), n_tiles)
    patches = [rng.random((int(s), int(s), 3), dtype=np.float32) for s in sizes]
    stacks = [_rand_stack(rng, int(s), int(rng.integers(1, 5))) for s in sizes]
    return patches, stacks


def _seg_d2(px, py, ax, ay, bx, by):
    vx, vy = bx - ax, by - ay
    t = (((px - ax) * vx + (py - ay) * vy) / (vx * vx + vy * vy + 1e-8)).clamp(0.0, 1.0)
    ex, ey = px - ax - t * vx, py - ay - t * vy
    return ex * ex + ey * ey


@functools.lru_cache(maxsize=None)
def residual_operator(ts):
    """Dense float64 (n, n) matrix I - B M: M = 4x4 block means, B = the decoder's bilinear
    upsampling of the 4x4 grid at pixel centres with edge clamping."""
    n = ts * ts
    b = ts // 4
    M = np.zeros((16, n))
    B = np.zeros((n, 16))
    for y in range(ts):
        for x in range(ts):
            p = y * ts + x
            M[(y // b) * 4 + x // b, p] = 1.0 / (b * b)
            gx = min(max((x + 0.5) * 4.0 / ts - 0.5, 0.0), 3.0)
            gy = min(max((y + 0.5) * 4.0 / ts - 0.5, 0.0), 3.0)
            x0, y0 = int(np.floor(gx)), int(np.floor(gy))
            x1, y1 = min(x0 + 1, 3), min(y0 + 1, 3)
            wx, wy = gx - x0, gy - y0
            for nx, ny, w in ((x0, y0, (1 - wx) * (1 - wy)), (x1, y0, wx * (1 - wy)), (x0, y1, (1 - wx) * wy),
                              (x1, y1, wx * wy)):
                B[p, ny * 4 + nx] += w
    return torch.from_numpy(np.eye(n) - B @ M)


def ref_tile_loss(rows, kinds, src, soft, residual=False):
    """Float64 restatement of the renderer + tile MSE, differentiable by torch.  With
    ``residual`` the error is first passed through I - B M (the decoded residual grid)."""
    ts = src.shape[0]
    base = torch.arange(ts, dtype=F64) + 0.5
    py, px = torch.meshgrid(base, base, indexing="ij")
    c = torch.zeros(ts, ts, 3, dtype=F64)
    tgrid = [float(np.float32(v)) for v in np.linspace(0, 1, 32, dtype=np.float32)]
    for r, k in zip(rows, kinds):
        A = r[13].clamp(0.0, 1.0)
        s = r[7:10].expand(ts, ts, 3)
        cov = torch.ones(ts, ts, dtype=F64)
        if k == 1:
            x0, y0, x1, y1 = r[0], r[1], r[2], r[3]
            vx, vy = x1 - x0, y1 - y0
            t = (((px - x0) * vx + (py - y0) * vy) / (vx * vx + vy * vy + 1e-8)).clamp(0.0, 1.0)[..., None]
            s = r[7:10] * (1 - t) + r[10:13] * t
        elif k in (2, 3):
            if k == 2:
                d2 = _seg_d2(px, py, r[0], r[1], r[2], r[3])
                th = r[4]
            else:
                pts = [((1 - t) ** 2 * r[0] + 2 * (1 - t) * t * r[2] + t * t * r[4],
                        (1 - t) ** 2 * r[1] + 2 * (1 - t) * t * r[3] + t * t * r[5]) for t in tgrid]
                d2 = torch.stack([_seg_d2(px, py, *pts[j], *pts[j + 1]) for j in range(31)]).min(0).values
                th = r[6]
            sig = th.clamp(min=0.5)
            cov = torch.exp(-d2 / (2 * sig * sig))
        elif k == 4:
            x = [r[0], r[2], r[4]]
            y = [r[1], r[3], r[5]]
            a2 = (x[1] - x[0]) * (y[2] - y[0]) - (y[1] - y[0]) * (x[2] - x[0])
            o = 1.0 if float(a2.detach()) >= 0 else -1.0
            cov = torch.ones(ts, ts, dtype=F64)
            for i in range(3):
                ia, ib = (i + 1) % 3, (i + 2) % 3
                ex, ey = x[ib] - x[ia], y[ib] - y[ia]
                C = ex * (py - y[ia]) - ey * (px - x[ia])
                sd = o * C / (torch.sqrt(ex * ex + ey * ey) + 1e-12)
                cov = cov * torch.sigmoid(sd / 0.5)
            assert soft
        a = (A * cov)[..., None]
        c = s * a + c * (1 - a)
    e = c.clamp(0.0, 1.0) - torch.from_numpy(src).to(F64)
    if residual:
        e = (residual_operator(ts) @ e.reshape(-1, 3)).reshape(ts, ts, 3)
    return (e ** 2).mean()


def _split(stacks):
    tri = [[p for p in s if p.kind == 4] for s in stacks]
    smooth = [[p for p in s if p.kind != 4] or [s[0]] for s in stacks]
    smooth = [[p for p in s if p.kind != 4] for s in smooth]
    return smooth, tri


@pytest.mark.parametrize("soft,residual", [(False, False), (True, False), (False, True), (True, True)])
def test_backward_matches_float64_autograd(soft, residual):
    from weft_b200.refine import StackSet

    patches, stacks = _workload(sizes=(8, 16, 32, 64) if residual else (8, 16, 32))
    stacks = [[p for p in s if (p.kind == 4) == soft] for s in stacks]
    keep = [i for i, s in enumerate(stacks) if s]
    patches = [patches[i] for i in keep]
    stacks = [stacks[i] for i in keep]
    assert len(stacks) >= 20
    ss, params = StackSet.from_stacks(patches, stacks)
    g = torch.rand(ss.n, device=params.device) + 0.5
    got = ss.loss_backward(params, g, soft=soft, residual=residual).cpu().numpy()
    rows = params.cpu().numpy().astype(np.float64)
    off = ss.prim_off_np
    worst = 0.0
    for t in range(ss.n):
        r = torch.tensor(rows[off[t]:off[t + 1]], dtype=F64, requires_grad=True)
        L = ref_tile_loss(list(r), [p.kind for p in stacks[t]], patches[t], soft, residual) * float(g[t])
        L.backward()
        want = r.grad.numpy()[:, :14]
        have = got[off[t]:off[t + 1], :14]
        # absolute floor: under the residual loss a lone constant layer's gradient is
        # zero up to rounding (the residual grid absorbs any constant shift)
        scale = max(np.abs(want).max(), 1e-5)
        err = np.abs(have - want).max() / scale
        worst = max(worst, err)
        assert err < 2e-3, f"tile {t} kinds {[p.kind for p in stacks[t]]}: rel err {err}"
    # loss values agree too
    loss = ss.loss(params, soft=soft, residual=residual).cpu().numpy()
    for t in range(0, ss.n, 5):
        r = torch.tensor(rows[off[t]:off[t + 1]], dtype=F64)
        want = float(ref_tile_loss(list(r), [p.kind for p in stacks[t]], patches[t], soft, residual))
        assert loss[t] == pytest.approx(want, rel=2e-5 if not residual else 1e-4)


@pytest.mark.parametrize("soft", [False, True])
def test_backward_matches_central_differences(soft):
    from weft_b200.refine import StackSet

    patches, stacks = _workload()
    stacks = [[p for p in s if (p.kind == 4) == soft] for s in stacks]
    keep = [i for i, s in enumerate(stacks) if s]
    patches = [patches[i] for i in keep]
    stacks = [stacks[i] for i in keep]
    ss, params = StackSet.from_stacks(patches, stacks)
    ones = torch.ones(ss.n, device=params.device)
    grad = ss.loss_backward(params, ones, soft=soft).cpu().numpy()
    off = ss.prim_off_np
    h = 1e-3
    kmax = int(np.diff(off).max())
    fd = np.zeros_like(grad)
    for k in range(kmax):
        rows_k = [off[t] + k for t in range(ss.n) if off[t] + k < off[t + 1]]
        tiles_k = [t for t in range(ss.n) if off[t] + k < off[t + 1]]
        for j in range(14):
            pp, pm = params.clone(), params.clone()
            pp[rows_k, j] += h
            pm[rows_k, j] -= h
            lp = ss.loss(pp, soft=soft).double().cpu().numpy()
            lm = ss.loss(pm, soft=soft).double().cpu().numpy()
            fd[rows_k, j] = (lp[tiles_k] - lm[tiles_k]) / (2 * h)
    checked = 0
    for t in range(ss.n):
        for k in range(off[t], off[t + 1]):
            kind = stacks[t][k - off[t]].kind
            cols = {0: [7, 8, 9, 13], 1: [0, 1, 2, 3, 7, 8, 9, 10, 11, 12, 13], 2: [0, 1, 2, 3, 4, 7, 8, 9, 13],
                    3: [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 13], 4: [0, 1, 2, 3, 4, 5, 7, 8, 9, 13]}[kind]
            a, b = grad[k, cols], fd[k, cols]
            scale = max(np.abs(b).max(), 1e-4)
            assert np.abs(a - b).max() / scale < 3e-2, f"tile {t} kind {kind}: {a} vs {b}"
            checked += 1
    assert checked >= 20


def test_refine_lowers_loss_and_stays_representable():
    from weft_b200 import candidates, quadtree
    from weft_b200.fit import BatchedFit
    from weft_b200.refine import StackSet, refine
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(256, 256, 40, 0)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, qts, 64)
    pools = [candidates.tile_candidates(p, 75) for p in patches]
    fit = BatchedFit(patches, pools, 75, caps=[16] * len(qts)).run()
    ss, params = StackSet.from_fit(fit)
    p0 = params.clone()
    ss.project_(p0)
    before = float((ss.loss(p0) * ss.weights).sum())
    out, hist = refine(ss, params, steps=60, lr=1e-2)
    after = float((ss.loss(out) * ss.weights).sum())
    assert after < before * 0.98 and len(hist) == 60
    q = ss.quantize(out)
    assert float(q[:, 7:14].min()) >= 0 and float(q[:, 7:14].max()) <= 1
    assert float((ss.loss(q) * ss.weights).sum()) < before
