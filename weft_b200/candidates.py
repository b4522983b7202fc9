"""Per-tile candidate pools for the greedy fit (host side, numpy).

The plain fit's result depends on the exact candidate pools, so this module
reproduces the reference's generators value for value:

* ``tile_candidates`` = edge-driven candidates + template candidates,
  de-duplicated (``_worker_gen_cands``, src/weft/encoder.py:2490-2517);
* ``edge_candidates``  (``generate_edge_driven_candidates``, src/weft/edge_analysis.py:139-315);
* ``template_candidates`` (``_generate_candidates``, src/weft/encoder.py:535-745);
* ``residual_candidates`` (``_generate_residual_candidates``, src/weft/encoder.py:1255-1366),
  used to re-seed stalled tiles;
* ``dedup`` (``_dedup_candidates``, src/weft/encoder.py:447-528).

The numpy call sequence (dtypes, reductions, sort calls) is kept where it
decides a value: means are float32 pairwise sums, sorts use numpy's default
kinds, k-means seeds come from ``default_rng(42)``.  Candidates are returned
as ``Cand`` records (kind, geom, color0, color1, alpha) with Python floats.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from functools import lru_cache

import numpy as np


@dataclass(slots=True)
class Cand:
    kind: int
    geom: tuple = ()
    color0: tuple = (0.0, 0.0, 0.0)
    color1: tuple | None = None
    alpha: float = 1.0


def clamp_rgb(a) -> tuple[float, float, float]:
    return (max(0.0, min(1.0, float(a[0]))), max(0.0, min(1.0, float(a[1]))), max(0.0, min(1.0, float(a[2]))))


def luminance(tile: np.ndarray) -> np.ndarray:
    return 0.2126 * tile[..., 0] + 0.7152 * tile[..., 1] + 0.0722 * tile[..., 2]


@lru_cache(maxsize=16)
def _int_grid(h: int, w: int) -> tuple[np.ndarray, np.ndarray]:
    return np.meshgrid(np.arange(h, dtype=np.float32), np.arange(w, dtype=np.float32), indexing="ij")


def palette_means(pixels: np.ndarray, k: int) -> np.ndarray:
    """k colours: luminance-sorted pixels cut into k equal-count runs, mean of each
    (``_kmeans_colors``, src/weft/encoder.py:414-439)."""
    n = len(pixels)
    if n <= k:
        out = np.zeros((k, 3), dtype=np.float32)
        out[:n] = pixels[:n]
        return out
    order = np.argsort(0.2126 * pixels[:, 0] + 0.7152 * pixels[:, 1] + 0.0722 * pixels[:, 2])
    srt = pixels[order]
    cuts = (np.arange(k + 1, dtype=np.float64) * (n / k)).astype(np.int64)
    out = np.empty((k, 3), dtype=np.float32)
    for j in range(k):
        a, b = int(cuts[j]), int(cuts[j + 1])
        out[j] = srt[min(a, n - 1)] if b <= a else srt[a:b].mean(axis=0)
    return out


def _near_any(c, pal) -> bool:
    return any(sum((a - b) ** 2 for a, b in zip(c, p)) < 0.002 for p in pal)


def build_palette(tile: np.ndarray, pixels: np.ndarray) -> list[tuple]:
    pal = [clamp_rgb(tile.mean(axis=(0, 1)))]
    for k in (2, 3, 4):
        for c in palette_means(pixels, k):
            ct = clamp_rgb(c)
            if not _near_any(ct, pal):
                pal.append(ct)
    return pal


def side_means(tile: np.ndarray, lines: np.ndarray) -> np.ndarray:
    """Mean colour on each side (side >= 0, side < 0) of each line, integer pixel
    coordinates, tile mean for an empty side (``_split_by_lines_batched``,
    src/weft/encoder.py:343-400)."""
    h, w, _ = tile.shape
    n = lines.shape[0]
    if n == 0:
        return np.empty((0, 2, 3), dtype=np.float32)
    ys, xs = _int_grid(h, w)
    x0, y0, x1, y1 = (lines[:, i, None, None] for i in range(4))
    am = ((xs - x0) * (y1 - y0) - (ys - y0) * (x1 - x0) >= 0).astype(np.float32)
    bm = 1.0 - am
    ac, bc = am.sum(axis=(1, 2)), bm.sum(axis=(1, 2))
    a_col = np.einsum("nhw,hwc->nc", am, tile) / np.maximum(ac, 1.0)[:, None]
    b_col = np.einsum("nhw,hwc->nc", bm, tile) / np.maximum(bc, 1.0)[:, None]
    fb = tile.mean(axis=(0, 1))
    a_col[ac == 0] = fb
    b_col[bc == 0] = fb
    return np.stack([a_col, b_col], axis=1).astype(np.float32, copy=False)


def side_means_one(tile: np.ndarray, x0, y0, x1, y1):
    """Single-line form with boolean masks (``_split_by_line``, src/weft/encoder.py:322-340)."""
    h, w, _ = tile.shape
    ys, xs = _int_grid(h, w)
    am = (xs - x0) * (y1 - y0) - (ys - y0) * (x1 - x0) >= 0
    bm = ~am
    ca = tile[am].mean(axis=0) if np.any(am) else tile.mean(axis=(0, 1))
    cb = tile[bm].mean(axis=0) if np.any(bm) else tile.mean(axis=(0, 1))
    return tuple(float(v) for v in ca), tuple(float(v) for v in cb)


# ----------------------------------------------------------------------------- de-duplication
def _q(v: float, s: float) -> int:
    return int(v * s + 0.5)


def dedup(cands: list[Cand]) -> list[Cand]:
    """Keep the first candidate of each coarse key: geometry x4, colours x64, alpha x32 (each
    ``int(v * s + 0.5)`` as ``_q``, written out inline: this loop runs over every candidate)."""
    seen, out = set(), []
    for c in cands:
        c0 = c.color0
        key = (c.kind, tuple([int(g * 4 + 0.5) for g in c.geom]), int(c0[0] * 64 + 0.5), int(c0[1] * 64 + 0.5),
               int(c0[2] * 64 + 0.5), int(c.alpha * 32 + 0.5))
        if c.kind == 1:
            c1 = c.color1
            key += (int(c1[0] * 64 + 0.5), int(c1[1] * 64 + 0.5), int(c1[2] * 64 + 0.5))
        if key not in seen:
            seen.add(key)
            out.append(c)
    return out


# ----------------------------------------------------------------------------- edge-driven pool
def sobel(tile: np.ndarray, atan2: str = "numpy"):
    """3x3 Sobel magnitude and orientation in [0, pi) with zero borders
    (``_sobel_edges``, src/weft/edge_analysis.py:17-41).  The reference's convolution reads
    ``lum[y-1, x-1]`` for every tap (its slices are offset), so interior gradients cancel to
    rounding residue and the values are small integer multiples of one luminance; their angles
    sit on the orientation histogram's bin edges, where the last bit of the float32 arctan2
    decides the bin.  ``atan2="numpy"`` uses numpy's float32 arctan2 (the reference; its last
    bit depends on the host CPU's SIMD path), ``"rounded"`` the float64 arctan2 rounded to
    float32, which does not (the device generator's rule)."""
    lum = luminance(tile)
    h, w = lum.shape
    kx = np.array([[-1, 0, 1], [-2, 0, 2], [-1, 0, 1]], dtype=np.float32)
    ky = np.array([[-1, -2, -1], [0, 0, 0], [1, 2, 1]], dtype=np.float32)
    gx = np.zeros_like(lum)
    gy = np.zeros_like(lum)
    for dy in range(3):
        for dx in range(3):
            src = lum[max(0, dy - 1):h - 1 + dy, max(0, dx - 1):w - 1 + dx]
            ty, tx = max(1, dy), max(1, dx)
            dst = gx[ty:min(h, h - 1 + dy), tx:min(w, w - 1 + dx)]
            sh, sw = min(src.shape[0], dst.shape[0]), min(src.shape[1], dst.shape[1])
            gx[ty:ty + sh, tx:tx + sw] += kx[dy, dx] * src[:sh, :sw]
            gy[ty:ty + sh, tx:tx + sw] += ky[dy, dx] * src[:sh, :sw]
    if atan2 == "rounded":
        ang = np.arctan2(gy.astype(np.float64), gx.astype(np.float64)).astype(np.float32)
    else:
        ang = np.arctan2(gy, gx)
    return np.sqrt(gx * gx + gy * gy), ang % np.pi, lum


def dominant_orientations(angle: np.ndarray, mag: np.ndarray, n_bins: int = 12) -> list[float]:
    edges = np.linspace(0, np.pi, n_bins + 1)
    fa, fm = angle.ravel(), mag.ravel()
    hist = np.zeros(n_bins, dtype=np.float32)
    for i in range(n_bins):
        hist[i] = float(np.sum(fm[(fa >= edges[i]) & (fa < edges[i + 1])]))
    if hist.max() < 1e-6:
        return [0.0, np.pi / 4, np.pi / 2, 3 * np.pi / 4]
    thr = hist.max() * 0.2
    peaks = [float((edges[i] + edges[i + 1]) / 2.0) for i in range(n_bins) if hist[i] >= thr]
    return peaks if peaks else [float(edges[np.argmax(hist)] + np.pi / (2 * n_bins))]


def edge_points(mag: np.ndarray, pct: float = 60.0) -> list[tuple[float, float]]:
    thr = float(np.percentile(mag, pct))
    if thr < 1e-6:
        return []
    ys, xs = np.where(mag >= thr)
    return [(float(x), float(y)) for x, y in zip(xs, ys)]


def pca_segment(points):
    if len(points) < 2:
        return None
    pts = np.array(points, dtype=np.float32)
    cx, cy = pts.mean(axis=0)
    cen = pts - np.array([cx, cy])
    _, vecs = np.linalg.eigh(cen.T @ cen)
    d = vecs[:, 1]
    proj = cen @ d
    lo, hi = float(proj.min()), float(proj.max())
    return (cx + d[0] * lo, cy + d[1] * lo, cx + d[0] * hi, cy + d[1] * hi)


def cluster_points(points, n_clusters: int = 4):
    """Lloyd k-means on edge points, seeds from default_rng(42), <= 15 iterations."""
    if len(points) <= n_clusters:
        return [points] if points else []
    pts = np.array(points, dtype=np.float32)
    centers = pts[np.random.default_rng(42).choice(len(pts), n_clusters, replace=False)].copy()
    for _ in range(15):
        labels = np.argmin(np.sum((pts[:, None, :] - centers[None, :, :]) ** 2, axis=2), axis=1)
        new = centers.copy()
        for j in range(n_clusters):
            m = labels == j
            if m.any():
                new[j] = pts[m].mean(axis=0)
        if np.allclose(new, centers, atol=0.1):
            break
        centers = new
    groups = [[] for _ in range(n_clusters)]
    for i, lab in enumerate(labels):
        groups[lab].append(points[i])
    return [g for g in groups if len(g) >= 2]


def _kmeans3_triangles(tile, pixels, wf, hf, alphas, clamp_geom):
    h, w = tile.shape[:2]
    km3 = palette_means(pixels, 3)
    labels = np.argmin(np.sum((pixels[:, None, :] - km3[None, :, :]) ** 2, axis=2), axis=1).reshape(h, w)
    out = []
    for lab in range(3):
        ys, xs = np.where(labels == lab)
        if len(ys) < 3:
            continue
        i0, i1 = np.argmin(xs), np.argmax(xs)
        cx, cy = float(np.mean(xs)), float(np.mean(ys))
        g = (float(xs[i0]), float(ys[i0]), float(xs[i1]), float(ys[i1]), cx, cy)
        if clamp_geom:
            g = tuple(max(0.0, min(wf if j % 2 == 0 else hf, v)) for j, v in enumerate(g))
        col = clamp_rgb(km3[lab])
        out += [Cand(4, g, col, None, a) for a in alphas]
    return out


def edge_candidates(tile: np.ndarray, quality: int = 75, kinds=None, atan2: str = "numpy") -> list[Cand]:
    """The edge-driven pool; ``kinds`` (a set) skips the generators of other kinds, which leaves the
    remaining candidates, their values and their order unchanged; ``atan2`` as for ``sobel``."""
    return dedup(_edge_raw(tile, quality, kinds, atan2))


def _edge_raw(tile: np.ndarray, quality: int, kinds, atan2: str = "numpy") -> list[Cand]:
    want = (lambda k: True) if kinds is None else (lambda k: k in kinds)
    h, w = tile.shape[:2]
    hf, wf = float(h - 1), float(w - 1)
    mag, angle, _ = sobel(tile, atan2)
    pixels = tile.reshape(-1, 3).astype(np.float32)
    avg = clamp_rgb(tile.mean(axis=(0, 1)))
    out: list[Cand] = []
    for col in build_palette(tile, pixels):
        out += [Cand(0, (), col, None, a) for a in (1.0, 0.7, 0.4, 0.2)]
    qh, qw = h // 2, w // 2
    for r in range(2):
        for c in range(2):
            qc = clamp_rgb(tile[r * qh:(r + 1) * qh, c * qw:(c + 1) * qw].mean(axis=(0, 1)))
            out += [Cand(0, (), qc, None, a) for a in (0.5, 0.3)]

    ys, xs = _int_grid(h, w)
    cx, cy = wf * 0.5, hf * 0.5
    for th in dominant_orientations(angle, mag):
        nx, ny = -math.sin(th), math.cos(th)
        x0, y0, x1, y1 = cx - nx * wf * 0.6, cy - ny * hf * 0.6, cx + nx * wf * 0.6, cy + ny * hf * 0.6
        am = (xs - x0) * (y1 - y0) - (ys - y0) * (x1 - x0) >= 0
        bm = ~am
        c0 = clamp_rgb(tile[am].mean(axis=0)) if am.any() else avg
        c1 = clamp_rgb(tile[bm].mean(axis=0)) if bm.any() else avg
        out += [Cand(1, (x0, y0, x1, y1), c0, c1, a) for a in (1.0, 0.7, 0.4)]
        for f in (0.25, 0.75):
            ox, oy = cx + nx * wf * (f - 0.5), cy + ny * hf * (f - 0.5)
            out.append(Cand(1, (ox - nx * wf * 0.4, oy - ny * hf * 0.4, ox + nx * wf * 0.4, oy + ny * hf * 0.4),
                            c0, c1, 0.5))

    pts = edge_points(mag, 60.0) if (want(2) or want(3)) else []
    if pts:
        groups = cluster_points(pts, min(6, max(2, len(pts) // 4)))
        base_alpha = min(1.0, 0.25 + float(np.mean(mag)) * 3.0)
        em = mag >= float(np.percentile(mag, 75))
        edge_col = clamp_rgb(tile[em].mean(axis=0)) if em.any() else avg
        for grp in groups:
            seg = pca_segment(grp)
            if seg is None:
                continue
            lx0, ly0 = max(0.0, min(wf, seg[0])), max(0.0, min(hf, seg[1]))
            lx1, ly1 = max(0.0, min(wf, seg[2])), max(0.0, min(hf, seg[3]))
            mx = int(max(0, min(w - 1, round((lx0 + lx1) / 2))))
            my = int(max(0, min(h - 1, round((ly0 + ly1) / 2))))
            lc = clamp_rgb(tile[my, mx])
            for t in (0.4, 0.8, 1.5, 2.5):
                out += [Cand(2, (lx0, ly0, lx1, ly1, t), col, None, base_alpha) for col in (lc, edge_col)]
        if len(pts) >= 6:
            for grp in groups:
                if len(grp) < 3:
                    continue
                p = np.array(grp, dtype=np.float32)
                mcx, mcy = p.mean(axis=0)
                cen = p - np.array([mcx, mcy])
                _, vecs = np.linalg.eigh(cen.T @ cen)
                srt = p[np.argsort(cen @ vecs[:, 1])]
                a, b, mid = srt[0], srt[-1], srt[len(srt) // 2]
                ctrl = 2 * mid - (a + b) / 2
                g = (max(0.0, min(wf, float(a[0]))), max(0.0, min(hf, float(a[1]))),
                     max(0.0, min(wf, float(ctrl[0]))), max(0.0, min(hf, float(ctrl[1]))),
                     max(0.0, min(wf, float(b[0]))), max(0.0, min(hf, float(b[1]))))
                col = clamp_rgb(tile[int(max(0, min(h - 1, round(float(mid[1]))))),
                                     int(max(0, min(w - 1, round(float(mid[0])))))])
                out += [Cand(3, g + (t,), col, None, base_alpha) for t in (0.5, 1.0, 2.0)]
    if quality >= 60 and want(4):
        out += _kmeans3_triangles(tile, pixels, wf, hf, (0.6, 0.3), clamp_geom=True)
    return out if kinds is None else [c for c in out if c.kind in kinds]


# ----------------------------------------------------------------------------- template pool
def template_candidates(tile: np.ndarray, quality: int = 75, kinds=None) -> list[Cand]:
    """The template pool; ``kinds`` as for ``edge_candidates``."""
    return dedup(_template_raw(tile, quality, kinds))


def _template_raw(tile: np.ndarray, quality: int, kinds) -> list[Cand]:
    want = (lambda k: True) if kinds is None else (lambda k: k in kinds)
    h, w, _ = tile.shape
    hf, wf = float(h - 1), float(w - 1)
    lum = luminance(tile)
    pixels = tile.reshape(-1, 3).astype(np.float32)
    gy, gx = np.gradient(lum)
    mag = np.sqrt(gx * gx + gy * gy)
    avg_mag = float(np.mean(mag))
    gmx, gmy = float(np.mean(gx)), float(np.mean(gy))
    gnorm = math.sqrt(gmx * gmx + gmy * gmy)
    out: list[Cand] = []

    avg = clamp_rgb(tile.mean(axis=(0, 1)))
    pal = build_palette(tile, pixels)
    p25, p75 = float(np.percentile(lum, 25)), float(np.percentile(lum, 75))
    bm, dm = lum > p75, lum < p25
    bright = clamp_rgb(tile[bm].mean(axis=0)) if np.any(bm) else avg
    dark = clamp_rgb(tile[dm].mean(axis=0)) if np.any(dm) else avg
    em = mag >= float(np.percentile(mag, 75))
    edge_col = clamp_rgb(tile[em].mean(axis=0)) if np.any(em) else avg
    for extra in (bright, dark, edge_col):
        if not _near_any(extra, pal):
            pal.append(extra)
    base_alpha = min(1.0, 0.25 + avg_mag * 3.0)

    for col in pal:
        out += [Cand(0, (), col, None, a) for a in (1.0, 0.7, 0.4, 0.2)]
    qh, qw = h // 2, w // 2
    for r in range(2):
        for c in range(2):
            qc = clamp_rgb(tile[r * qh:(r + 1) * qh, c * qw:(c + 1) * qw].mean(axis=(0, 1)))
            out += [Cand(0, (), qc, None, a) for a in (0.5, 0.3)]
    sh, sw = h // 4, w // 4
    for r in range(4):
        for c in range(4):
            out.append(Cand(0, (), clamp_rgb(tile[r * sh:(r + 1) * sh, c * sw:(c + 1) * sw].mean(axis=(0, 1))),
                            None, 0.25))

    n_ang = 16 if quality >= 80 else 12 if quality >= 50 else 8
    specs = []
    for ang in np.linspace(0, math.pi, n_ang, endpoint=False):
        vx, vy = math.cos(ang), math.sin(ang)
        cx, cy = wf * 0.5, hf * 0.5
        specs.append((cx - vx * wf * 0.6, cy - vy * hf * 0.6, cx + vx * wf * 0.6, cy + vy * hf * 0.6, True))
    for ox, oy in ((0.25, 0.25), (0.75, 0.25), (0.25, 0.75), (0.75, 0.75), (0.5, 0.25), (0.5, 0.75)):
        for ang in np.linspace(0, math.pi, 6, endpoint=False):
            vx, vy = math.cos(ang), math.sin(ang)
            cx, cy = wf * ox, hf * oy
            specs.append((cx - vx * wf * 0.4, cy - vy * hf * 0.4, cx + vx * wf * 0.4, cy + vy * hf * 0.4, False))
    cols = side_means(tile, np.array([s[:4] for s in specs], dtype=np.float32))
    for (x0, y0, x1, y1, centre), (c0, c1) in zip(specs, cols.tolist()):
        c0, c1 = tuple(c0), tuple(c1)  # float32 -> Python float, exact
        for a in ((1.0, 0.7, 0.4) if centre else (0.5,)):
            out.append(Cand(1, (x0, y0, x1, y1), c0, c1, a))

    thicks = (0.4, 0.8, 1.2, 2.0, 3.0)
    if want(2):
        for t in thicks:
            for f in (0.0, 0.25, 0.5, 0.75, 1.0):
                out.append(Cand(2, (wf * f, 0, wf * f, hf, t), edge_col, None, base_alpha))
                out.append(Cand(2, (0, hf * f, wf, hf * f, t), edge_col, None, base_alpha))
            for col in (edge_col, bright, dark):
                out.append(Cand(2, (0, 0, wf, hf, t), col, None, base_alpha))
                out.append(Cand(2, (0, hf, wf, 0, t), col, None, base_alpha))
        if gnorm > 1e-4:
            lx, ly = -gmy / (gnorm + 1e-8), gmx / (gnorm + 1e-8)
            cx, cy = wf * 0.5, hf * 0.5
            g = (cx - lx * wf * 0.7, cy - ly * hf * 0.7, cx + lx * wf * 0.7, cy + ly * hf * 0.7)
            for t in thicks:
                out += [Cand(2, g + (t,), col, None, base_alpha) for col in (edge_col, bright)]

    fr = (0.25, 0.5, 0.75)
    if want(3):
        for fy in fr:
            for fx in fr:
                out += [Cand(3, (0, hf * 0.5, wf * fx, hf * fy, wf, hf * 0.5, t), edge_col, None, base_alpha)
                        for t in (0.5, 1.0, 2.0)]
        for fx in fr:
            for fy in fr:
                out += [Cand(3, (wf * 0.5, 0, wf * fx, hf * fy, wf * 0.5, hf, t), edge_col, None, base_alpha)
                        for t in (0.5, 1.0)]

    if want(4):
        corners = [(0.0, 0.0), (wf, 0.0), (wf, hf), (0.0, hf)]
        for i in range(4):
            v0, v1 = corners[i], corners[(i + 1) % 4]
            g = (v0[0], v0[1], v1[0], v1[1], wf * 0.5, hf * 0.5)
            for col in pal[:3]:
                out += [Cand(4, g, col, None, a) for a in (0.6, 0.3)]
        for gv in ((0, 0, wf, 0, wf, hf), (0, 0, wf, hf, 0, hf), (0, 0, wf, 0, 0, hf), (wf, 0, wf, hf, 0, hf)):
            out += [Cand(4, tuple(float(v) for v in gv), avg, None, a) for a in (0.5, 0.3)]
        flat = lum.reshape(-1)
        n_pk = min(6, len(flat))
        for idx in (np.argpartition(flat, -n_pk)[-n_pk:], np.argpartition(flat, n_pk)[:n_pk]):
            py, px = np.unravel_index(idx, lum.shape)
            if n_pk >= 3:
                for i in range(min(n_pk - 2, 4)):
                    g = (float(px[i]), float(py[i]), float(px[i + 1]), float(py[i + 1]), float(px[i + 2]),
                         float(py[i + 2]))
                    out.append(Cand(4, g, clamp_rgb(tile[py[i:i + 3], px[i:i + 3]].mean(axis=0)), None, 0.5))
        if quality >= 80:
            out += _kmeans3_triangles(tile, pixels, wf, hf, (0.5, 0.3), clamp_geom=False)
    return out if kinds is None else [c for c in out if c.kind in kinds]


def tile_candidates(tile: np.ndarray, quality: int = 75, kinds=None, atan2: str = "numpy") -> list[Cand]:
    """The tile's initial pool: edge-driven then template candidates, de-duplicated.  With ``kinds``
    only those kinds are generated: the result is the full pool filtered to them, in pool order
    (the de-duplication key starts with the kind, so other kinds never shadow a candidate).
    ``atan2`` chooses the float32 arctan2 of the Sobel orientations (see ``sobel``)."""
    kinds = None if kinds is None else frozenset(int(k) for k in kinds)
    # one de-duplication of the concatenation keeps the same first occurrences as de-duplicating
    # each pool first
    return dedup(_edge_raw(tile, quality, kinds, atan2) + _template_raw(tile, quality, kinds))


# ----------------------------------------------------------------------------- re-seeding
def residual_candidates(tile: np.ndarray, pred: np.ndarray, quality: int = 75) -> list[Cand]:
    """Candidates aimed at the high-error region of ``tile - pred``."""
    h, w, _ = tile.shape
    hf, wf = float(h - 1), float(w - 1)
    err = tile - pred
    el = np.abs(err).mean(axis=2)
    hi = el >= float(np.percentile(el, 60))
    if not np.any(hi):
        return []
    hi_col = clamp_rgb(np.clip(tile[hi].mean(axis=0), 0, 1))
    corr_col = clamp_rgb(np.clip(pred[hi].mean(axis=0) + err[hi].mean(axis=0), 0, 1))
    out: list[Cand] = []
    for col in (hi_col, corr_col, hi_col):
        out += [Cand(0, (), col, None, a) for a in (0.6, 0.4, 0.25, 0.15, 0.08)]
    qh, qw = h // 2, w // 2
    for r in range(2):
        for c in range(2):
            qm = hi[r * qh:(r + 1) * qh, c * qw:(c + 1) * qw]
            if qm.any():
                qcol = clamp_rgb(np.clip(tile[r * qh:(r + 1) * qh, c * qw:(c + 1) * qw][qm].mean(axis=0), 0, 1))
                out += [Cand(0, (), qcol, None, a) for a in (0.35, 0.2, 0.1)]
    ey, ex = np.gradient(el)
    mx, my = float(np.mean(ex)), float(np.mean(ey))
    nrm = math.sqrt(mx * mx + my * my) + 1e-8
    vx, vy = mx / nrm, my / nrm
    for off in (0.5, 0.3, 0.7):
        cx, cy = wf * off, hf * off
        g = (cx - vx * wf * 0.6, cy - vy * hf * 0.6, cx + vx * wf * 0.6, cy + vy * hf * 0.6)
        c0, c1 = side_means_one(tile, *g)
        out += [Cand(1, g, c0, c1, a) for a in (0.5, 0.3, 0.15)]
    cx, cy = wf * 0.5, hf * 0.5
    g = (cx + vy * wf * 0.6, cy - vx * hf * 0.6, cx - vy * wf * 0.6, cy + vx * hf * 0.6)
    c0, c1 = side_means_one(tile, *g)
    out += [Cand(1, g, c0, c1, a) for a in (0.4, 0.2)]

    ys, xs = np.where(hi)
    ecx, ecy = float(np.mean(xs)), float(np.mean(ys))
    for t in (0.3, 0.6, 1.0, 1.5, 2.5):
        for col in (hi_col, hi_col):
            for a in (0.5, 0.3, 0.15):
                out.append(Cand(2, (ecx, 0, ecx, hf, t), col, None, a))
                out.append(Cand(2, (0, ecy, wf, ecy, t), col, None, a))
    for t in (0.5, 1.0):
        out.append(Cand(2, (0, 0, wf, hf, t), hi_col, None, 0.25))
        out.append(Cand(2, (0, hf, wf, 0, t), hi_col, None, 0.25))
    if len(xs) >= 6:
        order = np.argsort(xs)
        p0 = (float(xs[order[0]]), float(ys[order[0]]))
        pm = (float(xs[order[len(order) // 2]]), float(ys[order[len(order) // 2]]))
        p1 = (float(xs[order[-1]]), float(ys[order[-1]]))
        ctrl = (max(0.0, min(wf, 2 * pm[0] - (p0[0] + p1[0]) / 2)), max(0.0, min(hf, 2 * pm[1] - (p0[1] + p1[1]) / 2)))
        out += [Cand(3, (p0[0], p0[1], ctrl[0], ctrl[1], p1[0], p1[1], t), hi_col, None, 0.3) for t in (0.5, 1.0, 2.0)]
    if len(xs) >= 3:
        ix0, ix1 = np.argmin(xs), np.argmax(xs)
        iy0, iy1 = np.argmin(ys), np.argmax(ys)
        g1 = (float(xs[ix0]), float(ys[ix0]), float(xs[ix1]), float(ys[ix1]), ecx, ecy)
        g2 = (float(xs[ix0]), float(ys[iy0]), float(xs[ix1]), float(ys[iy1]), ecx, ecy)
        for g in (g1, g2):
            for a in (0.4, 0.2, 0.1):
                out += [Cand(4, g, hi_col, None, a), Cand(4, g, hi_col, None, a)]
    return dedup(out)
