"""Numpy restatement of the reference's DCT residual decode and raster upscale (test oracle).

Follows ``src/weft/dct_residual.py`` (per-tile inverse DCT residual layer), the BLOCK_DCT
parser ``unpack_dct`` (``src/weft/bitstream.py:599-703``) and the decoder's raster branch
(``src/weft/decoder.py:477-518``): render at the encoded size, add the per-tile residual,
clip, and — only when the target size differs — truncate to u8 and resize with Pillow's
BILINEAR filter, then divide by 255.

The inverse DCT is written as the orthonormal DCT-III matrix product ``A.T @ X @ A`` in
float64 (the reference calls ``scipy.fft.idctn(type=2, norm="ortho")``, pinned at
scipy 1.15.3 by its lock file; the two agree to ~1e-16 before the float32 cast).  The
resize restates Pillow's ``ImagingResample`` for 8-bit images (``libImaging/Resample.c``,
Pillow 12.1.1 in the reference's lock file): a triangle filter of support 1 scaled by the
down-scale factor, weights normalised per output pixel and rounded to 22-bit fixed point,
a horizontal pass into an 8-bit intermediate, then a vertical pass.

TEST INFRASTRUCTURE ONLY: the product never imports this module.
"""

from __future__ import annotations

import math
import struct

import numpy as np

YCBCR_TO_RGB = np.array([[1.0, 0.0, 1.402], [1.0, -0.344136, -0.714136], [1.0, 1.772, 0.0]], np.float64)
CHROMA_QUANT_SCALE = 1.5
RESAMPLE_BITS = 22


def zigzag(n: int) -> np.ndarray:
    """Row-major flat index of the k-th zigzag coefficient of an n x n block: even
    anti-diagonals run bottom-left to top-right, odd ones top-right to bottom-left
    (src/weft/dct_residual.py:91-123)."""
    order = []
    for s in range(2 * n - 1):
        rows = range(max(0, s - n + 1), min(s, n - 1) + 1)
        for i in (reversed(rows) if s % 2 == 0 else rows):
            order.append(i * n + (s - i))
    return np.asarray(order, np.int64)


def channel_sizes(size: int, chroma_mode: int) -> list[int]:
    """Block side of each channel (src/weft/dct_residual.py:126-138)."""
    if chroma_mode in (0, 1):
        return [size] * 3
    if chroma_mode == 2:
        return [size, size // 2, size // 2]
    raise ValueError(f"bad chroma_mode: {chroma_mode}")


def unpack_dct(blob: bytes) -> dict:
    """BLOCK_DCT v2-v5 (src/weft/bitstream.py:599-703)."""
    if len(blob) < 1:
        raise ValueError("truncated DCT block header")
    v = blob[0]
    fmt = {5: "<BBBBffHIII", 4: "<BBBBffHII", 3: "<BBffHII", 2: "<BBffHI"}.get(v)
    if fmt is None:
        raise ValueError(f"unsupported DCT block version {v}")
    hs = struct.calcsize(fmt)
    if len(blob) < hs:
        raise ValueError(f"truncated DCT v{v} block header")
    f = struct.unpack_from(fmt, blob, 0)
    if v >= 4:
        _, chroma, layout, _, step, alpha, channels, n_tiles, n_coeffs = f[:9]
        n_scales = f[9] if v == 5 else 0
    elif v == 3:
        _, chroma, step, alpha, channels, n_tiles, n_coeffs = f
        layout, n_scales = 0, 0
    else:
        _, chroma, step, alpha, channels, n_coeffs = f
        layout, n_scales, n_tiles = 0, 0, 0
    mask_len = (n_tiles + 7) // 8
    if len(blob) != hs + mask_len + n_scales + 2 * n_coeffs:
        raise ValueError(f"DCT v{v} block size mismatch")
    off = hs
    mask = bytes(blob[off:off + mask_len])
    off += mask_len
    scales = bytes(blob[off:off + n_scales])
    off += n_scales
    coeffs = np.frombuffer(blob, "<i2", n_coeffs, off).copy()
    return {"coeffs": coeffs, "quant_step": float(step), "channels": int(channels), "freq_alpha": float(alpha),
            "chroma_mode": int(chroma), "mask": mask, "n_tiles": int(n_tiles), "layout": int(layout),
            "scales_u8": scales}


def presence(mask: bytes, n_tiles: int) -> list[bool]:
    """LSB-first presence bits (src/weft/dct_residual.py:704-710)."""
    return [bool(mask[i >> 3] & (1 << (i & 7))) for i in range(n_tiles)]


def permute_band_to_tile(coeffs: np.ndarray, sizes: list[int], chroma_mode: int) -> np.ndarray:
    """Band-major zigzag layout -> tile-major row-major layout (src/weft/dct_residual.py:221-296).

    Bands are the (tile size, channel) groups in sorted order; inside a band the value of
    member m at zigzag position z sits at ``z * n_members + m``."""
    base, cur = [], 0
    for s in sizes:
        offs = []
        for n in channel_sizes(s, chroma_mode):
            offs.append(cur)
            cur += n * n
        base.append(offs)
    out = np.empty(cur, np.int16)
    groups: dict[tuple[int, int], list[int]] = {}
    for t, s in enumerate(sizes):
        for c in range(3):
            groups.setdefault((s, c), []).append(t)
    pos = 0
    for (s, c) in sorted(groups):
        n = channel_sizes(s, chroma_mode)[c]
        members = groups[(s, c)]
        band = coeffs[pos:pos + n * n * len(members)].reshape(n * n, len(members))
        pos += n * n * len(members)
        zz = zigzag(n)
        for j, t in enumerate(members):
            blk = np.empty(n * n, np.int16)
            blk[zz] = band[:, j]
            out[base[t][c]:base[t][c] + n * n] = blk
    if pos != coeffs.size:
        raise ValueError(f"band-major coefficient buffer size mismatch: used {pos}, got {coeffs.size}")
    return out


def freq_weights(n: int, alpha: float) -> np.ndarray:
    """1 + alpha * (i + j) / (2 (n - 1)) (src/weft/dct_residual.py:299-327)."""
    if n == 1:
        return np.ones((1, 1))
    i, j = np.mgrid[0:n, 0:n].astype(np.float64)
    return 1.0 + alpha * ((i + j) / (2.0 * (n - 1)))


def tile_scale(u: int) -> float:
    """u8 -> 2 ** (-2 + 4 u / 255) (src/weft/dct_residual.py:393-397)."""
    return float(2.0 ** (-2.0 + (max(0, min(255, int(u))) / 255.0) * 4.0))


def idct_matrix(n: int) -> np.ndarray:
    """A[k, x] = c_k cos(pi (2x + 1) k / (2n)), c_0 = sqrt(1/n), c_k = sqrt(2/n): the orthonormal
    DCT-II basis, whose transpose is the inverse transform."""
    k = np.arange(n, dtype=np.float64)[:, None]
    x = np.arange(n, dtype=np.float64)[None, :]
    a = np.cos(np.pi * (2.0 * x + 1.0) * k / (2.0 * n)) * math.sqrt(2.0 / n)
    a[0, :] = math.sqrt(1.0 / n)
    return a


def dequant_idct(q: np.ndarray, step: float, alpha: float, scales) -> np.ndarray:
    """Dequantize a stack of (n, n) int16 blocks and inverse-DCT them to float32; ``scales`` is
    None or one per-tile factor per block (src/weft/dct_residual.py:513-547)."""
    n = q.shape[-1]
    grid = step * freq_weights(n, alpha) if alpha > 0 else np.full((n, n), step)
    grid = grid[None] if scales is None else grid[None] * np.asarray(scales, np.float64)[:, None, None]
    a = idct_matrix(n)
    return (a.T @ (q.astype(np.float64) * grid) @ a).astype(np.float32)


def decode_tile_residuals(coeffs, sizes, quant_step, channels=3, freq_alpha=0.0, chroma_mode=0,
                          per_tile_scales=None) -> list[np.ndarray]:
    """Per-tile (size, size, 3) float32 RGB residuals, tiles bucketed by size and each bucket
    transformed as one stack (src/weft/dct_residual.py:550-701)."""
    if chroma_mode not in (0, 1, 2):
        raise ValueError(f"bad chroma_mode: {chroma_mode}")
    sizes = [int(s) for s in sizes]
    if per_tile_scales is not None and len(per_tile_scales) != len(sizes):
        raise ValueError("per_tile_scales length does not match tile_sizes length")
    buckets: dict[int, tuple[list[int], list[list[np.ndarray]]]] = {}
    cur = 0
    for t, s in enumerate(sizes):
        idx, blocks = buckets.setdefault(s, ([], [[], [], []]))
        idx.append(t)
        for c, n in enumerate(channel_sizes(s, chroma_mode)):
            blocks[c].append(coeffs[cur:cur + n * n].reshape(n, n))
            cur += n * n
    out: list[np.ndarray] = [None] * len(sizes)  # type: ignore[list-item]
    for s, (idx, blocks) in buckets.items():
        sc = None if per_tile_scales is None else [float(per_tile_scales[t]) for t in idx]
        chans = []
        for c in range(3):
            st = quant_step if (chroma_mode == 0 or c == 0) else quant_step * CHROMA_QUANT_SCALE
            chans.append(dequant_idct(np.stack(blocks[c]), st, freq_alpha, sc))
        if chroma_mode == 0:
            rgb = np.stack(chans, axis=-1)
        else:
            y, cb, cr = chans
            if chroma_mode == 2:
                cb = np.repeat(np.repeat(cb, 2, axis=-2), 2, axis=-1)
                cr = np.repeat(np.repeat(cr, 2, axis=-2), 2, axis=-1)
            ycc = np.stack([y, cb, cr], axis=-1).astype(np.float64)
            rgb = (ycc @ YCBCR_TO_RGB.T).astype(np.float32)
        for j, t in enumerate(idx):
            out[t] = rgb[j]
    return out


def apply_residual_to_image(recon: np.ndarray, coeffs, quad_tiles, quant_step: float, channels: int = 3,
                            freq_alpha: float = 0.0, chroma_mode: int = 0, presence_bitmask: bytes | None = None,
                            per_tile_scales=None) -> np.ndarray:
    """recon + per-tile residual (cropped to the image), clipped to [0, 1]
    (src/weft/dct_residual.py:727-783).  ``quad_tiles``: (x, y, size) triples."""
    n = len(quad_tiles)
    pres = presence(presence_bitmask, n) if presence_bitmask else [True] * n
    tiles = [qt for qt, p in zip(quad_tiles, pres) if p]
    res = decode_tile_residuals(coeffs, [int(s) for _, _, s in tiles], quant_step, channels, freq_alpha,
                                chroma_mode, per_tile_scales)
    out = recon.copy()
    h, w = out.shape[:2]
    for (x0, y0, s), r in zip(tiles, res):
        x1, y1 = min(x0 + s, w), min(y0 + s, h)
        if x1 > x0 and y1 > y0:
            out[y0:y1, x0:x1] += r[:y1 - y0, :x1 - x0]
    return np.clip(out, 0.0, 1.0)


def apply_dct_block(image: np.ndarray, blob: bytes, quad_tiles) -> np.ndarray:
    """The decoder's DCT step: unpack, undo the band layout, apply
    (src/weft/decoder.py:477-507)."""
    d = unpack_dct(blob)
    coeffs = d["coeffs"]
    if d["layout"] == 1:
        pres = presence(d["mask"], d["n_tiles"]) if (d["n_tiles"] > 0 and d["mask"]) else [True] * len(quad_tiles)
        sizes = [int(s) for (_, _, s), p in zip(quad_tiles, pres) if p]
        coeffs = permute_band_to_tile(coeffs, sizes, d["chroma_mode"])
    scales = [tile_scale(b) for b in d["scales_u8"]] if d["scales_u8"] else None
    return apply_residual_to_image(image, coeffs, quad_tiles, d["quant_step"], d["channels"], d["freq_alpha"],
                                   d["chroma_mode"], d["mask"], scales)


def resample_coeffs(in_size: int, out_size: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Pillow's per-output (first tap, tap count, 22-bit weights) for BILINEAR
    (libImaging/Resample.c precompute_coeffs + normalize_coeffs_8bpc)."""
    scale = float(in_size) / out_size
    fscale = max(scale, 1.0)
    support = 1.0 * fscale
    ksize = int(math.ceil(support)) * 2 + 1
    first = np.zeros(out_size, np.int64)
    count = np.zeros(out_size, np.int64)
    kk = np.zeros((out_size, ksize), np.int64)
    for xx in range(out_size):
        center = (xx + 0.5) * scale
        xmin = max(int(center - support + 0.5), 0)
        xmax = min(int(center + support + 0.5), in_size) - xmin
        w = []
        for x in range(xmax):
            d = abs((x + xmin - center + 0.5) * (1.0 / fscale))
            w.append(1.0 - d if d < 1.0 else 0.0)
        ww = 0.0
        for v in w:
            ww += v
        for x, v in enumerate(w):
            v = v / ww if ww != 0.0 else v
            kk[xx, x] = int(-0.5 + v * (1 << RESAMPLE_BITS)) if v < 0 else int(0.5 + v * (1 << RESAMPLE_BITS))
        first[xx], count[xx] = xmin, xmax
    return first, count, kk


def _clip8(acc: np.ndarray) -> np.ndarray:
    return np.clip(acc >> RESAMPLE_BITS, 0, 255).astype(np.uint8)


def resize_bilinear_u8(u8: np.ndarray, out_w: int, out_h: int) -> np.ndarray:
    """``PIL.Image.fromarray(u8).resize((out_w, out_h), BILINEAR)`` for an (h, w, 3) u8 image:
    horizontal pass (skipped when the width is unchanged), then vertical pass (skipped when
    the height is unchanged), each rounding to 8 bits."""
    h, w = u8.shape[:2]
    img = u8
    if out_w != w:
        first, count, kk = resample_coeffs(w, out_w)
        acc = np.full((h, out_w, 3), 1 << (RESAMPLE_BITS - 1), np.int64)
        for k in range(kk.shape[1]):
            src = np.minimum(first + k, w - 1)
            wk = np.where(k < count, kk[:, k], 0)
            acc += img[:, src, :].astype(np.int64) * wk[None, :, None]
        img = _clip8(acc)
    if out_h != h:
        first, count, kk = resample_coeffs(h, out_h)
        acc = np.full((out_h, img.shape[1], 3), 1 << (RESAMPLE_BITS - 1), np.int64)
        for k in range(kk.shape[1]):
            src = np.minimum(first + k, h - 1)
            wk = np.where(k < count, kk[:, k], 0)
            acc += img[src, :, :].astype(np.int64) * wk[:, None, None]
        img = _clip8(acc)
    return img


def raster_finish(image: np.ndarray, target_w: int, target_h: int) -> np.ndarray:
    """Truncate to u8, Pillow BILINEAR resize, back to float32 / 255 (src/weft/decoder.py:514-518)."""
    h, w = image.shape[:2]
    if (target_w, target_h) == (w, h):
        return image
    u8 = np.clip(image * np.float32(255.0), 0.0, 255.0).astype(np.uint8)
    return resize_bilinear_u8(u8, target_w, target_h).astype(np.float32) / np.float32(255.0)
