"""The decoder's raster branch on the GPU (host side): DCT residual layer and u8 BILINEAR resize.

When a file carries a BLOCK_DCT, the reference decoder renders the primitive walk at the
encoded size, adds the per-tile inverse-DCT residual and clips (src/weft/decoder.py:477-507,
src/weft/dct_residual.py:727-783); if the requested size differs from the encoded one it then
truncates to u8, resizes with Pillow's BILINEAR filter and divides by 255
(src/weft/decoder.py:514-518).

Here the host only parses the block and turns the presence mask, per-tile scales and the
coefficient layout (tile-major, or band-major zigzag, src/weft/dct_residual.py:221-296) into
one 64-byte descriptor per tile holding each channel's coefficient base and stride; the
gather, dequantization, inverse DCT, colour transform, add and clip run in
``weftk_dct_apply``, the resize in ``weftk_raster_resize``.  Errors follow the reference's:
a malformed block raises ``ValueError``.
"""

from __future__ import annotations

import ctypes
import struct
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import DCT_TILE_DTYPE

_HEADERS = {5: "<BBBBffHIII", 4: "<BBBBffHII", 3: "<BBffHII", 2: "<BBffHI"}


@dataclass
class DctBlock:
    """A parsed BLOCK_DCT (format versions 2-5, src/weft/bitstream.py:520-703)."""

    coeffs: np.ndarray      # int16
    quant_step: float
    channels: int
    freq_alpha: float
    chroma_mode: int
    presence_bitmask: bytes
    n_tiles: int
    layout: int
    scales_u8: bytes


def unpack_dct(blob: bytes) -> DctBlock:
    """Parse BLOCK_DCT bytes; raises ``ValueError`` on a truncated or inconsistent block."""
    if len(blob) < 1:
        raise ValueError("truncated DCT block header")
    version = blob[0]
    fmt = _HEADERS.get(version)
    if fmt is None:
        raise ValueError(f"unsupported DCT block version {version}")
    hs = struct.calcsize(fmt)
    if len(blob) < hs:
        raise ValueError(f"truncated DCT v{version} block header")
    f = struct.unpack_from(fmt, blob, 0)
    n_scales = 0
    if version >= 4:
        chroma, layout, step, alpha, channels, n_tiles, n_coeffs = f[1], f[2], f[4], f[5], f[6], f[7], f[8]
        if version == 5:
            n_scales = f[9]
    elif version == 3:
        chroma, step, alpha, channels, n_tiles, n_coeffs = f[1], f[2], f[3], f[4], f[5], f[6]
        layout = 0
    else:
        chroma, step, alpha, channels, n_coeffs = f[1], f[2], f[3], f[4], f[5]
        layout, n_tiles = 0, 0
    mask_len = (n_tiles + 7) // 8
    expected = hs + mask_len + n_scales + 2 * n_coeffs
    if len(blob) != expected:
        raise ValueError(f"DCT v{version} block size mismatch: got {len(blob)}, expected {expected}")
    off = hs + mask_len
    coeffs = np.frombuffer(blob, "<i2", n_coeffs, off + n_scales).astype(np.int16)
    return DctBlock(coeffs, float(step), int(channels), float(alpha), int(chroma), bytes(blob[hs:off]),
                    int(n_tiles), int(layout), bytes(blob[off:off + n_scales]))


def tile_scale(u: int) -> float:
    """Per-tile quant-step factor of a u8 scale: 2 ** (-2 + 4 u / 255) (src/weft/dct_residual.py:393-397)."""
    return float(2.0 ** (-2.0 + (max(0, min(255, int(u))) / 255.0) * 4.0))


def _bits(mask: bytes, n: int) -> np.ndarray:
    if len(mask) * 8 < n:
        raise ValueError(f"presence bitmask of {len(mask)} bytes is too short for {n} tiles")
    b = np.unpackbits(np.frombuffer(mask, np.uint8), bitorder="little")
    return b[:n].astype(bool)


def _channel_sides(size: np.ndarray, chroma_mode: int) -> np.ndarray:
    """(n, 3) block side per tile and channel."""
    half = size // 2 if chroma_mode == 2 else size
    return np.stack([size, half, half], axis=1)


def tile_table(block: DctBlock, quad_tiles, width: int, height: int, scales=None) -> np.ndarray:
    """Descriptors (``DCT_TILE_DTYPE``) of the tiles that carry coefficients and touch the image,
    sorted by tile side.

    ``quad_tiles``: (x, y, size) per tile in quadtree order, the order the coefficient stream
    follows.  ``scales``: per-present-tile quant-step factors as floats, instead of the block's u8
    scales (the reference's ``per_tile_scales`` argument)."""
    if block.chroma_mode not in (0, 1, 2):
        raise ValueError(f"bad chroma_mode: {block.chroma_mode}")
    if block.layout not in (0, 1):
        raise ValueError(f"bad DCT layout: {block.layout}")
    if block.channels != 3:
        raise ValueError(f"DCT residual with {block.channels} channels: only 3 are decoded")
    qt = np.asarray([tuple(q) for q in quad_tiles], np.int64).reshape(-1, 3)
    n = len(qt)
    # presence: the apply step reads the mask over the tile list (src/weft/dct_residual.py:754-757)
    present = _bits(block.presence_bitmask, n) if len(block.presence_bitmask) > 0 else np.ones(n, bool)
    if block.layout == 1 and not (block.n_tiles > 0 and len(block.presence_bitmask) > 0):
        present = np.ones(n, bool)
    elif block.layout == 1 and block.n_tiles != n:
        raise ValueError(f"presence mask covers {block.n_tiles} tiles, the file has {n}")
    tiles = qt[present]
    sizes = tiles[:, 2]
    m = len(tiles)
    if m and (np.any(sizes < 4) or np.any(sizes > 64) or np.any(sizes & (sizes - 1))):
        raise ValueError("DCT tiles must have a power-of-two side in 4..64")
    if scales is None and block.scales_u8:
        scales = [tile_scale(u) for u in block.scales_u8]
    if scales is not None:
        if len(scales) != m:
            raise ValueError(f"per_tile_scales length {len(scales)} does not match tile_sizes length {m}")
        scale = np.asarray(scales, np.float64).reshape(m)
    else:
        scale = np.ones(m, np.float64)
    sides = _channel_sides(sizes, block.chroma_mode)           # (m, 3)
    counts = sides * sides
    base = np.zeros((m, 3), np.int64)
    stride = np.ones((m, 3), np.int64)
    if block.layout == 0:
        flat = np.cumsum(counts.reshape(-1))
        used = int(flat[-1]) if m else 0
        base = (flat - counts.reshape(-1)).reshape(m, 3)
        if used > block.coeffs.size:
            raise ValueError(f"tile-major coefficient buffer too short: needs {used}, got {block.coeffs.size}")
    else:
        pos = 0
        for s in sorted(set(int(v) for v in sizes)):
            members = np.flatnonzero(sizes == s)
            for c in range(3):
                nn = int(counts[members[0], c])
                base[members, c] = pos + np.arange(len(members))
                stride[members, c] = len(members)
                pos += nn * len(members)
        if pos != block.coeffs.size:
            raise ValueError(f"band-major coefficient buffer size mismatch: used {pos}, got {block.coeffs.size}")
    d = np.zeros(m, DCT_TILE_DTYPE)
    d["x"], d["y"], d["size"] = tiles[:, 0], tiles[:, 1], sizes
    d["step_scale"] = scale
    d["coef_base"] = base
    d["coef_stride"] = stride
    keep = (d["x"] < width) & (d["y"] < height)
    d = d[keep]
    return d[np.argsort(d["size"], kind="stable")]


class DctLaunch:
    """A BLOCK_DCT bound to a tile list and an image size, with its descriptors and coefficients
    resident on the device; ``run`` enqueues the layer (one ``weftk_dct_apply`` launch per tile
    side, then the whole-image clip) without host synchronisation."""

    def __init__(self, block: DctBlock, quad_tiles, width: int, height: int, device: int = 0, scales=None):
        import torch

        self.block = block
        self.descs = tile_table(block, quad_tiles, width, height, scales)
        self.width, self.height = int(width), int(height)
        self.device = torch.device("cuda", device)
        self.lib = _lib.lib_for_device(device)
        c = self.block.coeffs if self.block.coeffs.size else np.zeros(1, np.int16)
        self.t_coeffs = torch.from_numpy(c).to(self.device)
        self.t_descs = torch.from_numpy(self.descs.view(np.uint8)).to(self.device) if len(self.descs) else None
        sizes = self.descs["size"]
        self.groups = [(int(v), int(np.searchsorted(sizes, v, "left")), int(np.searchsorted(sizes, v, "right")))
                       for v in np.unique(sizes)]

    @classmethod
    def from_payload(cls, payload: bytes, quad_tiles, width: int, height: int, device: int = 0) -> "DctLaunch":
        return cls(unpack_dct(payload), quad_tiles, width, height, device)

    @property
    def launches(self) -> int:
        return len(self.groups) + 1

    def flops(self) -> float:
        """Float64 operations of the two transform passes: 2 n^3 multiply-adds per n x n block."""
        n = _channel_sides(self.descs["size"].astype(np.int64), self.block.chroma_mode).astype(np.float64)
        return float(np.sum(4.0 * n ** 3))

    def run(self, image, stream: int, clip_all: bool = True) -> None:
        b = self.block
        for s, lo, hi in self.groups:
            _lib.check(self.lib.weftk_dct_apply(_lib.ptr(self.t_descs) + lo * DCT_TILE_DTYPE.itemsize, hi - lo,
                                                _lib.ptr(self.t_coeffs), int(b.coeffs.size), b.chroma_mode, b.layout,
                                                b.quant_step, b.freq_alpha, s, _lib.ptr(image), self.width,
                                                self.height, 0, stream), "weftk_dct_apply")
        if clip_all:
            _lib.check(self.lib.weftk_dct_apply(0, 0, 0, 0, b.chroma_mode, b.layout, b.quant_step, b.freq_alpha, 4,
                                                _lib.ptr(image), self.width, self.height, 1, stream),
                       "weftk_dct_apply")


def apply_dct(image, payload: bytes, quad_tiles, clip_all: bool = True):
    """Add a BLOCK_DCT's residual to ``image`` (torch float32 CUDA tensor, (h, w, 3)) in place and
    return it; ``clip_all`` clips the whole image to [0, 1] as the reference does."""
    import torch

    if image.dtype != torch.float32 or not image.is_cuda or image.dim() != 3 or image.shape[2] != 3:
        raise ValueError("image must be a float32 (h, w, 3) CUDA tensor")
    image = image.contiguous() if not image.is_contiguous() else image
    h, w = int(image.shape[0]), int(image.shape[1])
    _run_checked(DctLaunch.from_payload(payload, quad_tiles, w, h, image.device.index), image, clip_all)
    return image


def _run_checked(layer: DctLaunch, image, clip_all: bool = True) -> None:
    import torch

    status = ctypes.c_int(0)
    layer.lib.weftk_device_status(ctypes.addressof(status))  # clear any earlier report
    layer.run(image, torch.cuda.current_stream(image.device).cuda_stream, clip_all)
    if len(layer.descs):
        _lib.check(layer.lib.weftk_device_status(ctypes.addressof(status)), "weftk_device_status")
        if status.value:
            raise ValueError("a DCT tile reads past its coefficient stream or has an unsupported side")


def apply_residual_to_image(recon, coeffs, quad_tiles, *, quant_step: float, channels: int = 3,
                            freq_alpha: float = 0.0, chroma_mode: int = 0, presence_bitmask: bytes | None = None,
                            per_tile_scales=None) -> np.ndarray:
    """Drop-in for the reference's ``apply_residual_to_image`` (src/weft/dct_residual.py:727-783), same
    arguments: ``recon`` (h, w, 3) host image, ``coeffs`` the tile-major int16 stream (the decoder has
    already undone a band layout), ``quad_tiles`` objects with ``x``, ``y``, ``size``.  Returns the
    float32 image with the residual added and clipped to [0, 1], computed on the current GPU."""
    import torch

    qt = [(int(q.x), int(q.y), int(q.size)) for q in quad_tiles]
    mask = bytes(presence_bitmask) if presence_bitmask else b""
    block = DctBlock(np.ascontiguousarray(coeffs, np.int16).reshape(-1), float(quant_step), int(channels),
                     float(freq_alpha), int(chroma_mode), mask, len(qt) if mask else 0, 0, b"")
    img = torch.from_numpy(np.ascontiguousarray(recon, np.float32)).cuda()
    if img.dim() != 3 or img.shape[2] != 3:
        raise ValueError("recon must be (h, w, 3)")
    h, w = int(img.shape[0]), int(img.shape[1])
    _run_checked(DctLaunch(block, qt, w, h, img.device.index, per_tile_scales), img)
    return img.cpu().numpy()


def resize_into(image, out, tmp, stream: int) -> None:
    """Enqueue ``weftk_raster_resize`` from ``image`` (h, w, 3) into ``out`` (H, W, 3) with the caller's
    u8 scratch ``tmp`` of h * W * 3 bytes."""
    h, w = int(image.shape[0]), int(image.shape[1])
    th, tw = int(out.shape[0]), int(out.shape[1])
    if tmp.numel() < h * tw * 3:
        raise ValueError("resize scratch too small")
    lib = _lib.lib_for_device(image.device.index)
    _lib.check(lib.weftk_raster_resize(_lib.ptr(image), w, h, _lib.ptr(out), tw, th, _lib.ptr(tmp), stream),
               "weftk_raster_resize")


def resize(image, target_w: int, target_h: int):
    """u8-truncate, Pillow-BILINEAR-resize and rescale a (h, w, 3) float32 CUDA tensor."""
    import torch

    h, w = int(image.shape[0]), int(image.shape[1])
    if (target_w, target_h) == (w, h):
        return image
    image = image.contiguous()
    out = torch.empty((target_h, target_w, 3), dtype=torch.float32, device=image.device)
    tmp = torch.empty(h * target_w * 3, dtype=torch.uint8, device=image.device)
    resize_into(image, out, tmp, torch.cuda.current_stream(image.device).cuda_stream)
    return out
