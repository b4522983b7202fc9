"""The fit's front end on the device: from an sRGB u8 image to fitted tiles without host work
per pixel (host side of ``include/weftk_quadtree.h``).

``decompose_device`` is the variance-rule quadtree of ``quadtree.decompose(rule="variance")``
(src/weft/quadtree.py:42-91 with the batched workloads' split rule), ``extract_device`` the tile
extraction of ``quadtree.extract_tiles`` (src/weft/quadtree.py:94-108) with the sRGB decode of
``synth.srgb_u8_to_linear`` (src/weft/image_io.py:9-24), and ``refine_image`` the whole refined fit
of one image: quadtree, extraction, pool generation, init round, Adam steps and the wire-grid snap
on the GPU, one small host read (the tile list) in between.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .synth import srgb_u8_to_linear

_LUT: dict[int, torch.Tensor] = {}


def srgb_table(device) -> torch.Tensor:
    """The host's float32 sRGB decode of every u8 value (256 entries), on ``device``."""
    dev = torch.device(device)
    key = dev.index or 0
    if key not in _LUT:
        lut = srgb_u8_to_linear(np.arange(256, dtype=np.uint8).reshape(1, 256, 1)).reshape(256)
        _LUT[key] = torch.from_numpy(np.ascontiguousarray(lut, np.float32)).to(dev)
    return _LUT[key]


def decompose_device(img_u8: torch.Tensor, threshold: float = 100.0, min_tile: int = 8, max_tile: int = 64):
    """Quadtree of an (h, w, 3) uint8 device image: (tiles int32 (n, 3) device tensor of (x, y, side),
    n).  Reads the tile count back (one synchronisation)."""
    h, w = int(img_u8.shape[0]), int(img_u8.shape[1])
    dev = img_u8.device
    lib = _lib.lib_for_device(dev.index or 0)
    need = ctypes.c_int64(0)
    _lib.check(lib.weftk_quadtree_work_bytes(h, w, max_tile, min_tile, ctypes.addressof(need)),
               "weftk_quadtree_work_bytes")
    work = torch.empty(int(need.value), dtype=torch.uint8, device=dev)
    cap = ((h + max_tile - 1) // max_tile) * ((w + max_tile - 1) // max_tile) * (max_tile // min_tile) ** 2
    tiles = torch.empty((cap, 3), dtype=torch.int32, device=dev)
    n = torch.zeros(1, dtype=torch.int32, device=dev)
    img = img_u8.contiguous()
    _lib.check(lib.weftk_quadtree_variance(_lib.ptr(img), h, w, float(threshold), max_tile, min_tile,
                                           _lib.ptr(tiles), cap, _lib.ptr(n), _lib.ptr(work),
                                           torch.cuda.current_stream(dev).cuda_stream), "weftk_quadtree_variance")
    count = int(n.item())
    return tiles[:count], count


def extract_device(img_u8: torch.Tensor, tiles: torch.Tensor, sizes: np.ndarray):
    """Tile pixels of ``tiles`` (device (n, 3) int32, sides ``sizes`` on the host) as the fit's float4
    layout: (src4 (sum side^2, 4) float32, px_off int32 device tensor)."""
    dev = img_u8.device
    lib = _lib.lib_for_device(dev.index or 0)
    px = np.asarray(sizes, np.int64) ** 2
    px_off = torch.from_numpy(np.concatenate([[0], np.cumsum(px)[:-1]]).astype(np.int32)).to(dev)
    src4 = torch.empty((int(px.sum()), 4), dtype=torch.float32, device=dev)
    img = img_u8.contiguous()
    _lib.check(lib.weftk_extract_tiles(_lib.ptr(img), int(img.shape[0]), int(img.shape[1]),
                                       _lib.ptr(srgb_table(dev)), _lib.ptr(tiles), int(len(px)), _lib.ptr(px_off),
                                       _lib.ptr(src4), torch.cuda.current_stream(dev).cuda_stream),
               "weftk_extract_tiles")
    return src4, px_off


def refine_image_steps(u8: np.ndarray, quality: int = 75, cap: int = 16, steps: int = 10, lr: float = 1e-2,
                       threshold: float = 100.0, device: int = 0, timings: dict | None = None):
    """``refine_image`` driven one entry point at a time from Python (fresh fit objects per call):
    the same results, bit for bit.  ``timings``: a dict that receives the host wall milliseconds
    of each phase (the device is synchronised between phases, which the plain call does not do)."""
    import time

    from .pools import DeviceRefinedFit

    dev = torch.device("cuda", device)
    marks = []

    def mark(name):
        if timings is not None:
            torch.cuda.synchronize(dev)
            marks.append((name, time.perf_counter()))

    mark("start")
    img = torch.from_numpy(np.ascontiguousarray(u8, np.uint8)).to(dev, non_blocking=True)
    mark("h2d")
    tiles, n = decompose_device(img, threshold)
    mark("quadtree")
    tiles_h = tiles.cpu().numpy()
    sizes = tiles_h[:, 2].copy()
    mark("tiles_d2h")
    src4, _ = extract_device(img, tiles, sizes)
    mark("extract")
    drf = DeviceRefinedFit(src4, sizes, quality, caps=[cap] * n, steps=steps, lr=lr, use_graph=False,
                           autotune=False)
    mark("setup")
    rows = drf.run()
    mark("fit")
    out = tiles_h, rows.cpu().numpy(), drf.rf.kinds.cpu().numpy()
    mark("d2h")
    if timings is not None:
        for (_, a), (name, b) in zip(marks, marks[1:]):
            timings[name] = (b - a) * 1e3
        timings["total"] = (marks[-1][1] - marks[0][1]) * 1e3
    return out


class Refiner:
    """The refined fit of whole images through the native per-image pipeline
    (``weftk_refine_image``, include/weftk_pipeline.h): one call per image, a device workspace
    kept between calls (it grows to the largest image seen)."""

    def __init__(self, quality: int = 75, cap: int = 16, steps: int = 10, lr: float = 1e-2, threshold: float = 100.0,
                 device: int = 0, min_tile: int = 8, max_tile: int = 64):
        from . import rate
        from .fit import CHUNK
        from .pools import tables_for

        self.device = torch.device("cuda", device)
        self.lib = _lib.lib_for_device(device)
        self.tables = tables_for(quality, device)
        self.lut = srgb_table(self.device)
        p = _lib.WeftRefineParams()
        p.cap, p.steps, p.min_tile, p.max_tile = int(cap), int(steps), int(min_tile), int(max_tile)
        for i, cls in enumerate((8, 16, 32)):
            p.chunk[i] = int(CHUNK[cls])
            p.variant[i] = 0
        p.lr, p.beta1, p.beta2, p.eps = float(lr), 0.9, 0.999, 1e-8
        p.threshold = float(threshold)
        p.lam = float(rate.tile_lambda(quality))
        p.complex_threshold = float(rate.complexity_threshold(quality))
        p.tables = ctypes.addressof(self.tables.st)
        p.srgb_lut = _lib.ptr(self.lut)
        self.params = p
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.weftk_refiner_create(ctypes.addressof(p), ctypes.addressof(handle)),
                       "weftk_refiner_create")
        self.handle = handle
        self._cap_tiles = 0
        self._out = None

    def __call__(self, u8: np.ndarray):
        """(tiles int32 (n, 3) of (x, y, side), rows float32 (n, 16) on the wire grid, kinds int32 (n,))."""
        img = np.ascontiguousarray(u8, np.uint8)
        if img.ndim != 3 or img.shape[2] != 3:
            raise ValueError("expected an (h, w, 3) uint8 image")
        h, w = int(img.shape[0]), int(img.shape[1])
        p = self.params
        cap = (-(-h // p.max_tile)) * (-(-w // p.max_tile)) * (p.max_tile // p.min_tile) ** 2
        if self._out is None or self._cap_tiles < cap:
            # page-locked, so the results come back by DMA (the caller gets copies of them)
            self._out_t = (torch.empty((cap, 3), dtype=torch.int32, pin_memory=True),
                           torch.empty((cap, 16), dtype=torch.float32, pin_memory=True),
                           torch.empty(cap, dtype=torch.int32, pin_memory=True))
            self._out = tuple(t.numpy() for t in self._out_t)
            self._cap_tiles = cap
        tiles, rows, kinds = self._out
        n = ctypes.c_int(0)
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            _lib.check(self.lib.weftk_refine_image(self.handle, img.ctypes.data, h, w, tiles.ctypes.data,
                                                   rows.ctypes.data, kinds.ctypes.data, cap, ctypes.addressof(n),
                                                   stream), "weftk_refine_image")
        k = n.value
        return tiles[:k].copy(), rows[:k].copy(), kinds[:k].copy()

    def close(self) -> None:
        if getattr(self, "handle", None) and self.handle.value:
            self.lib.weftk_refiner_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_REFINERS: dict[tuple, Refiner] = {}


def refine_image(u8: np.ndarray, quality: int = 75, cap: int = 16, steps: int = 10, lr: float = 1e-2,
                 threshold: float = 100.0, device: int = 0):
    """The refined fit of one sRGB u8 image (host array, page-locked memory copies fastest), end to
    end on the GPU through the native pipeline: quadtree, tile extraction, pool generation, init
    round, ``steps`` Adam steps and the wire-grid snap, one host read of the tile list in between.
    Returns (tiles int32 (n, 3) of (x, y, side), rows float32 (n, 16) on the wire grid, kinds int32
    (n,), -1 = no primitive) as host arrays.  The refiner (and its device workspace) is kept per
    device and settings."""
    key = (int(device), int(quality), int(cap), int(steps), float(lr), float(threshold))
    r = _REFINERS.get(key)
    if r is None:
        r = _REFINERS[key] = Refiner(quality, cap, steps, lr, threshold, device)
    return r(u8)
