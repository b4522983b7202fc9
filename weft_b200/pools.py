"""Initial candidate pools generated on the GPU (host side of ``include/weftk_pool.h``).

``PoolTables`` builds, once per quality, the geometry the device generator needs: the
template split lines of ``_generate_candidates`` (src/weft/encoder.py:535-745), the
orientation splits of ``generate_edge_driven_candidates`` (src/weft/edge_analysis.py:139-315)
for each of its 16 possible orientations (the 12 histogram bin centres and the 4 fallback
angles), the histogram's bin edges and the palette's run boundaries.  They are computed here
with the reference's own float64 Python / numpy expressions, so the device reads exactly the
values the reference would compute; the pixel-dependent work (Sobel, histogram, sorts,
percentiles, every mean, de-duplication) runs in ``weftk_gen_pools``.

``generate_pools`` fills the constant + linear pools of tiles that are already resident on the
device (``WeftFitState``-style float4 pixels).  It is the device counterpart of
``candidates.tile_candidates(tile, quality, kinds=(0, 1), atan2="rounded")``.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib

SIDES = (8, 16, 32, 64)
MAX_SPECS = 52
MAX_CONST_LINEAR = 272
ORIENT_FALLBACK = (0.0, np.pi / 4, np.pi / 2, 3 * np.pi / 4)


SPLITS = 16 + MAX_SPECS
SIDE_WORDS = SPLITS * sum(s * s // 32 for s in SIDES)


class WeftPoolTables(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("spec_geom", "spec_mask", "orient_geom", "orient_mask", "bin_edges",
                                               "cuts", "side_bits")] + [("n_spec", ctypes.c_int32),
                                                                        ("n_centre", ctypes.c_int32)]


assert ctypes.sizeof(WeftPoolTables) == 64


class WeftPoolJob(ctypes.Structure):
    _fields_ = [("src", ctypes.c_void_p), ("px_off", ctypes.c_void_p), ("pool_off", ctypes.c_void_p),
                ("pool_cap", ctypes.c_int32), ("kinds_mask", ctypes.c_int32), ("cand", ctypes.c_void_p),
                ("pool_cnt", ctypes.c_void_p), ("tiles", ctypes.c_void_p * 4), ("n_tiles", ctypes.c_int32 * 4)]


def template_specs(size: int, quality: int):
    """(x0, y0, x1, y1, centre) of the template split lines, as ``_generate_candidates``."""
    hf = wf = float(size - 1)
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
    return specs, n_ang


def orientation_angles() -> list[float]:
    """The 16 orientations the edge pool can use: bin centres of the 12-bin histogram over
    [0, pi), then the fallback for a flat tile."""
    edges = np.linspace(0, np.pi, 13)
    return [float((edges[i] + edges[i + 1]) / 2.0) for i in range(12)] + list(ORIENT_FALLBACK)


def orientation_lines(size: int, th: float):
    """Centre split and the two offset splits of the edge pool for orientation ``th``."""
    hf = wf = float(size - 1)
    cx, cy = wf * 0.5, hf * 0.5
    nx, ny = -math.sin(th), math.cos(th)
    centre = (cx - nx * wf * 0.6, cy - ny * hf * 0.6, cx + nx * wf * 0.6, cy + ny * hf * 0.6)
    out = [centre]
    for f in (0.25, 0.75):
        ox, oy = cx + nx * wf * (f - 0.5), cy + ny * hf * (f - 0.5)
        out.append((ox - nx * wf * 0.4, oy - ny * hf * 0.4, ox + nx * wf * 0.4, oy + ny * hf * 0.4))
    return out


def build_tables(quality: int) -> dict[str, np.ndarray]:
    """Host arrays of ``WeftPoolTables`` for one quality."""
    spec_geom = np.zeros((4, MAX_SPECS, 4), np.float64)
    spec_mask = np.zeros((4, MAX_SPECS, 4), np.float32)
    orient_geom = np.zeros((4, 16, 3, 4), np.float64)
    orient_mask = np.zeros((4, 16, 4), np.float32)
    cuts = np.zeros((4, 3, 5), np.int32)
    n_spec = n_centre = 0
    for si, size in enumerate(SIDES):
        specs, n_centre = template_specs(size, quality)
        n_spec = len(specs)
        lines = np.array([s[:4] for s in specs], dtype=np.float32)  # the side test runs on float32 copies
        spec_geom[si, :n_spec] = [s[:4] for s in specs]
        spec_mask[si, :n_spec, 0] = lines[:, 0]
        spec_mask[si, :n_spec, 1] = lines[:, 1]
        spec_mask[si, :n_spec, 2] = lines[:, 3] - lines[:, 1]
        spec_mask[si, :n_spec, 3] = lines[:, 2] - lines[:, 0]
        for oi, th in enumerate(orientation_angles()):
            ls = orientation_lines(size, th)
            orient_geom[si, oi] = ls
            x0, y0, x1, y1 = ls[0]
            # side test with the line's Python floats: each cast to float32 where it meets the
            # float32 pixel grid, the differences y1 - y0 and x1 - x0 taken in float64 first
            orient_mask[si, oi] = (np.float32(x0), np.float32(y0), np.float32(y1 - y0), np.float32(x1 - x0))
        n = size * size
        for ki, k in enumerate((2, 3, 4)):
            c = (np.arange(k + 1, dtype=np.float64) * (n / k)).astype(np.int64)
            cuts[si, ki, :k + 1] = c
    return {"spec_geom": spec_geom, "spec_mask": spec_mask, "orient_geom": orient_geom,
            "orient_mask": orient_mask, "bin_edges": np.linspace(0, np.pi, 13), "cuts": cuts,
            "n_spec": n_spec, "n_centre": n_centre}


class PoolTables:
    """``WeftPoolTables`` resident on one device."""

    def __init__(self, quality: int, device: int = 0):
        self.quality = int(quality)
        self.device = torch.device("cuda", device)
        host = build_tables(self.quality)
        self._t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(self.device) for k, v in host.items()
                   if isinstance(v, np.ndarray)}
        self.side_bits = torch.zeros(SIDE_WORDS, dtype=torch.int32, device=self.device)
        self.st = WeftPoolTables(*[_lib.ptr(self._t[k]) for k in ("spec_geom", "spec_mask", "orient_geom",
                                                                  "orient_mask", "bin_edges", "cuts")],
                                 None, int(host["n_spec"]), int(host["n_centre"]))
        lib = _lib.lib_for_device(self.device.index or 0)
        _lib.check(lib.weftk_pool_side_bits(ctypes.addressof(self.st), _lib.ptr(self.side_bits),
                                            torch.cuda.current_stream(self.device).cuda_stream),
                   "weftk_pool_side_bits")
        torch.cuda.current_stream(self.device).synchronize()
        self.st.side_bits = _lib.ptr(self.side_bits)

    def side_masks(self, side: int) -> np.ndarray:
        """The side-bit table of tile side ``side`` unpacked: bool (SPLITS, side, side), True on
        side a (rows: the 16 orientations' centre lines, then the template lines)."""
        si = SIDES.index(int(side))
        before = SPLITS * sum(s * s // 32 for s in SIDES[:si])
        words = self.side_bits[before:before + SPLITS * side * side // 32].cpu().numpy().view(np.uint32)
        bits = (words[:, None] >> np.arange(32, dtype=np.uint32)[None, :]) & 1
        return bits.reshape(SPLITS, side, side).astype(bool)


_TABLES: dict[tuple[int, int], PoolTables] = {}


def tables_for(quality: int, device: int = 0) -> PoolTables:
    key = (int(quality), int(device))
    if key not in _TABLES:
        _TABLES[key] = PoolTables(quality, device)
    return _TABLES[key]


def generate_pools(src: torch.Tensor, px_off: torch.Tensor, sizes: np.ndarray, pool_off: torch.Tensor,
                   cand: torch.Tensor, pool_cnt: torch.Tensor, quality: int, kinds=(0, 1),
                   pool_cap: int = MAX_CONST_LINEAR, tiles_by_side=None) -> None:
    """Enqueue the generation of every tile's constant / linear pool (``weftk_gen_pools``).

    ``src`` float4 pixels, ``px_off`` / ``pool_off`` int32 per tile (device), ``sizes`` tile sides
    (host), ``cand`` the 60-byte record slots (uint8 device tensor), ``pool_cnt`` int32 per tile
    (output).  ``tiles_by_side`` (optional) reuses device index lists per side."""
    dev = src.device
    tb = tables_for(quality, dev.index or 0)
    lib = _lib.lib_for_device(dev.index or 0)
    if tiles_by_side is None:
        tiles_by_side = tile_lists(sizes, dev)
    mask = sum(1 << int(k) for k in kinds)
    job = WeftPoolJob(_lib.ptr(src), _lib.ptr(px_off), _lib.ptr(pool_off), int(pool_cap), mask, _lib.ptr(cand),
                      _lib.ptr(pool_cnt))
    for i, t in enumerate(tiles_by_side):
        job.tiles[i] = _lib.ptr(t) if t is not None else None
        job.n_tiles[i] = int(t.numel()) if t is not None else 0
    _lib.check(lib.weftk_gen_pools(ctypes.addressof(tb.st), ctypes.addressof(job),
                                   torch.cuda.current_stream(dev).cuda_stream), "weftk_gen_pools")


def tile_lists(sizes: np.ndarray, device) -> list:
    """Device int32 index lists of the tiles of each side (8, 16, 32, 64), None when empty."""
    out = []
    for s in SIDES:
        idx = np.nonzero(np.asarray(sizes) == s)[0].astype(np.int32)
        out.append(torch.from_numpy(idx).to(device) if idx.size else None)
    return out


class DeviceRefinedFit:
    """The refined fit with its candidate pools generated on the device: ``weftk_gen_pools``
    (constant + linear patches), the init round, the fused Adam steps and the wire-grid snap,
    replayed from one CUDA graph over tiles resident on the device (``src4`` float4 pixels,
    tile-major, sides ``sizes``).  ``run()`` returns the refined rows on the wire grid
    (``RefinedFit.q_rows``: one row per tile)."""

    def __init__(self, src4: torch.Tensor, sizes, quality: int = 75, caps=None, steps: int = 10, lr: float = 1e-2,
                 kinds=(0, 1), use_graph: bool = True, autotune: bool = True, generate_in_run: bool = True):
        """``generate_in_run=False`` generates the pools once here and leaves them resident: ``run()``
        is then the fit alone over device-resident pools."""
        from .fit import BatchedFit
        from .refine import RefinedFit

        self.src4 = src4
        self.sizes = np.asarray(sizes, np.int32)
        self.quality = int(quality)
        self.kinds = tuple(kinds)
        n = len(self.sizes)
        dev = src4.device
        self.stride = MAX_CONST_LINEAR
        self.cand = torch.zeros(n * self.stride * _lib.PRIM_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        self.cnt = torch.zeros(n, dtype=torch.int32, device=dev)
        self.lists = tile_lists(self.sizes, dev)
        mask = sum(1 << int(k) for k in self.kinds)
        self.fit = BatchedFit.from_device_pools(src4, self.sizes, self.cand, self.cnt, self.stride, quality, caps,
                                                kinds_mask=mask)
        self.fit.use_closed_form_init(True).init_only()
        self._gen = self._generator()
        if autotune or not generate_in_run:
            self.generate()  # the autotuner times scoring launches over real pools
        if autotune:
            self.fit.autotune()
        # the prelude holds the generation's arguments, not this object: no reference cycle keeps
        # the device buffers alive past the last reference
        self.rf = RefinedFit(self.fit, steps=steps, lr=lr, use_graph=use_graph,
                             prelude=self._gen if generate_in_run else None)

    def _generator(self):
        src4, f, sizes, cand, cnt = self.src4, self.fit, self.sizes, self.cand, self.cnt
        quality, kinds, stride, lists = self.quality, self.kinds, self.stride, self.lists

        def gen() -> None:
            generate_pools(src4, f.t_px_off, sizes, f.t_pool_off, cand, cnt, quality, kinds, stride, lists)

        return gen

    def generate(self) -> None:
        """Enqueue the pool generation (device work only)."""
        self._gen()

    def run(self) -> torch.Tensor:
        self.rf.run()
        return self.rf.q_rows

    def pool_records(self) -> list[np.ndarray]:
        """The generated pools as per-tile 60-byte records (host copy)."""
        recs = self.cand.cpu().numpy().view(_lib.PRIM_DTYPE)
        cnt = self.cnt.cpu().numpy()
        return [recs[t * self.stride:t * self.stride + int(cnt[t])] for t in range(len(self.sizes))]


def refine_tiles(pixels: np.ndarray, sizes, quality: int = 75, caps=None, steps: int = 10, lr: float = 1e-2,
                 device: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Fit tiles given in host memory end to end on one GPU: upload the tile pixels
    (``(sum ts^2, 3)`` float32, tile-major, row-major inside a tile; page-locked memory copies
    fastest), generate the constant + linear candidate pools on the device, run the refined fit
    (init round, ``steps`` Adam steps) and return each tile's primitive snapped to the wire grid as
    (rows float32[n, 16] in the ``weftk_refine.h`` layout, kinds int32[n], -1 = none)."""
    dev = torch.device("cuda", device)
    sizes = np.asarray(sizes, np.int32)
    n_px = int((sizes.astype(np.int64) ** 2).sum())
    if pixels.shape != (n_px, 3):
        raise ValueError(f"pixels must be ({n_px}, 3)")
    src4 = torch.zeros((n_px, 4), dtype=torch.float32, device=dev)
    src4[:, :3] = torch.from_numpy(np.ascontiguousarray(pixels, np.float32)).to(dev, non_blocking=True)
    drf = DeviceRefinedFit(src4, sizes, quality, caps=caps, steps=steps, lr=lr, use_graph=False, autotune=False)
    rows = drf.run()
    return rows.cpu().numpy(), drf.rf.kinds.cpu().numpy()
