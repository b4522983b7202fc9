"""Batched greedy candidate-scoring fit with all state resident on the GPU.

Host side of ``include/weftk_fit.h``.  ``BatchedFit`` takes the tiles of one or
many images and their candidate pools, uploads them once, and runs the
reference's greedy (src/weft/encoder.py:2668-2831) with one
``weftk_fit_round`` launch sequence per round for every tile at once:

    init  : best single candidate per tile (accepted unconditionally)
    rounds: score selected+candidate for every live candidate of every complex
            tile, accept the argmin if it lowers the objective
    stall : when no tile improved, re-seed the complex tiles that have room
            with residual-targeted candidates (at most 3 times)

Per round the host reads back 16 bytes of counters.  Candidate slots are
sorted by kind for scoring (``perm``) so work items have uniform cost; the
argmin still breaks ties by original pool order, as the reference's
``np.argmin`` does.  Device memory comes from torch; the kernels come from
libweftk.so (no fallback).
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, rate
from ._lib import FIT_ITEM_DTYPE, PRIM_DTYPE
from .candidates import Cand, residual_candidates
from .quadtree import MAX_PRIMS_BY_SIZE

# FP32 operations per pixel to evaluate one primitive of each kind over a pixel
# (the blend included); used to balance scoring work items.
KIND_COST = np.array([10, 24, 28, 509, 26, 112, 10, 10], np.int64)
RESEED_RESERVE = 3 * 128  # slots kept per tile for up to 3 re-seeds (<= 117 candidates each)
CHUNK = {8: 128, 16: 64, 32: 32}
FIT_INIT, FIT_ROUND = 0, 1
TILE_COMPLEX, TILE_EVAL, TILE_IMPROVED = 1, 2, 4


def pack_cands(cands) -> np.ndarray:
    n = len(cands)
    arr = np.zeros(n, PRIM_DTYPE)
    if n == 0:
        return arr
    arr["kind"] = [c.kind for c in cands]
    arr["alpha"] = [c.alpha for c in cands]
    arr["color0"] = [tuple(c.color0) for c in cands]
    arr["color1"] = [tuple(c.color1) if c.color1 is not None else (0.0, 0.0, 0.0) for c in cands]
    arr["geom"] = [tuple(c.geom)[:7] + (0.0,) * (7 - min(7, len(c.geom))) for c in cands]
    return arr


def unpack_cands(arr: np.ndarray) -> list:
    glen = {0: 0, 1: 4, 2: 5, 3: 7, 4: 6}
    out = []
    for r in arr:
        k = int(r["kind"])
        out.append(Cand(k, tuple(float(v) for v in r["geom"][:glen.get(k, 7)]), tuple(float(v) for v in r["color0"]),
                        tuple(float(v) for v in r["color1"]) if k == 1 else None, float(r["alpha"])))
    return out


def slot_layout(records: np.ndarray, counts: np.ndarray, pool_off: np.ndarray, n_slots: int):
    """Kind of every slot (int8; 7 = empty or unknown kind) and the slot of every packed record
    (``pool_off`` of its tile + its index in the tile's pool), or ``None`` for the slots when that is
    the record's own index (no slots reserved for re-seeding), so the records are the slot array."""
    rec_kind = np.minimum(records["kind"], 7).astype(np.int8)
    if len(records) == n_slots:
        return rec_kind, None
    n = len(counts)
    first = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64) if n else np.zeros(0, np.int64)
    slots = np.repeat(pool_off - first, counts) + np.arange(int(counts.sum()))
    kinds = np.full(n_slots, 7, np.int8)
    kinds[slots] = rec_kind
    return kinds, slots


def _dev(a: np.ndarray, device) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).to(device, non_blocking=False)


@dataclass
class FitStats:
    rounds: int = 0
    reseeds: int = 0
    reseed_tiles: int = 0
    evals: int = 0
    launches: int = 0
    t_reseed_s: float = 0.0
    per_round: list = field(default_factory=list)


class BatchedFit:
    """All tiles of a fit, resident on one GPU."""

    def __init__(self, patches, pools, quality: int = 75, caps=None, device: int = 0, reserve: int = RESEED_RESERVE):
        """``patches``: per-tile (ts, ts, 3) float32 arrays; ``pools``: per-tile candidate
        lists (``Cand``-like objects) or packed record arrays."""
        patches = [np.ascontiguousarray(p, np.float32) for p in patches]
        sizes = np.array([p.shape[0] for p in patches], np.int32)
        pixels = np.concatenate([p.reshape(-1, 3) for p in patches]) if patches else np.zeros((0, 3), np.float32)
        packed = [p if isinstance(p, np.ndarray) else pack_cands(p) for p in pools]
        counts = np.array([len(p) for p in packed], np.int64)
        records = np.concatenate(packed) if packed else np.zeros(0, PRIM_DTYPE)
        self._setup(pixels, sizes, records, counts, quality, caps, device, reserve)
        self.pools = [p if isinstance(p, np.ndarray) else list(p) for p in pools]
        self.patches = patches

    @classmethod
    def from_arrays(cls, pixels: np.ndarray, sizes, records: np.ndarray, counts, quality: int = 75, caps=None,
                    device: int = 0, reserve: int = RESEED_RESERVE) -> "BatchedFit":
        """Flat inputs: ``pixels`` (sum ts^2, 3) float32 tile-major (row-major inside a
        tile), ``sizes`` per tile, ``records`` all pools' 60-byte records back to back,
        ``counts`` pool length per tile."""
        self = cls.__new__(cls)
        self._setup(np.asarray(pixels, np.float32), np.asarray(sizes, np.int32), np.asarray(records, PRIM_DTYPE),
                    np.asarray(counts, np.int64), quality, caps, device, reserve)
        self.pools = None
        self.patches = None
        return self

    @classmethod
    def from_device_pools(cls, src4: torch.Tensor, sizes, cand: torch.Tensor, counts: torch.Tensor, stride: int,
                          quality: int = 75, caps=None, kinds_mask: int = 0b11) -> "BatchedFit":
        """Tiles and pools already resident on the device, e.g. made by ``pools.generate_pools``:
        ``src4`` float4 pixels (tile-major), ``sizes`` tile sides (host), ``cand`` the 60-byte
        records of ``len(sizes) * stride`` slots (tile t owns slots [t * stride, (t + 1) * stride)),
        ``counts`` the filled slots per tile (device int32; read only on the device), and
        ``kinds_mask`` the primitive kinds the pools may hold (bit k for kind k).  Nothing here reads
        the pools' contents, so they may be (re)generated after construction, e.g. inside the same
        captured graph as the fit; the scoring work depends on the layout only.  No host copy of the
        pools exists, so re-seeding runs on the device only."""
        self = cls.__new__(cls)
        sizes = np.asarray(sizes, np.int32)
        n = len(sizes)
        self._layout(sizes, np.full(n, int(stride), np.int64), quality, caps, src4.device.index or 0)
        if src4.shape != (int((sizes.astype(np.int64) ** 2).sum()), 4) or cand.numel() != self.n_slots * PRIM_DTYPE.itemsize:
            raise ValueError("pixels or candidate slots do not match the tile layout")
        d = self.device
        self.pool_cnt = self.init_cnt = None
        self._init_kinds = self.kinds = None
        self._kinds_mask = int(kinds_mask)
        t_init_cnt = counts.to(device=d, dtype=torch.int32).contiguous()
        self._finish(src4, cand, t_init_cnt.clone(), t_init_cnt, None)
        self.pools = None
        self.patches = None
        return self

    def _layout(self, sizes, pool_cap, quality, caps, device) -> None:
        """Tile and slot layout (host): sizes, caps, pixel offsets, slot offsets."""
        self.device = torch.device("cuda", device)
        self.lib = _lib.lib_for_device(device)
        self.quality = int(quality)
        self.lam = rate.tile_lambda(quality)
        self.thr = rate.complexity_threshold(quality)
        n = len(sizes)
        self.n = n
        self.sizes = sizes
        if np.any(~np.isin(self.sizes, (8, 16, 32, 64))):
            raise ValueError("tile sizes must be 8, 16, 32 or 64")
        self.caps = np.array(caps if caps is not None else [MAX_PRIMS_BY_SIZE.get(int(s), 48) for s in self.sizes],
                             np.int32)
        self.cap_max = int(self.caps.max()) if n else 1
        self.pool_cap = np.asarray(pool_cap, np.int64)
        self.pool_off = np.zeros(n, np.int64)
        if n > 1:
            np.cumsum(self.pool_cap[:-1], out=self.pool_off[1:])
        self.n_slots = int(self.pool_cap.sum()) if n else 0
        if self.n_slots >= 2 ** 31:
            raise ValueError("too many candidate slots")
        px = self.sizes.astype(np.int64) ** 2
        self.px_off = np.zeros(n, np.int64)
        if n > 1:
            np.cumsum(px[:-1], out=self.px_off[1:])
        self.n_px = int(px.sum())

    def _setup(self, pixels, sizes, records, counts, quality, caps, device, reserve) -> None:
        cnt = counts.astype(np.int64)
        self._layout(sizes, cnt + reserve, quality, caps, device)
        self.pool_cnt = cnt.astype(np.int32)
        self.init_cnt = self.pool_cnt.copy()
        if pixels.shape != (self.n_px, 3):
            raise ValueError(f"pixels must be ({self.n_px}, 3)")
        if len(records) != int(cnt.sum()):
            raise ValueError("records and counts disagree")
        d = self.device
        t_src = torch.zeros((self.n_px, 4), dtype=torch.float32, device=d)
        t_src[:, :3] = _dev(pixels, d)
        self.kinds, slots = slot_layout(records, cnt, self.pool_off, self.n_slots)
        rec_bytes = np.ascontiguousarray(records).view(np.uint8).reshape(-1, PRIM_DTYPE.itemsize)
        if slots is None:
            t_cand = _dev(rec_bytes, d).view(-1) if len(records) else torch.zeros(0, dtype=torch.uint8, device=d)
        else:
            t_cand = torch.zeros((self.n_slots, PRIM_DTYPE.itemsize), dtype=torch.uint8, device=d)
            if len(records):
                t_cand[_dev(slots, d)] = _dev(rec_bytes, d)
            t_cand = t_cand.view(-1)
        self._init_kinds = self.kinds.copy()
        self._finish(t_src, t_cand, _dev(self.pool_cnt, d), _dev(self.init_cnt, d), _dev(self._init_kinds, d))

    def _finish(self, t_src, t_cand, t_pool_cnt, t_init_cnt, t_init_kinds) -> None:
        """Device state of the fit around the given pixels, records, counts and slot kinds."""
        d = self.device
        n = self.n
        self.t_src = t_src
        self.t_cand = t_cand
        self.t_pool_cnt = t_pool_cnt
        self.t_init_cnt = t_init_cnt
        self.t_init_kinds = t_init_kinds
        self.t_bg = torch.zeros((self.n_px, 4), dtype=torch.float32, device=d)
        self.t_px_off = _dev(self.px_off.astype(np.int32), d)
        self.t_size = _dev(self.sizes, d)
        self.t_cap = _dev(self.caps, d)
        self.t_pool_off = _dev(self.pool_off.astype(np.int32), d)
        self.t_pool_cap = _dev(self.pool_cap.astype(np.int32), d)
        self.t_n_alive = torch.zeros(n, dtype=torch.int32, device=d)
        self.t_n_sel = torch.zeros(n, dtype=torch.int32, device=d)
        self.t_sel_bits = torch.full((n,), 8, dtype=torch.int32, device=d)
        self.t_flags = torch.zeros(n, dtype=torch.int32, device=d)
        self.t_cur_obj = torch.zeros(n, dtype=torch.float64, device=d)
        self.t_sel = torch.full((n * self.cap_max,), -1, dtype=torch.int32, device=d)
        self.t_prep = torch.empty(self.n_slots * 16, dtype=torch.float32, device=d)
        self.t_alive = torch.zeros(self.n_slots, dtype=torch.uint8, device=d)
        self.t_kind = torch.zeros(self.n_slots, dtype=torch.uint8, device=d)
        self.t_partial = torch.empty(self.n_slots * 4, dtype=torch.float32, device=d)
        self.t_status = torch.zeros(4, dtype=torch.int32, device=d)
        self.t_work = torch.zeros(2, dtype=torch.int64, device=d)
        self.t_zero_first = torch.zeros(n, dtype=torch.int32, device=d)
        self.h_status = torch.zeros(4, dtype=torch.int32).pin_memory()
        self.st = _lib.WeftFitState(
            n, self.cap_max, self.n_slots,
            *[_lib.ptr(x) for x in (self.t_src, self.t_bg, self.t_px_off, self.t_size, self.t_cap, self.t_pool_off,
                                    self.t_pool_cnt, self.t_pool_cap, self.t_n_alive, self.t_n_sel, self.t_sel_bits,
                                    self.t_flags, self.t_cur_obj, self.t_sel, self.t_cand, self.t_prep, self.t_alive,
                                    self.t_kind, self.t_partial, self.t_status, self.t_work)])
        self.stats = FitStats()
        self.device_reseeded = False
        self.n_items = {}
        self.chunk = dict(CHUNK)  # candidates per scoring CTA, per size class (set by autotune)
        self.tuning = None
        _lib.check(self.lib.weftk_fit_prepare(ctypes_ref(self.st), _lib.ptr(self.t_zero_first), self._stream()),
                   "weftk_fit_prepare")
        self._build_work()

    # ------------------------------------------------------------------ plumbing
    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def _prepare(self, first_new: np.ndarray) -> None:
        t_first = _dev(first_new.astype(np.int32), self.device)
        _lib.check(self.lib.weftk_fit_prepare(ctypes_ref(self.st), _lib.ptr(t_first), self._stream()),
                   "weftk_fit_prepare")
        self._keep = t_first  # keep alive until the launch has consumed it

    def _build_work(self) -> None:
        """perm and cost-sorted work items per size class, covering every reserved slot.

        The initial pool is scored in kind order (curves first) so a work item
        holds candidates of similar cost; re-seeded slots are scored in slot
        order.  Items cover the reserved slots too; the kernel only scores the
        filled ones, so re-seeding needs no new items.  Sorting runs on the GPU.
        Over device pools the layout alone decides (``_build_static_work``).
        """
        if self._init_kinds is None:
            self._build_static_work()
            return
        d = self.device
        n = self.n
        cap = torch.from_numpy(self.pool_cap).to(d)
        cnt = self.t_init_cnt.to(torch.int64)
        off = torch.from_numpy(self.pool_off).to(d)
        kinds = self.t_init_kinds.to(torch.int64)
        tile_of = torch.repeat_interleave(torch.arange(n, device=d), cap)
        local = torch.arange(self.n_slots, device=d) - torch.repeat_interleave(off, cap)
        filled = local < cnt[tile_of]
        cost = torch.from_numpy(KIND_COST).to(d)[kinds]
        # order inside each tile: filled slots by descending cost (stable), then the reserve
        key = tile_of * (1 << 20) + torch.where(filled, 1023 - cost, torch.full_like(cost, 1 << 12))
        order = torch.sort(key, stable=True).indices
        perm = local[order].to(torch.int32)
        self.t_perm = perm.contiguous()
        slot_cost = torch.where(filled, cost, torch.zeros_like(cost))[order]
        csum = torch.cat([torch.zeros(1, dtype=torch.int64, device=d), torch.cumsum(slot_cost, 0)])
        sizes = torch.from_numpy(self.sizes.astype(np.int64)).to(d)
        items = {}
        for cls, members in ((8, (8,)), (16, (16,)), (32, (32, 64))):
            chunk = self.chunk[cls]
            sel = torch.zeros(n, dtype=torch.bool, device=d)
            for m in members:
                sel |= sizes == m
            ts_idx = torch.nonzero(sel).flatten()
            if ts_idx.numel() == 0:
                items[cls] = None
                self.n_items[cls] = 0
                continue
            nch = (cap[ts_idx] + chunk - 1) // chunk
            t_rep = torch.repeat_interleave(ts_idx, nch)
            k = torch.arange(int(nch.sum()), device=d) - torch.repeat_interleave(torch.cumsum(nch, 0) - nch, nch)
            first = k * chunk
            count = torch.minimum(torch.full_like(first, chunk), cap[t_rep] - first)
            g0 = off[t_rep] + first
            px = sizes[t_rep] ** 2
            c = (csum[g0 + count] - csum[g0]) * px
            blocks = torch.clamp(px // 1024, min=1)
            b_rep = torch.repeat_interleave(torch.arange(t_rep.numel(), device=d), blocks)
            blk = torch.arange(b_rep.numel(), device=d) - torch.repeat_interleave(torch.cumsum(blocks, 0) - blocks, blocks)
            rows = torch.stack([t_rep[b_rep], blk, first[b_rep], count[b_rep]], 1).to(torch.int32)
            o = torch.sort(-c[b_rep], stable=True).indices
            items[cls] = rows[o].contiguous()
            self.n_items[cls] = int(rows.shape[0])
        self.t_items = items
        self._alloc_queue()

    def _build_static_work(self) -> None:
        """Work that depends on the tile layout only, not on the pools' contents (which live on
        the device and may be regenerated inside a captured graph): identity scoring order, and
        per size class every tile's slot range cut into runs of ``chunk`` candidates x 1024-pixel
        blocks, largest tiles first.  Runs past a tile's filled slots end at once."""
        d = self.device
        cap = self.pool_cap.astype(np.int64)
        if self.n and np.all(cap == cap[0]):  # uniform stride: the identity order on the device
            self.t_perm = torch.remainder(torch.arange(self.n_slots, dtype=torch.int32, device=d), int(cap[0]))
        else:
            local = np.arange(self.n_slots, dtype=np.int64) - np.repeat(self.pool_off, cap)
            self.t_perm = torch.from_numpy(local.astype(np.int32)).to(d)
        items = {}
        for cls, members in ((8, (8,)), (16, (16,)), (32, (32, 64))):
            chunk = self.chunk[cls]
            ts_idx = np.nonzero(np.isin(self.sizes, members))[0]
            if ts_idx.size == 0:
                items[cls] = None
                self.n_items[cls] = 0
                continue
            ts_idx = ts_idx[np.argsort(-self.sizes[ts_idx].astype(np.int64), kind="stable")]
            nch = (cap[ts_idx] + chunk - 1) // chunk
            blocks = np.maximum(1, self.sizes[ts_idx].astype(np.int64) ** 2 // 1024)
            per_tile = nch * blocks
            t_rep = np.repeat(ts_idx, per_tile)
            j = np.arange(int(per_tile.sum())) - np.repeat(np.cumsum(per_tile) - per_tile, per_tile)
            b_rep = np.repeat(blocks, per_tile)
            first = (j // b_rep) * chunk
            cnt = np.minimum(chunk, cap[t_rep] - first)
            arr = np.stack([t_rep, j % b_rep, first, cnt], 1).astype(np.int32)
            items[cls] = torch.from_numpy(arr).to(d)
            self.n_items[cls] = len(arr)
        self.t_items = items
        self._alloc_queue()

    def _alloc_queue(self) -> None:
        """The rounds' work queue (``WeftFitState.queue``): room for every item of the three size
        classes, or off when ``use_queue(False)`` was set."""
        if not getattr(self, "_queue_on", True):
            self.st.queue = self.st.queue_ctl = None
            return
        total = max(1, sum(self.n_items.get(k, 0) for k in (8, 16, 32)))
        if getattr(self, "t_queue", None) is None or self.t_queue.numel() < total:
            self.t_queue = torch.empty(total, dtype=torch.int32, device=self.device)
            self.t_queue_ctl = torch.zeros(8, dtype=torch.int32, device=self.device)
        self.st.queue = _lib.ptr(self.t_queue)
        self.st.queue_ctl = _lib.ptr(self.t_queue_ctl)

    def use_queue(self, on: bool = True) -> "BatchedFit":
        """Persistent queue-driven scoring launches (default) or one CTA per work item."""
        self._queue_on = bool(on)
        self._alloc_queue()
        return self

    def _round(self, mode: int) -> tuple[int, int]:
        ti = self.t_items
        n8, n16, n32 = (self.n_items[k] for k in (8, 16, 32))
        rc = self.lib.weftk_fit_round(ctypes_ref(self.st), mode, self.lam, self.thr, _lib.ptr(self.t_perm),
                                      _lib.ptr(ti[8]), n8, _lib.ptr(ti[16]), n16, _lib.ptr(ti[32]), n32,
                                      self._stream())
        _lib.check(rc, "weftk_fit_round")
        self.stats.launches += 1
        self.h_status.copy_(self.t_status, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        ev, imp = int(self.h_status[0]), int(self.h_status[1])
        self.stats.per_round.append((mode, ev, imp))
        return ev, imp

    # ------------------------------------------------------------------ re-seed
    def _reseed(self, reseed, reseed_batch=None) -> None:
        if self.init_cnt is None:
            raise ValueError("a fit over device pools re-seeds on the device only")
        t0 = time.perf_counter()
        flags = self.t_flags.cpu().numpy()
        n_sel = self.t_n_sel.cpu().numpy()
        tiles = np.nonzero((flags & TILE_COMPLEX) & (n_sel < self.caps))[0]
        if tiles.size == 0:
            return
        bg = self.t_bg.cpu().numpy()
        first_new = self.pool_cnt.copy()
        new_recs, new_slots = [], []
        preds = []
        for t in tiles:
            s = int(self.sizes[t])
            a = int(self.px_off[t])
            preds.append(np.clip(bg[a:a + s * s, :3].reshape(s, s, 3), 0.0, 1.0))
        if self.patches is None:
            raise ValueError("host re-seeding needs the per-tile patches; use the device re-seed")
        if reseed_batch is not None:
            batch = reseed_batch([int(t) for t in tiles], [self.patches[t] for t in tiles], preds)
        else:
            fn = reseed if reseed is not None else \
                (lambda t, patch, pred: residual_candidates(patch, pred, self.quality))
            batch = [fn(int(t), self.patches[t], p) for t, p in zip(tiles, preds)]
        for t, cands in zip(tiles, batch):
            if not cands:
                continue
            k = len(cands)
            c0 = int(self.pool_cnt[t])
            if c0 + k > self.pool_cap[t]:
                raise RuntimeError(f"tile {t}: re-seed overflows its {self.pool_cap[t]} candidate slots")
            if self.pools is not None:
                if isinstance(self.pools[t], np.ndarray):
                    self.pools[t] = unpack_cands(self.pools[t])
                self.pools[t].extend(cands)
            new_recs.append(pack_cands(cands))
            new_slots.append(self.pool_off[t] + c0 + np.arange(k))
            self.pool_cnt[t] = c0 + k
        self.stats.reseeds += 1
        self.stats.reseed_tiles += int(tiles.size)
        if new_recs:
            recs = np.concatenate(new_recs)
            slots = np.concatenate(new_slots)
            self.kinds[slots] = np.where(recs["kind"] < 7, recs["kind"], 7)
            view = self.t_cand.view(-1, PRIM_DTYPE.itemsize)
            view[_dev(slots.astype(np.int64), self.device)] = _dev(recs.view(np.uint8).reshape(-1, PRIM_DTYPE.itemsize),
                                                                    self.device)
            self.t_pool_cnt.copy_(torch.from_numpy(self.pool_cnt))
            self._prepare(first_new)
        self.stats.t_reseed_s += time.perf_counter() - t0

    def _reseed_device(self) -> None:
        _lib.check(self.lib.weftk_fit_reseed(ctypes_ref(self.st), self.quality, self._stream()), "weftk_fit_reseed")
        self.stats.reseeds += 1
        self.device_reseeded = True

    def reset(self) -> None:
        """Forget the fit (selections, re-seeds) but keep pixels and initial pools resident."""
        if self.init_cnt is not None:
            self.pool_cnt[:] = self.init_cnt
        self.device_reseeded = False
        for t in range(self.n if self.pools is not None else 0):
            p = self.pools[t]
            if not isinstance(p, np.ndarray) and len(p) > self.init_cnt[t]:
                del p[self.init_cnt[t]:]
        if self._init_kinds is not None:
            self.kinds[:] = self._init_kinds
        self._moments()
        _lib.check(self.lib.weftk_fit_reset(ctypes_ref(self.st), _lib.ptr(self.t_init_cnt), self._stream()),
                   "weftk_fit_reset")
        _lib.check(self.lib.weftk_fit_prepare(ctypes_ref(self.st), _lib.ptr(self.t_zero_first), self._stream()),
                   "weftk_fit_prepare")
        self.stats = FitStats()
        self.device_reseeded = False

    # -------------------------------------------------------------- graph-capturable init-only fit
    def run_init_only(self) -> None:
        """Reset and run only the init round (best single candidate per tile), launching
        device work only: no host copies or syncs, so it can be captured in a CUDA graph.
        With the closed-form init on, the per-tile moments are computed beside the reset and the
        preparation (on a side stream, joined before the round)."""
        s = self._stream()
        joined = None
        if self.st.moments:
            main = torch.cuda.current_stream(self.device)
            if not hasattr(self, "_side"):
                self._side = torch.cuda.Stream(self.device)
            fork = torch.cuda.Event()
            fork.record(main)
            self._side.wait_event(fork)
            _lib.check(self.lib.weftk_fit_moments(ctypes_ref(self.st), self.st.moments, self._side.cuda_stream),
                       "weftk_fit_moments")
            joined = torch.cuda.Event()
            joined.record(self._side)
        _lib.check(self.lib.weftk_fit_reset(ctypes_ref(self.st), _lib.ptr(self.t_init_cnt), s), "weftk_fit_reset")
        _lib.check(self.lib.weftk_fit_prepare(ctypes_ref(self.st), _lib.ptr(self.t_zero_first), s),
                   "weftk_fit_prepare")
        if joined is not None:
            torch.cuda.current_stream(self.device).wait_event(joined)
        ti = self.t_items
        rc = self.lib.weftk_fit_round(ctypes_ref(self.st), FIT_INIT, self.lam, self.thr, _lib.ptr(self.t_perm),
                                      _lib.ptr(ti[8]), self.n_items[8], _lib.ptr(ti[16]), self.n_items[16],
                                      _lib.ptr(ti[32]), self.n_items[32], s)
        _lib.check(rc, "weftk_fit_round")

    def _moments(self) -> None:
        """Per-tile pixel moments for the closed-form init, when it is on (device work only)."""
        if self.st.moments:
            _lib.check(self.lib.weftk_fit_moments(ctypes_ref(self.st), self.st.moments, self._stream()),
                       "weftk_fit_moments")

    def quantize_selected(self) -> None:
        """Snap every tile's selected stack to the wire grid into ``t_qrows`` / ``t_qkind``
        (``weftk_fit_selected_rows``: row ``t * cap_max + j`` is the j-th primitive of tile t,
        kind -1 past the stack).  Device work only."""
        if not hasattr(self, "t_qrows"):
            self.t_qrows = torch.zeros((self.n * self.cap_max, 16), dtype=torch.float32, device=self.device)
            self.t_qkind = torch.full((self.n * self.cap_max,), -1, dtype=torch.int32, device=self.device)
        _lib.check(self.lib.weftk_fit_selected_rows(ctypes_ref(self.st), _lib.ptr(self.t_qrows),
                                                    _lib.ptr(self.t_qkind), self._stream()),
                   "weftk_fit_selected_rows")

    def quantized_stacks(self) -> list[np.ndarray]:
        """The last ``quantize_selected`` output as per-tile 60-byte records (host)."""
        from .refine import rows_to_records

        rows = self.t_qrows.cpu().numpy()
        kinds = self.t_qkind.cpu().numpy()
        out = []
        for t in range(self.n):
            k = kinds[t * self.cap_max:(t + 1) * self.cap_max]
            m = int((k >= 0).sum())
            out.append(rows_to_records(rows[t * self.cap_max:t * self.cap_max + m], k[:m]))
        return out

    def run_device(self, max_rounds: int | None = None) -> "BatchedFit":
        """Reset and run the whole fit with device re-seeding, enqueued without any host
        synchronisation (``weftk_fit_run``), so it can be captured in a CUDA graph, and snap the
        selected stacks to the wire grid (``quantize_selected``).  Same decisions as ``run()``
        with device re-seeding; ``control()`` reads the outcome."""
        if not hasattr(self, "t_ctl"):
            self.t_ctl = torch.zeros(4, dtype=torch.int32, device=self.device)
        s = self._stream()
        self._moments()
        _lib.check(self.lib.weftk_fit_reset(ctypes_ref(self.st), _lib.ptr(self.t_init_cnt), s), "weftk_fit_reset")
        _lib.check(self.lib.weftk_fit_prepare(ctypes_ref(self.st), _lib.ptr(self.t_zero_first), s),
                   "weftk_fit_prepare")
        rounds = rate.max_rounds(self.quality) if max_rounds is None else int(max_rounds)
        ti = self.t_items
        rc = self.lib.weftk_fit_run(ctypes_ref(self.st), rounds, self.lam, self.thr, _lib.ptr(self.t_perm),
                                    _lib.ptr(ti[8]), self.n_items[8], _lib.ptr(ti[16]), self.n_items[16],
                                    _lib.ptr(ti[32]), self.n_items[32], _lib.ptr(self.t_ctl), s)
        _lib.check(rc, "weftk_fit_run")
        self.quantize_selected()
        self.device_reseeded = True
        return self

    def control(self) -> dict:
        """Outcome of the last ``run_device``: rounds run, stall count, whether it ended early."""
        c = self.t_ctl.cpu().numpy()
        return {"done": bool(c[0]), "stalls": int(c[1]), "rounds": int(c[3])}

    def graph(self, max_rounds: int | None = None) -> "FitGraph":
        """The device-driven fit captured once in a CUDA graph (replay() refits from scratch)."""
        return FitGraph(self, max_rounds)

    def init_only(self) -> "BatchedFit":
        """Declare that this fit runs only its init round (the refined fit): accepted candidates
        are then not composited into the per-pixel composite, which nothing reads afterwards;
        greedy rounds and re-seeding refuse such a fit."""
        self.st.bg = None
        return self

    def use_closed_form_init(self, on: bool = True) -> "BatchedFit":
        """Score constant candidates of the init round in closed form from per-tile pixel
        moments (``WeftFitState.moments``, computed by every ``run_init_only``) instead of per
        pixel; equal up to rounding, so a near tie may pick differently from the reference's
        per-pixel sum (off for the plain fit)."""
        if on:
            if not hasattr(self, "t_moments"):
                self.t_moments = torch.zeros(max(self.n, 1) * 6, dtype=torch.float64, device=self.device)
            self.st.moments = _lib.ptr(self.t_moments)
        else:
            self.st.moments = None
        return self

    def init_kinds(self) -> np.ndarray:
        """Primitive kind of every filled slot of the initial pools (host copy)."""
        if self._init_kinds is None:
            cnt = self.t_init_cnt.cpu().numpy().astype(np.int64)
            rec = self.t_cand.view(torch.int32).view(-1, PRIM_DTYPE.itemsize // 4)[:, 0].cpu().numpy()
            filled = (np.arange(self.n_slots) - np.repeat(self.pool_off, self.pool_cap)) < np.repeat(cnt, self.pool_cap)
            return rec[filled].astype(np.int32)
        k = self._init_kinds
        return k[k < 7].astype(np.int32)

    def init_kinds_mask(self) -> int:
        """Bit k set when kind k (0..6) occurs in the initial pools: ``kinds_mask_of(init_kinds())``
        from one count over the slot kinds (device pools: the mask they were declared with)."""
        if self._init_kinds is None:
            return self._kinds_mask
        k = self._init_kinds
        if k.size == 0:
            return 0
        if int(k.min()) < 0:
            from .refine import kinds_mask_of

            return kinds_mask_of(self.init_kinds())
        c = np.bincount(k, minlength=8)[:7]
        return int(sum(1 << j for j in range(7) if c[j]))

    # ------------------------------------------------------------------ autotuner
    def configure(self, variants=None, chunks=None) -> "BatchedFit":
        """Set the scoring shape per size class ({8|16|32: variant}) and candidates per CTA
        ({8|16|32: count}, at most 128); rebuilds the work items."""
        for ci, cls in enumerate((8, 16, 32)):
            if variants and cls in variants:
                v = int(variants[cls])
                if not 0 <= v < _lib.FIT_VARIANTS:
                    raise ValueError(f"no scoring variant {v} for {cls}-px tiles")
                self.st.variant[ci] = v
            if chunks and cls in chunks:
                c = int(chunks[cls])
                if not 1 <= c <= 128:
                    raise ValueError("candidates per CTA must be in 1..128")
                self.chunk[cls] = c
        self._build_work()
        return self

    def autotune(self, chunks=(32, 64, 128), reps: int = 2) -> dict:
        """Choose, per tile-size class, the scoring kernel's shape (pixels per lane x warps per
        candidate x CTAs per SM, ``weftk_fit_variant``) and the candidates per CTA that score this
        fit's init round fastest (CUDA events around the class's scoring launch, best of ``reps``).
        Leaves the fit reset with the winners in place; returns {class: (variant, chunk, ms)}."""
        import ctypes

        result = {}
        for ci, cls in enumerate((8, 16, 32)):
            if not self.n_items.get(cls):
                continue
            best = None
            for v in range(_lib.FIT_VARIANTS):
                for ch in chunks:
                    self.st.variant[ci] = v
                    self.chunk[cls] = ch
                    self._build_work()
                    times = []
                    for _ in range(reps):
                        self.reset()
                        ms, n = ctypes.c_double(0), ctypes.c_int(0)
                        self.lib.weftk_fit_timing(1, None, None)
                        ti = self.t_items
                        args = [(_lib.ptr(ti[k]), self.n_items[k]) if k == cls else (0, 0) for k in (8, 16, 32)]
                        rc = self.lib.weftk_fit_round(ctypes_ref(self.st), FIT_INIT, self.lam, self.thr,
                                                      _lib.ptr(self.t_perm), *args[0], *args[1], *args[2],
                                                      self._stream())
                        _lib.check(rc, "weftk_fit_round")
                        torch.cuda.current_stream(self.device).synchronize()
                        self.lib.weftk_fit_timing(0, ctypes.addressof(ms), ctypes.addressof(n))
                        times.append(ms.value)
                    t = min(times)
                    if best is None or t < best[2]:
                        best = (v, ch, t)
            self.st.variant[ci] = best[0]
            self.chunk[cls] = best[1]
            result[cls] = best
        self._build_work()
        self.reset()
        self.tuning = result
        return result

    def work_counters(self) -> tuple[int, int]:
        """(candidate-pixels scored, algorithmic FP32 ops) since the last reset."""
        w = self.t_work.cpu().numpy()
        return int(w[0]), int(w[1])

    # ------------------------------------------------------------------ driver
    def run(self, reseed=None, max_rounds: int | None = None, reseed_batch=None) -> "BatchedFit":
        """Run init plus up to ``max_rounds`` greedy rounds (default: the quality's budget).

        ``reseed(tile, patch, pred) -> list[Cand]`` supplies re-seed candidates
        (default ``candidates.residual_candidates``); ``reseed_batch(tiles,
        patches, preds) -> list[list[Cand]]`` does all stalled tiles at once.
        """
        self._moments()
        self._round(FIT_INIT)
        rounds = rate.max_rounds(self.quality) if max_rounds is None else int(max_rounds)
        stalls = 0
        for _ in range(rounds):
            ev, imp = self._round(FIT_ROUND)
            if ev == 0:
                break
            self.stats.rounds += 1
            if imp == 0:
                stalls += 1
                if stalls > 3:
                    break
                if reseed is None and reseed_batch is None:
                    self._reseed_device()
                else:
                    self._reseed(reseed, reseed_batch)
            else:
                stalls = 0
        return self

    # ------------------------------------------------------------------ results
    def selected_indices(self) -> list[list[int]]:
        sel = self.t_sel.cpu().numpy().reshape(self.n, self.cap_max)
        n_sel = self.t_n_sel.cpu().numpy()
        return [sel[t, :n_sel[t]].tolist() for t in range(self.n)]

    def selected_records(self) -> list[np.ndarray]:
        """The selected primitives of every tile as 60-byte records, read from the device."""
        idx = self.selected_indices()
        flat = np.concatenate([self.pool_off[t] + np.asarray(i, np.int64) for t, i in enumerate(idx)]) \
            if self.n else np.zeros(0, np.int64)
        recs = self.t_cand.view(-1, PRIM_DTYPE.itemsize)[_dev(flat, self.device)].cpu().numpy()
        recs = recs.reshape(-1).view(PRIM_DTYPE)
        out, k = [], 0
        for i in idx:
            out.append(recs[k:k + len(i)])
            k += len(i)
        return out

    def selected(self) -> list[list]:
        """The selected primitives of every tile as ``Cand`` objects (float32-rounded values)."""
        return [unpack_cands(r) for r in self.selected_records()]

    def bicubic_swap(self):
        """The reference fit's per-tile bicubic alternative (``bicubic_replaced_per_tile``,
        src/weft/encoder.py:2841-2873) for this fit's selections: (replace flags, u8-rounded
        control grids (n, 48), the stacks with the replaced tiles as kind-5 primitives)."""
        from . import bicubic

        stacks = self.selected()
        flags, grids, _ = bicubic.swap(self.t_src, self.t_px_off, self.t_size, stacks, self.quality)
        return flags, grids, bicubic.replaced_stacks(stacks, flags, grids)

    def stack_set(self):
        """The selected stacks as a ``refine.StackSet`` over this fit's resident tiles, with the
        parameter rows gathered on the device (no host round trip of the records)."""
        from .refine import StackSet

        n_sel = self.t_n_sel.to(torch.int64)
        counts = n_sel.cpu().numpy()
        prim_off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        sel = self.t_sel.view(self.n, self.cap_max).to(torch.int64)
        col = torch.arange(self.cap_max, device=self.device)[None, :]
        mask = col < n_sel[:, None]
        slots = (torch.from_numpy(self.pool_off).to(self.device)[:, None] + sel)[mask]
        recs = self.t_cand.view(-1, PRIM_DTYPE.itemsize)[slots]
        f = recs.view(torch.float32).view(-1, 15)
        kinds = recs.view(torch.int32)[:, 0].contiguous()
        params = torch.zeros((slots.numel(), 16), dtype=torch.float32, device=self.device)
        params[:, 0:7] = f[:, 1:8]
        params[:, 7:10] = f[:, 8:11]
        params[:, 10:13] = f[:, 11:14]
        params[:, 13] = f[:, 14]
        ss = StackSet(self.t_src, self.t_px_off, self.t_size, prim_off, kinds.cpu().numpy(), self.device.index or 0,
                      moments=self.t_moments if self.st.moments else None)
        return ss, params

    def objectives(self) -> np.ndarray:
        return self.t_cur_obj.cpu().numpy()

    def recon_tiles(self) -> list[np.ndarray]:
        """Per-tile clipped composite of the selected stacks (what the decoder renders before residuals)."""
        bg = self.t_bg.clamp(0.0, 1.0).cpu().numpy()
        out = []
        for t in range(self.n):
            s = int(self.sizes[t])
            a = int(self.px_off[t])
            out.append(bg[a:a + s * s, :3].reshape(s, s, 3))
        return out


class FitGraph:
    """``BatchedFit.run_device`` captured in one CUDA graph: every replay resets the fit and runs
    the init round, the greedy rounds and the device re-seeds with no host round trip."""

    def __init__(self, fit: BatchedFit, max_rounds: int | None = None):
        self.fit = fit
        side = torch.cuda.Stream(fit.device)
        side.wait_stream(torch.cuda.current_stream(fit.device))
        with torch.cuda.stream(side):
            fit.run_device(max_rounds)  # warm-up outside capture (lazy state, kernel attributes)
        torch.cuda.current_stream(fit.device).wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            fit.run_device(max_rounds)

    def replay(self) -> BatchedFit:
        self.graph.replay()
        return self.fit


def ctypes_ref(st) -> int:
    import ctypes

    return ctypes.addressof(st)
