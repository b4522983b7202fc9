"""Benchmark: the primitive-stack fit of a 1024x1024 synthetic image on one B200, in MPix/s at
iso RD score (PSNR - lambda * BPP) with the plain GPU fit.

Workload: the canonical synthetic image (1024x1024, 600 alpha-composited rectangles/ellipses, seed =
rank), quadtree tiles of 8-64 px split while sRGB-u8 luminance variance > 100, candidate pools from
the reference's generators (host-side, untimed, reported as ``cand_gen_s``), quality 75, at most 16
primitives per tile.  Pixels and candidate records are resident in HBM when a timed step starts.

* headline (``value``): the gradient-refined fit -- init round over the constant + linear candidates,
  then ``--refine-steps`` fused Adam steps -- replayed from one CUDA graph, reported when its RD
  (file written and decoded) is within 0.05 dB of the plain fit's or better;
* ``plain``: the reference's greedy (init, rounds, device re-seeds) for all tiles at once, replayed
  from one CUDA graph;
* also: e2e through the public API from host buffers, the FP32 rooflines of the scoring and refine
  kernels, the decoder walk at 3840x2160, the decoder's raster branch (DCT residual layer + u8
  BILINEAR resize to 3840x2160), the 2048^2 differentiable-fit workload, an RD table of
  refined-fit variants, clocks during the timed region, and the CPU baselines (the numpy oracle of the
  reference's greedy on a bounded sample of the same tiles, all host cores; the oracle decoder walk and
  raster branch on one core).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl weft|reference]

The reference arm times that CPU implementation alone.  Multi-GPU runs are independent replicas (one
image per rank), timed as the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time
from concurrent.futures import ProcessPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from weft_b200 import candidates, quadtree, rate  # noqa: E402
from weft_b200.synth import make_image_u8, srgb_u8_to_linear  # noqa: E402

METRIC = "primitive-stack fit MPix/s at iso RD score (PSNR−λ·BPP) vs plain GPU fit"
QUALITY = 75
CAP = 16


def _pool_cands(args):
    patch, q = args[:2]
    kinds = args[2] if len(args) > 2 else None
    atan2 = args[3] if len(args) > 3 else "numpy"
    from weft_b200.fit import pack_cands

    return pack_cands(candidates.tile_candidates(patch, q, kinds=kinds, atan2=atan2))


def restricted_pools(patches, kinds, executor, atan2: str = "rounded"):
    """Pools of the given kinds generated on the host (``executor`` processes), timed; with the
    device generator's float32 arctan2 rule they are the device pools' reference."""
    t0 = time.perf_counter()
    got = list(executor.map(_pool_cands, [(p, QUALITY, tuple(kinds), atan2) for p in patches], chunksize=32))
    return got, time.perf_counter() - t0


def _oracle_shard(args):
    """CPU baseline worker: the oracle greedy over a shard of tiles (with ``schedule``, the round
    decisions of the whole fit those tiles belong to); returns (seconds, selections, objectives)."""
    patches, pools, q, schedule = args
    from oracle import fit as ofit

    t0 = time.perf_counter()
    sel, cur, _ = ofit.greedy_fit(patches, [p.shape[0] for p in patches], pools, q,
                                  reseed=lambda i, patch, pred: candidates.residual_candidates(patch, pred, q),
                                  caps=[CAP] * len(patches), schedule=schedule)
    return time.perf_counter() - t0, sel, [float(v) for v in cur]


def build_workload(size: int, n_prims: int, seed: int, executor):
    u8 = make_image_u8(size, size, n_prims, seed)
    img = srgb_u8_to_linear(u8)
    tiles = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, tiles, 64)
    t0 = time.perf_counter()
    pools = list(executor.map(_pool_cands, [(p, QUALITY) for p in patches], chunksize=32))
    cand_s = time.perf_counter() - t0
    build_workload.u8 = u8  # the sRGB image the end-to-end call starts from
    return img, tiles, patches, pools, cand_s


def _cost_units(patch, pool) -> float:
    # oracle cost model: per candidate a fixed Python/numpy overhead plus per-pixel work
    return len(pool) * (1.0 + patch.shape[0] ** 2 / 512.0)


def cpu_sample(patches, pools, budget_s: float, executor, seed: int = 0):
    """Deterministic tile sample whose oracle fit takes about ``budget_s`` on all cores.

    Seconds per cost unit are calibrated on a small shard of the same tiles first.
    """
    rng = np.random.default_rng(seed)
    order = [int(i) for i in rng.permutation(len(patches))]
    cores = os.cpu_count() or 1
    calib = order[: min(len(order), 2 * cores)]
    _, wall, _ = run_cpu(patches, pools, calib, executor, cores)
    units = sum(_cost_units(patches[i], pools[i]) for i in calib)
    per_unit = wall * cores / max(units, 1e-9)
    pick, cost = [], 0.0
    for i in order:
        c = _cost_units(patches[i], pools[i]) * per_unit
        if cost + c > budget_s * cores and pick:
            break
        pick.append(i)
        cost += c
    return sorted(pick)


def run_cpu(patches, pools, pick, executor, cores: int, schedule=None, results: dict | None = None):
    """The oracle greedy over the tiles ``pick`` on ``cores`` processes; returns (MPix/s, wall
    seconds, pixels).  ``results`` (a dict) receives tile -> (selection, objective)."""
    from weft_b200.fit import unpack_cands

    shards = [s for s in (pick[k::cores] for k in range(cores)) if s]
    args = [([patches[i] for i in s], [unpack_cands(pools[i]) for i in s], QUALITY, schedule) for s in shards]
    t0 = time.perf_counter()
    out = list(executor.map(_oracle_shard, args))
    wall = time.perf_counter() - t0
    if results is not None:
        for s, (_, sel, cur) in zip(shards, out):
            results.update({t: (a, b) for t, a, b in zip(s, sel, cur)})
    px = sum(patches[i].shape[0] ** 2 for i in pick)
    return px / wall / 1e6, wall, px


def cpu_model() -> str:
    """The host CPU's model name (first processor of /proc/cpuinfo; empty when unknown)."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return ""


def fit_parity(fit, results: dict) -> dict:
    """The device fit's selections and objectives against the oracle's on the sampled tiles."""
    sel = fit.selected_indices()
    obj = fit.objectives()
    equal = sum(1 for t, (s, _) in results.items() if sel[t] == s)
    rel = max((abs(float(obj[t]) - c) / max(abs(c), 1e-30) for t, (_, c) in results.items()), default=0.0)
    return {"tiles": len(results), "equal_selections": equal, "max_obj_rel": rel,
            "what": "device plain fit vs the oracle greedy (the reference's algorithm, host re-seeding) on the "
                    "CPU baseline's sampled tiles, replaying the device fit's round decisions"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


B2B_LAUNCHES, B2B_BUFFERS = 9, 3
INIT_SAMPLES = 5

# DRAM bytes (read + write) of one init round's three scoring launches and of one refine launch
# pair (constant + tiles kernels), 1024^2 workload, from one ncu capture of the eager pipeline
INIT_ROUND_TRAFFIC = 82_512_384 + 2_255_104
REFINE_TRAFFIC = 1_919_232 + 930_048
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum, summed over the kernel's launches "
                  "(python bench.py --profile-refined --steps 1 --warmup 1)")


def decode_bench(fit, tiles, width, height, out_w, out_h, iters, peak, patches=None):
    """Decoder primitive walk of the fitted stacks at out_w x out_h (one launch renders the image),
    with each tile's RES0 offset and RES1 grid (computed from ``patches`` as the encoder does)
    when ``patches`` is given.

    Each launch is timed alone with CUDA events; a 256 MiB buffer is written between launches so the
    99.5 MB output is not served from L2, and a short GPU sleep after it keeps the stream busy while
    the host enqueues the timed launch (host launch latency is not counted).  ``back_to_back`` times
    the same launch in the steady state of a frame-after-frame decoder (rotating output buffers
    larger than L2 together, one event pair around all launches).
    """
    import ctypes

    import torch

    from weft_b200 import _lib
    from weft_b200.render import build_scene, decode_items

    class _Rec:
        __slots__ = ("primitives", "residual_rgb")

        def __init__(self, p):
            self.primitives = p
            self.residual_rgb = (0, 0, 0)

    recs = [_Rec(s) for s in fit.selected()]
    maps = None
    if patches is not None:
        from weft_b200.encode import residuals_from_recon

        res0, res1 = residuals_from_recon(patches, fit.recon_tiles())
        for r, v in zip(recs, res0):
            r.residual_rgb = v
        maps = [g.astype(np.float32) / np.float32(255.0) for g in res1]
    descs, prims, cp48, res1_tab, th, tw = build_scene(recs, tiles, width, height, maps, out_w, out_h)
    dev = torch.device("cuda", torch.cuda.current_device())
    t_d = torch.from_numpy(descs.view(np.uint8)).to(dev)
    t_p = torch.from_numpy(prims.view(np.uint8)).to(dev)
    t_c = torch.from_numpy(np.ascontiguousarray(cp48)).to(dev)
    n_res1 = 0 if res1_tab is None else len(res1_tab)
    t_r = torch.from_numpy(np.ascontiguousarray(res1_tab)).to(dev) if n_res1 else None
    out = torch.empty((th, tw, 3), dtype=torch.float32, device=dev)
    items = decode_items(descs, th, tw, prims)
    t_i = torch.from_numpy(items).to(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    lib = _lib.lib_for_device(dev.index)
    stream = torch.cuda.current_stream()

    def launch(o=out):
        _lib.check(lib.weftk_render_tiles(_lib.ptr(t_d), len(descs), _lib.ptr(t_i), len(items), _lib.ptr(t_p),
                                          _lib.ptr(t_c), len(cp48), _lib.ptr(t_r) if n_res1 else 0, n_res1,
                                          _lib.ptr(o), th, tw, 0,
                                          stream.cuda_stream), "weftk_render_tiles")

    for _ in range(3):
        launch()
    times = []
    for _ in range(iters):
        flush.fill_(1.0)
        torch.cuda._sleep(100000)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        launch()
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    # reference: a plain streaming write of the same output buffer, timed the same way
    fill_times = []
    for _ in range(max(iters, 3)):
        flush.fill_(1.0)
        torch.cuda._sleep(100000)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        out.fill_(0.5)
        b.record(stream)
        torch.cuda.synchronize()
        fill_times.append(a.elapsed_time(b))
    fill_ms = statistics.median(fill_times)
    # steady state, as a decoder rendering one frame after another: B2B_LAUNCHES launches back to
    # back into three rotating output buffers (3 x 99.5 MB at 3840x2160, more than L2, so no
    # launch finds its buffer in L2), one event pair around all of them; the fixed cost of an event
    # pair and a launch (an empty kernel measures about 6 us this way) is paid once, not per launch
    outs = [out] + [torch.empty_like(out) for _ in range(B2B_BUFFERS - 1)]
    b2b, b2b_fill = [], []
    for _ in range(max(3, iters // 2)):
        for fn, acc in ((launch, b2b), (lambda o: o.fill_(0.5), b2b_fill)):
            flush.fill_(1.0)
            torch.cuda._sleep(1000000)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for i in range(B2B_LAUNCHES):
                fn(outs[i % B2B_BUFFERS])
            b.record(stream)
            torch.cuda.synchronize()
            acc.append(a.elapsed_time(b) / B2B_LAUNCHES)
    del outs
    launch()  # the timed output, not the fill, is what the status check follows
    torch.cuda.synchronize()
    st = ctypes.c_int(0)
    _lib.check(lib.weftk_device_status(ctypes.addressof(st)), "weftk_device_status")
    if st.value:
        raise RuntimeError("decode walk reported a bad descriptor")
    ms = statistics.median(times)
    nbytes = 12 * tw * th + 48 * len(descs) + 60 * len(prims) + 192 * n_res1
    gbs = nbytes / (ms * 1e-3) / 1e9
    peak_gbs, peak_source = peak
    return {"target": f"{tw}x{th}", "ms": ms, "mpix_per_s": tw * th / (ms * 1e-3) / 1e6, "bytes": nbytes,
            "achieved_gbs": gbs, "peak_gbs": peak_gbs, "frac": gbs / peak_gbs,
            "peak_source": peak_source,
            "fill_reference": {"ms": fill_ms, "gbs": 12 * tw * th / (fill_ms * 1e-3) / 1e9,
                               "what": "torch fill_ of the same output buffer, timed the same way"},
            "frac_of_fill": (12 * tw * th / (ms * 1e-3)) / (12 * tw * th / (fill_ms * 1e-3)),
            "back_to_back": {"ms": statistics.median(b2b), "frac": nbytes / (statistics.median(b2b) * 1e-3) / 1e9 / peak_gbs,
                             "fill_ms": statistics.median(b2b_fill), "launches": B2B_LAUNCHES,
                             "buffers": B2B_BUFFERS,
                             "what": "launches back to back into rotating output buffers larger than L2 together, "
                                     "one event pair around them; ms per launch"},
            "l2": "256 MiB written between timed launches", "tiles": len(descs), "prims": int(len(prims)),
            "residuals": "RES0 + RES1 grids" if n_res1 else "none"}


def pinned_copy(a: np.ndarray, keep: list) -> np.ndarray:
    """A copy of ``a`` in page-locked host memory (its torch buffer is appended to ``keep``)."""
    import torch

    buf = torch.empty(max(a.nbytes, 1), dtype=torch.uint8, pin_memory=True)
    keep.append(buf)
    out = buf.numpy()[:a.nbytes].view(a.dtype).reshape(a.shape)
    out[...] = a
    return out


def synthetic_dct_block(tiles, quality: int, seed: int = 0) -> bytes:
    """A BLOCK_DCT (format v5) covering every tile, in the reference encoder's default configuration
    (YCbCr 4:2:0, frequency-weight alpha 4.0, tile-major layout, the quality's quant step): seeded
    Laplacian coefficients whose scale falls with frequency, 6 / (1 + u + v), as a residual's do."""
    import struct

    rng = np.random.default_rng(seed)
    parts = []
    for t in tiles:
        for n in (t.size, t.size // 2, t.size // 2):
            f = np.arange(n, dtype=np.float64)
            scale = 6.0 / (1.0 + f[:, None] + f[None, :])
            parts.append(np.clip(np.round(rng.laplace(0.0, scale)), -32768, 32767).astype("<i2").reshape(-1))
    coeffs = np.concatenate(parts)
    q = max(10, min(99, int(quality)))
    step = float(max(0.003, min(0.20, ((101 - q) / 100.0) ** 2 * 0.20)))
    n = len(tiles)
    mask = np.packbits(np.ones(n, np.uint8), bitorder="little").tobytes()
    head = struct.pack("<BBBBffHIII", 5, 2, 0, 0, step, 4.0, 3, n, coeffs.size, 0)
    return head + mask + coeffs.tobytes()


def raster_bench(fit, tiles, patches, size, out_w, out_h, iters, peak):
    """The decoder's raster branch (a file with a DCT residual layer, decoded at another size): walk at
    the encoded size, DCT layer, u8 + BILINEAR resize, on a synthetic DCT block over every tile."""
    import ctypes

    import torch

    from weft_b200 import _lib, raster
    from weft_b200.encode import residuals_from_recon
    from weft_b200.render import build_scene, decode_items

    class _Rec:
        __slots__ = ("primitives", "residual_rgb")

        def __init__(self, p, r):
            self.primitives, self.residual_rgb = p, r

    res0, res1 = residuals_from_recon(patches, fit.recon_tiles())
    recs = [_Rec(st, r) for st, r in zip(fit.selected(), res0)]
    maps = [g.astype(np.float32) / np.float32(255.0) for g in res1]
    descs, prims, cp48, res1_tab, th, tw = build_scene(recs, tiles, size, size, maps)
    dev = torch.device("cuda", torch.cuda.current_device())
    lib = _lib.lib_for_device(dev.index)
    stream = torch.cuda.current_stream()
    t_d = torch.from_numpy(descs.view(np.uint8)).to(dev)
    t_p = torch.from_numpy(prims.view(np.uint8)).to(dev)
    t_c = torch.from_numpy(np.ascontiguousarray(cp48)).to(dev) if len(cp48) else None
    t_r = torch.from_numpy(np.ascontiguousarray(res1_tab)).to(dev)
    items = decode_items(descs, th, tw, prims)
    t_i = torch.from_numpy(items).to(dev)
    img = torch.zeros((th, tw, 3), dtype=torch.float32, device=dev)
    base = torch.empty_like(img)
    out = torch.empty((out_h, out_w, 3), dtype=torch.float32, device=dev)
    tmp = torch.empty(th * out_w * 3, dtype=torch.uint8, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    layer = raster.DctLaunch.from_payload(synthetic_dct_block(tiles, QUALITY), [(t.x, t.y, t.size) for t in tiles],
                                          tw, th, dev.index)

    def walk():
        _lib.check(lib.weftk_render_tiles(_lib.ptr(t_d), len(descs), _lib.ptr(t_i), len(items), _lib.ptr(t_p),
                                          _lib.ptr(t_c), len(cp48), _lib.ptr(t_r), len(res1_tab), _lib.ptr(img),
                                          th, tw, 0, stream.cuda_stream), "weftk_render_tiles")

    def timed(fn, prep=None):
        for _ in range(3):
            if prep:
                prep()
            fn()
        times = []
        for _ in range(iters):
            if prep:
                prep()
            flush.fill_(1.0)
            torch.cuda._sleep(100000)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
        return statistics.median(times)

    st = ctypes.c_int(0)
    lib.weftk_device_status(ctypes.addressof(st))
    walk()
    base.copy_(img)
    apply_ms = timed(lambda: layer.run(img, stream.cuda_stream), prep=lambda: img.copy_(base))
    resize_ms = timed(lambda: raster.resize_into(img, out, tmp, stream.cuda_stream))

    def whole():
        walk()
        layer.run(img, stream.cuda_stream)
        raster.resize_into(img, out, tmp, stream.cuda_stream)

    whole_ms = timed(whole)
    torch.cuda.synchronize()
    _lib.check(lib.weftk_device_status(ctypes.addressof(st)), "weftk_device_status")
    if st.value:
        raise RuntimeError("the raster branch reported a bad descriptor")
    rbytes = 12 * tw * th + 2 * 3 * th * out_w + 12 * out_w * out_h
    gbs = rbytes / (resize_ms * 1e-3) / 1e9
    peak_gbs, peak_source = peak
    return {"encoded": f"{tw}x{th}", "target": f"{out_w}x{out_h}", "ms": whole_ms,
            "mpix_per_s": out_w * out_h / (whole_ms * 1e-3) / 1e6,
            "launches": 1 + layer.launches + 2,
            "dct_apply": {"ms": apply_ms, "tiles": len(layer.descs), "coefficients": int(layer.block.coeffs.size),
                          "fp64_flops": layer.flops(), "fp64_tflops": layer.flops() / (apply_ms * 1e-3) / 1e12,
                          "launches": layer.launches},
            "resize": {"ms": resize_ms, "bytes": rbytes, "achieved_gbs": gbs, "peak_gbs": peak_gbs,
                       "frac": gbs / peak_gbs, "peak_source": peak_source},
            "payload": "synthetic BLOCK_DCT v5 over every tile (4:2:0, alpha 4, q75 step, Laplacian coefficients)",
            "l2": "256 MiB written between timed launches"}


def cpu_decode_baselines(fit, tiles, patches, size, out_w, out_h) -> tuple[dict, dict]:
    """CPU baselines of the two decode lines, one process each (the reference decoder is single
    threaded numpy): the oracle's analytic walk at the output size (no residual grids, like the
    ``decode`` line), and the raster branch of ``decode_raster`` -- oracle walk at the encoded size with
    RES0/RES1, oracle DCT layer on the same synthetic block, then u8 and Pillow's own BILINEAR resize."""
    from PIL import Image

    from oracle import dct as odct
    from oracle import render as orender
    from weft_b200.encode import residuals_from_recon

    class _Rec:
        __slots__ = ("primitives", "residual_rgb")

        def __init__(self, p, r):
            self.primitives, self.residual_rgb = p, r

    sel = fit.selected()
    t0 = time.perf_counter()
    orender.render_scene_adaptive([_Rec(st, (0, 0, 0)) for st in sel], tiles, size, size, None, 4, out_w, out_h)
    walk_s = time.perf_counter() - t0
    res0, res1 = residuals_from_recon(patches, fit.recon_tiles())
    maps = [g.astype(np.float32) / np.float32(255.0) for g in res1]
    payload = synthetic_dct_block(tiles, QUALITY)
    t0 = time.perf_counter()
    img = orender.render_scene_adaptive([_Rec(st, r) for st, r in zip(sel, res0)], tiles, size, size, maps, 4)
    img = odct.apply_dct_block(img, payload, [(t.x, t.y, t.size) for t in tiles])
    u8 = np.clip(img * np.float32(255.0), 0.0, 255.0).astype(np.uint8)
    np.asarray(Image.fromarray(u8).resize((out_w, out_h), Image.BILINEAR), dtype=np.float32) / np.float32(255.0)
    raster_s = time.perf_counter() - t0
    px = out_w * out_h
    walk = {"value": px / walk_s / 1e6, "unit": "MPix/s", "ms": walk_s * 1e3, "cores": 1, "kind": "port",
            "sample": f"oracle render_scene_adaptive of the whole scene at {out_w}x{out_h}, one process"}
    raster = {"value": px / raster_s / 1e6, "unit": "MPix/s", "ms": raster_s * 1e3, "cores": 1, "kind": "port",
              "sample": f"oracle walk at {size}x{size} with RES0/RES1 + oracle DCT layer + Pillow BILINEAR to "
                        f"{out_w}x{out_h}, one process"}
    return walk, raster


def _recon_of(stack_set, params, tiles, size):
    """Per-tile clipped renders of parameter rows (no residuals), via the GPU decoder walk."""
    from weft_b200 import render

    class _R:
        def __init__(self, p):
            self.primitives = p
            self.residual_rgb = (0, 0, 0)

    stacks = stack_set.to_stacks(params)
    pw = ((size + 63) // 64) * 64
    full = render.render_scene_adaptive([_R(s) for s in stacks], tiles, pw, pw)
    return stacks, [full[t.y:t.y + t.size, t.x:t.x + t.size] for t in tiles]


REFINE_POOLS = {"nocurve": (0, 1, 2, 4, 5), "smooth": (0, 1, 2), "constlin": (0, 1)}


def rd_of_params(ss, params, tiles, patches, img, size) -> dict:
    """RD of refined parameter rows written as a WEFT file (quantised rows, RES0/RES1 from
    their render) and decoded."""
    from weft_b200.encode import encode_fit, rd_score

    q = ss.quantize(params)
    recon = _recon_of(ss, q, tiles, size)[1]
    return rd_score(img, encode_fit(size, size, QUALITY, tiles, patches, ss.to_stacks(q), recon), QUALITY)


def rd_compare(args, fit, tiles, patches, pools, img, stream):
    """RD of the plain fit vs refined fast fits, both written as WEFT files the same way
    (quantised primitives, RES0/RES1 from the render of the quantised primitives) and
    decoded; RD = PSNR - 4 BPP.

    A refined fast fit scores only the init round over a kind-filtered pool (best single
    candidate per tile), then runs fused Adam steps on that primitive; the whole pipeline
    is one CUDA graph.  Times are CUDA-event device times of a graph replay, state
    resident, after warm-up (mean of ``--refine-reps`` replays).
    """
    import torch

    from weft_b200.fit import BatchedFit
    from weft_b200.refine import RefinedFit

    size = args.size
    n_px = size * size
    plain_stacks = fit.selected()
    plain = rd_of_params(*fit.stack_set(), tiles, patches, img, size)
    pixels = np.concatenate([p.reshape(-1, 3) for p in patches])
    sizes = np.array([p.shape[0] for p in patches], np.int32)
    variants = []
    for spec in args.refine_variants.split(","):
        name, steps, *opt = spec.split(":")
        residual = "r" in opt
        keep = REFINE_POOLS[name]
        fast_pools = [p[np.isin(p["kind"], keep)] for p in pools]
        fast = BatchedFit.from_arrays(pixels, sizes, np.concatenate(fast_pools),
                                      np.array([len(p) for p in fast_pools], np.int64), QUALITY,
                                      caps=[CAP] * len(patches), device=torch.cuda.current_device(), reserve=0)
        rf = RefinedFit(fast, steps=int(steps), lr=args.refine_lr, use_graph=True, residual=residual)
        for _ in range(2):
            rf.run()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.refine_reps):
            out = rf.run()
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / args.refine_reps
        ss = rf.ss
        sc = rd_of_params(ss, out, tiles, patches, img, size)
        variants.append({"pool": name, "kinds": list(keep), "adam_steps": int(steps),
                         "loss": "decoded (after residual grid)" if residual else "primitives only", **sc, "ms": ms,
                         "mpix_per_s": n_px / (ms * 1e-3) / 1e6, "rd_delta_db": sc["rd_score"] - plain["rd_score"]})
        del rf, fast
    return {"plain": {**plain, "prims": sum(len(s) for s in plain_stacks)}, "lr": args.refine_lr,
            "refined": variants,
            "init": "best single candidate per tile from the kind-filtered pool, no greedy rounds"}


# FP32 operations per pixel and layer of one refine step (loss + gradient + Adam is
# negligible per pixel): the forward composite evaluates the layer (the scoring kernel's
# per-kind count) and blends it (9), the backward re-evaluates it and chains the gradient
# (per-kind count of the chain rule in layer_grad), plus 9 per pixel for the loss.
REFINE_EVAL = {0: 10, 1: 24, 2: 28, 3: 509, 4: 26, 5: 0}
REFINE_CHAIN = {0: 12, 1: 45, 2: 40, 3: 60, 4: 40, 5: 0}


def refine_flops(stack_set) -> float:
    """FP32 operations of one refine launch over the stack set."""
    import torch

    kinds = stack_set.t_kind.cpu().numpy()
    off = stack_set.prim_off_np
    px = (stack_set.sizes.to(torch.int64) ** 2).cpu().numpy().astype(np.float64)
    per_row = np.array([2 * REFINE_EVAL.get(int(k), 0) + 9 + REFINE_CHAIN.get(int(k), 0) for k in kinds], np.float64)
    starts = np.minimum(off[:-1], max(len(per_row) - 1, 0))
    tile_cost = np.add.reduceat(per_row, starts) if len(per_row) else np.zeros(len(px))
    tile_cost[np.diff(off) == 0] = 0.0
    return float((px * (tile_cost + 9.0)).sum())


def refined_headline(args, local, pixels, sizes, pools, stream, world):
    """The gradient-refined batched fit: init round over the kind-filtered pool, then
    ``--refine-steps`` fused Adam steps, replayed from one CUDA graph.  Each timed step is
    preceded by a 256 MiB write (the step's working set fits in L2) and a short GPU sleep
    (host launch latency is not counted)."""
    import torch

    from weft_b200.fit import BatchedFit
    from weft_b200.refine import RefinedFit

    keep = REFINE_POOLS[args.refine_pool]
    fast_pools = [p[np.isin(p["kind"], keep)] for p in pools]
    rec = np.concatenate(fast_pools)
    cnt = np.array([len(p) for p in fast_pools], np.int64)
    fast = BatchedFit.from_arrays(pixels, sizes, rec, cnt, QUALITY, caps=[CAP] * len(sizes), device=local, reserve=0)
    fast.use_closed_form_init(True)
    fast.autotune()
    rf = RefinedFit(fast, steps=args.refine_steps, lr=args.refine_lr, use_graph=True)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")
    for _ in range(args.warmup):
        rf.run()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda._sleep(100000)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rf.run()
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    del flush
    return rf, fast, rec, cnt, statistics.mean(times)


def device_headline(args, fit, sizes, caps, stream, world, generate_in_run: bool):
    """The refined fit over pools generated on the device: (with ``generate_in_run``) pool
    generation, then init round, fused Adam steps and wire-grid snap replayed from one CUDA graph over
    the resident tiles; without it the pools are generated once beforehand and stay resident.  Each
    timed step is preceded by a 256 MiB write and a short GPU sleep (host launch latency not
    counted)."""
    import torch

    from weft_b200.pools import DeviceRefinedFit

    drf = DeviceRefinedFit(fit.t_src, sizes, QUALITY, caps=caps, steps=args.refine_steps, lr=args.refine_lr,
                           generate_in_run=generate_in_run)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=fit.device)
    for _ in range(args.warmup):
        drf.run()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda._sleep(100000)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        drf.run()
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    return drf, statistics.mean(times)


def device_breakdown(args, drf, lib, stream) -> dict:
    """Eager run of the device pipeline with CUDA events around its parts: pool generation, the
    init round's scoring kernels (events inside the library), the Adam steps."""
    import ctypes

    import torch

    def ev():
        return torch.cuda.Event(enable_timing=True)

    torch.cuda.synchronize()
    a, b = ev(), ev()
    a.record(stream)
    drf.generate()
    b.record(stream)
    torch.cuda.synchronize()
    gen_ms = a.elapsed_time(b)
    # the init round's scoring launches, median of INIT_SAMPLES eager runs (each run resets the
    # fit and its work counters, so every sample is one round)
    samples = []
    for _ in range(INIT_SAMPLES):
        lib.weftk_fit_timing(1, None, None)
        drf.fit.run_init_only()
        torch.cuda.synchronize()
        score_ms, n_score = ctypes.c_double(0), ctypes.c_int(0)
        lib.weftk_fit_timing(0, ctypes.addressof(score_ms), ctypes.addressof(n_score))
        samples.append(score_ms.value)
    fr = drf.rf.refiner
    fr.restart(drf.rf.start)
    torch.cuda.synchronize()
    a, b = ev(), ev()
    a.record(stream)
    fr.run(args.refine_steps)
    b.record(stream)
    torch.cuda.synchronize()
    return {"gen_ms": gen_ms, "init_score_ms": statistics.median(samples), "init_score_samples": samples,
            "init_score_launches": n_score.value,
            "refine_ms": a.elapsed_time(b), "work": drf.fit.work_counters()}


def refined_breakdown(args, rf, fast, lib, stream):
    """Eager run of the same pipeline: scoring-kernel time of the init round (events inside
    the library) and the mean refine-step kernel time (events around the steps)."""
    import ctypes

    import torch

    lib.weftk_fit_timing(1, None, None)
    fast.run_init_only()
    torch.cuda.synchronize()
    score_ms, n_score = ctypes.c_double(0), ctypes.c_int(0)
    lib.weftk_fit_timing(0, ctypes.addressof(score_ms), ctypes.addressof(n_score))
    fr = rf.refiner
    fr.restart(rf.start)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    fr.run(args.refine_steps)
    b.record(stream)
    torch.cuda.synchronize()
    step_ms = a.elapsed_time(b) / max(args.refine_steps, 1)
    return score_ms.value, n_score.value, step_ms, fast.work_counters()


def differentiable_fit(args, executor, local, stream):
    """The differentiable-fit workload: a 2048x2048 synthetic image of 2500 primitives, the plain
    batched fit, then ``--diff-steps`` Adam steps (lr 1e-2, FP32 parameters and moments) on the
    fitted stacks through the autograd.Function (torch Adam) and, separately, through the fused
    one-launch step; RD of the files before and after."""
    import torch

    from weft_b200.batch import ImageBatch, prepare_image
    from weft_b200.refine import FusedRefiner, refine

    size, n_prims = 2048, 2500
    t0 = time.perf_counter()
    im = prepare_image(make_image_u8(size, size, n_prims, 0), QUALITY, executor)
    cand_s = time.perf_counter() - t0
    batch = ImageBatch([im], QUALITY, CAP, device=local)
    fit = batch.plain_fit()

    def timed(fn):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r = fn()
        b.record(stream)
        torch.cuda.synchronize()
        return r, a.elapsed_time(b)

    fit.reset()
    fit.run()  # warm-up
    fit.reset()
    _, plain_ms = timed(fit.run)
    parity = None
    if not args.no_cpu:
        # the plain fit's selections against the oracle greedy on a sample of the tiles, replaying
        # the device fit's round decisions (as the 1024^2 line's parity)
        schedule = [imp > 0 for mode, ev, imp in fit.stats.per_round if mode == 1 and ev > 0]
        pick = cpu_sample(im.patches, im.pools, 2.0, executor, seed=1)
        results: dict = {}
        run_cpu(im.patches, im.pools, pick, executor, os.cpu_count() or 1, schedule, results)
        parity = {k: v for k, v in fit_parity(fit, results).items() if k != "what"}
    ss, p0 = fit.stack_set()
    steps = args.diff_steps
    refine(ss, p0, steps=3, lr=1e-2)  # warm-up
    (out, hist), auto_ms = timed(lambda: refine(ss, p0, steps=steps, lr=1e-2))
    fr = FusedRefiner(ss, p0, lr=1e-2)
    fr.run(3)
    fr.restart(p0)
    _, fused_ms = timed(lambda: fr.run(steps))
    rd0 = batch.rd_per_image(ss.to_stacks(ss.quantize(p0)))[0]
    rd1 = batch.rd_per_image(ss.to_stacks(ss.quantize(out)))[0]
    return {"image": f"{size}x{size}, {n_prims} prims, seed 0", "tiles": len(im.tiles),
            "stack_rows": int(p0.shape[0]), "max_prims": ss.max_prims, "cand_gen_s": cand_s,
            "plain_fit_ms": plain_ms, "adam_steps": steps, "lr": 1e-2,
            "autograd_ms_per_step": auto_ms / steps, "fused_ms_per_step": fused_ms / steps,
            "loss_first_last": [hist[0], hist[-1]] if hist else None,
            "rd_plain": rd0["rd_score"], "rd_refined": rd1["rd_score"], "rd_delta_db": rd1["rd_score"] - rd0["rd_score"],
            "psnr_plain_db": rd0["psnr_db"], "psnr_refined_db": rd1["psnr_db"], "parity": parity}


def image_batch_fit(args, executor, local, stream):
    """The multi-image workload (``--batch-images``, e.g. "16x256,16x512,16x1024,16x2048"): images
    of the canonical generator (seeds 0.., primitives rising from 50 to 2500 over the list), all tiles in one
    plain batched fit and in one refined fit; MPix/s of both and each image's RD."""
    import torch

    from weft_b200.batch import ImageBatch, prepare_image

    specs = []
    for part in args.batch_images.split(","):
        n, side = part.lower().split("x")
        specs += [int(side)] * int(n)
    ims = []
    t0 = time.perf_counter()
    for seed, side in enumerate(specs):
        # image i of n: 50 + 2450 i / (n - 1) primitives (50 .. 2500; seeds 0 .. n - 1)
        n_prims = 50 + (2450 * seed) // max(1, len(specs) - 1)
        ims.append(prepare_image(make_image_u8(side, side, n_prims, seed), QUALITY, executor))
    cand_s = time.perf_counter() - t0
    batch = ImageBatch(ims, QUALITY, CAP, device=local)
    n_px = batch.n_pixels

    def timed(fn, reps=1):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            r = fn()
        b.record(stream)
        torch.cuda.synchronize()
        return r, a.elapsed_time(b) / reps

    fit = batch.plain_fit()
    fit.run()

    def plain_step():
        fit.reset()
        fit.run()

    _, plain_ms = timed(plain_step)
    ss, p = fit.stack_set()
    plain_rd = batch.rd_per_image(ss.to_stacks(ss.quantize(p)))
    del fit, ss, p
    drf = batch.refined_fit_device(steps=args.batch_steps, lr=args.refine_lr)
    drf.run()
    rows, ref_ms = timed(drf.run, 3)
    rss = drf.rf.ss
    ref_rd = batch.rd_per_image(rss.to_stacks(rss.quantize(drf.rf.refiner.p)))
    deltas = [b["rd_score"] - a["rd_score"] for a, b in zip(plain_rd, ref_rd)]
    per_image = [{"side": im.size[0], "plain_rd": a["rd_score"], "refined_rd": b["rd_score"]}
                 for im, a, b in zip(ims, plain_rd, ref_rd)]
    return {"images": args.batch_images, "n_images": len(ims), "mpix": n_px / 1e6, "tiles": int(batch.tile_off[-1]),
            "cand_gen_s": cand_s, "plain_ms": plain_ms, "plain_mpix_per_s": n_px / (plain_ms * 1e-3) / 1e6,
            "refined_ms": ref_ms, "refined_mpix_per_s": n_px / (ref_ms * 1e-3) / 1e6,
            "refined": f"pools generated on the device (constant + linear), init round + {args.batch_steps} fused "
                       f"Adam steps + wire-grid snap, one CUDA graph over every tile of every image",
            "rd_delta_db_min": min(deltas), "rd_delta_db_mean": float(np.mean(deltas)),
            "images_within_0.05db": int(sum(d >= -0.05 for d in deltas)), "per_image": per_image}


def _hbm_peak() -> tuple[float, str]:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured copy)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s (earlier measurement on this pool)"


def workload_name(args) -> str:
    """The workload both arms run (the same string in both JSON lines)."""
    return (f"{args.size}x{args.size} synthetic, {args.prims} prims, quadtree 8-64 px (u8 lum variance > 100), "
            f"q=75, cap {CAP}, the reference's candidate pools")


def bench_config(args, n_tiles: int, n_candidates: int) -> dict:
    """The ``config`` object, identical in both arms' lines (what each arm fits is under ``fit``)."""
    return {"workload": workload_name(args), "tiles": n_tiles, "candidates": n_candidates, "global_batch": args.gpus,
            "seq_len": 0, "parallelism": f"replicas x{args.gpus}"}


def max_over_ranks(x: float, world: int) -> float:
    """The slowest rank's time (every rank calls this at the same point)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl" if n_gpus > 0 else "gloo", timeout=datetime.timedelta(seconds=600),
                                device_id=None)
    return world, rank, local


def reference_arm(args, world, rank, executor):
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    img, tiles, patches, pools, _ = build_workload(args.size, args.prims, 0, executor)
    pick = cpu_sample(patches, pools, args.ref_step_s, executor)
    for _ in range(args.warmup):
        run_cpu(patches, pools, pick[: max(1, len(pick) // 8)], executor, cores)
    vals = []
    walls = []
    for _ in range(args.steps):
        v, wall, px = run_cpu(patches, pools, pick, executor, cores)
        vals.append(v)
        walls.append(wall)
    value = sum(px for _ in vals) / sum(walls) / 1e6 if walls else 0.0
    sample = f"{len(pick)} of {len(tiles)} tiles ({px / 1e6:.3f} MPix) of the {args.size}^2 workload per step"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "MPix/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(walls),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(args, len(tiles), int(sum(len(p) for p in pools))),
        "fit": "the reference's plain greedy (init, rounds, residual re-seeds), the oracle's restatement on "
               "all host cores; its RD is the iso-RD target",
        "cpu_baseline": {"value": value, "unit": "MPix/s", "cores": cores, "kind": "port", "sample": sample,
                         "cpu": cpu_model()},
        "e2e": {"value": value, "unit": "MPix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="weft", choices=["weft", "reference"])
    ap.add_argument("--size", type=int, default=1024)
    ap.add_argument("--prims", type=int, default=600)
    ap.add_argument("--cpu-budget-s", type=float, default=8.0)
    ap.add_argument("--ref-step-s", type=float, default=8.0)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling runs)")
    ap.add_argument("--decode-iters", type=int, default=10)
    ap.add_argument("--refine-pool", default="constlin", choices=sorted(REFINE_POOLS),
                    help="candidate kinds the refined fit's init round scores")
    ap.add_argument("--refine-steps", type=int, default=10, help="Adam steps of the refined fit")
    ap.add_argument("--refine-variants", default="constlin:0,constlin:10,constlin:20,constlin:20:r,nocurve:20:r",
                    help="refined fits whose RD is reported, pool:adam_steps[:r] (r: decoded-error loss)")
    ap.add_argument("--refine-reps", type=int, default=5)
    ap.add_argument("--refine-lr", type=float, default=1e-2)
    ap.add_argument("--diff-steps", type=int, default=200,
                    help="Adam steps of the 2048^2 differentiable fit (0: skip that workload)")
    ap.add_argument("--batch-images", default="",
                    help='multi-image batch, e.g. "16x256,16x512,16x1024,16x2048" (empty: skip)')
    ap.add_argument("--batch-steps", type=int, default=100, help="Adam steps of the multi-image refined fit")
    ap.add_argument("--batch-only", action="store_true",
                    help="only the multi-image batch (--batch-images, default the 64-image set), one JSON line")
    ap.add_argument("--profile-refined", action="store_true",
                    help="only the refined fit with device pool generation (eager launches), for profilers")
    args = ap.parse_args()

    # Process pools first: spawned before any CUDA initialisation.
    cores = os.cpu_count() or 1
    executor = ProcessPoolExecutor(max_workers=cores, mp_context=mp.get_context("spawn"))
    world, rank, local = dist_setup(args.gpus if args.impl == "weft" else 0)
    try:
        if args.impl == "reference":
            reference_arm(args, world, rank, executor)
            return
        run_weft(args, world, rank, local, executor, cores)
    finally:
        executor.shutdown(wait=True, cancel_futures=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


def profile_refined(args, local, patches):
    """The refined fit with its pools generated on the device, eager launches only (no CUDA graph,
    no host-generated pools): what a kernel profiler should see of the headline pipeline."""
    import torch

    from weft_b200.pools import DeviceRefinedFit

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pixels = np.concatenate([p.reshape(-1, 3) for p in patches])
    sizes = np.array([p.shape[0] for p in patches], np.int32)
    src4 = torch.zeros((len(pixels), 4), dtype=torch.float32, device=dev)
    src4[:, :3] = torch.from_numpy(pixels).to(dev)
    drf = DeviceRefinedFit(src4, sizes, QUALITY, caps=[CAP] * len(sizes), steps=args.refine_steps,
                           lr=args.refine_lr, use_graph=False, autotune=False)
    for _ in range(args.warmup + args.steps):
        drf.run()
    torch.cuda.synchronize()
    print(json.dumps({"profile_refined": {"tiles": len(sizes), "steps": args.warmup + args.steps}}), flush=True)


def batch_only(args, local, executor, cores):
    """The multi-image workload alone: 64 images (16 each of 256^2, 512^2, 1024^2, 2048^2) unless
    --batch-images names another set; all tiles in one plain fit and one refined fit."""
    import torch

    torch.cuda.set_device(local)
    if not args.batch_images:
        args.batch_images = "16x256,16x512,16x1024,16x2048"
    stream = torch.cuda.current_stream()
    sampler = ClockSampler(local)
    sampler.start()
    r = image_batch_fit(args, executor, local, stream)
    clocks = sampler.stop()
    iso = r["images_within_0.05db"] == r["n_images"]
    print(json.dumps({"metric": METRIC, "value": r["refined_mpix_per_s"] if iso else r["plain_mpix_per_s"],
                      "unit": "MPix/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
                      "config": {"workload": f"multi-image batch {r['images']}, seeds 0..{r['n_images'] - 1}, "
                                             f"q=75, cap {CAP}", "tiles": r["tiles"], "mpix": r["mpix"]},
                      "clocks": clocks, "host_processes": cores, "image_batch": r}), flush=True)


def run_weft(args, world, rank, local, executor, cores):
    import torch

    if args.batch_only:
        batch_only(args, local, executor, cores)
        return
    if args.profile_refined:
        u8 = make_image_u8(args.size, args.size, args.prims, rank)
        img = srgb_u8_to_linear(u8)
        tiles = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
        profile_refined(args, local, quadtree.extract_tiles(img, tiles, 64))
        return
    img, tiles, patches, pools, cand_s = build_workload(args.size, args.prims, rank, executor)

    torch.cuda.set_device(local)
    from weft_b200 import _lib
    from weft_b200.fit import BatchedFit

    lib = _lib.lib_for_device(local)
    # flat host inputs of the public API (what a caller hands over)
    pixels = np.concatenate([p.reshape(-1, 3) for p in patches])
    sizes = np.array([p.shape[0] for p in patches], np.int32)
    records = np.concatenate(pools)
    counts = np.array([len(p) for p in pools], np.int64)
    caps = [CAP] * len(patches)
    fit = BatchedFit.from_arrays(pixels, sizes, records, counts, QUALITY, caps=caps, device=local)
    tuned_plain = fit.autotune()  # scoring shape and candidates per CTA per tile-size class
    n_px = int(sum(p.shape[0] ** 2 for p in patches))
    stream = torch.cuda.current_stream()

    # the whole greedy fit (init, rounds, device re-seeds) replayed from one CUDA graph
    fit_graph = fit.graph()
    for _ in range(args.warmup):
        fit_graph.replay()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_classes = sum(1 for k in (8, 16, 32) if fit.n_items[k])
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        fit_graph.replay()
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ctl = fit.control()
    max_rounds = rate.max_rounds(QUALITY)
    # kernels per step: reset, prepare; init round: begin, scoring per class, select, end; every
    # greedy round (run or skipped): begin, scoring per class, select, end, control, re-seed; the
    # selected stacks snapped to the wire grid
    launches_per_step = 2 + (3 + n_classes) + max_rounds * (5 + n_classes) + 1
    import ctypes

    ms_total = ev0.elapsed_time(ev1)
    ms_step = ms_total / args.steps
    ms_step = max_over_ranks(ms_step, world)
    value = world * n_px / (ms_step * 1e-3) / 1e6
    # scoring-kernel time: one host-driven run of the same fit with events around the scoring
    # launches (the graph cannot host-synchronise); the same kernels and work
    fit.reset()
    lib.weftk_fit_timing(1, None, None)
    fit.run()
    torch.cuda.synchronize()
    score_ms = ctypes.c_double(0)
    n_score = ctypes.c_int(0)
    lib.weftk_fit_timing(0, ctypes.addressof(score_ms), ctypes.addressof(n_score))
    work = [fit.work_counters()]
    rounds = [len(fit.stats.per_round)]
    # the device fit's round decisions (a greedy round ran with evaluated tiles: did any improve?),
    # replayed by the oracle on the CPU baseline's sampled tiles for the parity check
    schedule = [imp > 0 for mode, ev, imp in fit.stats.per_round if mode == 1 and ev > 0]
    score_ms.value *= args.steps  # per-step figures below divide by the step count

    # roofline of the scoring kernels (FP32-bound): algorithmic ops / scoring device time
    ops = sum(w[1] for w in work) * args.steps
    score_s = score_ms.value * 1e-3
    achieved_tflops = ops / score_s / 1e12 if score_s > 0 else 0.0
    peak = ctypes.c_double(0)
    _lib.check(lib.weftk_measure_fp32_peak(ctypes.addressof(peak)), "weftk_measure_fp32_peak")
    peak_tflops = peak.value / 1e3
    # bytes the scoring kernels must move per launch: src+bg per pixel per item, prep per candidate
    cand_px = sum(w[0] for w in work) * args.steps

    # PSNR and payload of the fitted primitives alone (no residual grids)
    sel = fit.selected()
    recon = fit.recon_tiles()
    mse = float(np.mean([np.mean((p - r) ** 2) for p, r in zip(patches, recon)]))
    psnr_prims = 100.0 if mse <= 1e-12 else 10 * np.log10(1.0 / mse)
    prims_total = sum(len(s) for s in sel)
    prim_bytes = sum(1 + sum(2 + rate.PRIM_BYTES.get(c.kind, 48) for c in s) for s in sel)

    decode = decode_bench(fit, tiles, args.size, args.size, 3840, 2160, args.decode_iters, _hbm_peak()) \
        if args.decode_iters > 0 else None
    decode_res = decode_bench(fit, tiles, args.size, args.size, 3840, 2160, args.decode_iters, _hbm_peak(),
                              patches) if args.decode_iters > 0 else None

    rd = rd_compare(args, fit, tiles, patches, pools, img, stream) if args.refine_variants else None
    plain_value, plain_ms = value, ms_step

    # e2e of the plain fit through the public API from host buffers (pinned, as a caller that
    # streams images would keep them)
    pin_keep = []
    pixels_h, records_h = pinned_copy(pixels, pin_keep), pinned_copy(records, pin_keep)

    def plain_e2e():
        f2 = BatchedFit.from_arrays(pixels_h, sizes, records_h, counts, QUALITY, caps=caps, device=local)
        f2.run()
        f2.quantize_selected()
        q_rows, q_kind = f2.t_qrows.cpu(), f2.t_qkind.cpu()
        return (int(pixels.nbytes + records.nbytes + 4 * 6 * f2.n),
                int(q_rows.numel() * 4 + q_kind.numel() * 4 + 16 * len(f2.stats.per_round)))

    e2e_wall = {}

    def timed_e2e(fn):
        ms, wall, io = [], [], (0, 0)
        if args.e2e_steps > 0:
            for _ in range(args.warmup):  # untimed, like the device-timed steps
                fn()
        for _ in range(args.e2e_steps):
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            a.record(stream)
            io = fn()
            b.record(stream)
            torch.cuda.synchronize()
            wall.append((time.perf_counter() - t0) * 1e3)
            ms.append(a.elapsed_time(b))
        if not ms:
            return None, io
        e2e_wall[fn.__name__] = {"event_ms": ms, "host_wall_ms": wall}
        return world * n_px / (max_over_ranks(statistics.mean(ms), world) * 1e-3) / 1e6, io

    plain_e2e_val, (p_h2d, p_d2h) = timed_e2e(plain_e2e)

    # the refined fit over host-generated pools (the reference's generators, kind-filtered)
    rf, fast, frec, fcnt, host_ref_ms = refined_headline(args, local, pixels, sizes, pools, stream, world)
    host_ref_ms = max_over_ranks(host_ref_ms, world)
    r_score_ms, r_n_score, r_step_ms, r_work = refined_breakdown(args, rf, fast, lib, stream)
    r_flops = refine_flops(rf.ss)
    refine_tflops = r_flops / (r_step_ms * 1e-3) / 1e12 if r_step_ms > 0 else 0.0
    init_tflops = r_work[1] / (r_score_ms * 1e-3) / 1e12 if r_score_ms > 0 else 0.0
    host_ref_rd = rd_of_params(rf.ss, rf.refiner.p, tiles, patches, img, args.size)
    del rf, fast

    # headline: the gradient-refined fit over device-resident pools (generated on the device before
    # the timed steps, as the plain fit's pools are before its own), one CUDA graph, at iso RD with
    # the plain fit; then the same with the generation inside the graph (fit_total)
    sampler2 = ClockSampler(local)
    sampler2.start()
    drf, ref_ms = device_headline(args, fit, sizes, caps, stream, world, generate_in_run=False)
    clocks2 = sampler2.stop()
    drf_total, total_ms = device_headline(args, fit, sizes, caps, stream, world, generate_in_run=True)
    total_ms = max_over_ranks(total_ms, world)
    del drf_total
    dbd = device_breakdown(args, drf, lib, stream)
    # host generation of the same pools (the device generator's arctan2 rule), timed, outside the
    # clock window (no GPU work); the device pools must equal them record for record
    host_cl, cl_gen_s = restricted_pools(patches, REFINE_POOLS[args.refine_pool], executor)
    dev_cl = drf.pool_records()
    pools_equal = sum(1 for a, b in zip(dev_cl, host_cl) if a.tobytes() == b.tobytes())
    cl_gen_s, gen_s = max_over_ranks(cl_gen_s, world), max_over_ranks(cand_s, world)
    ref_ms = max_over_ranks(ref_ms, world)
    ref_value = world * n_px / (ref_ms * 1e-3) / 1e6
    plain_rd = rd["plain"] if rd else rd_of_params(*fit.stack_set(), tiles, patches, img, args.size)
    dss = drf.rf.ss
    ref_rd = rd_of_params(dss, drf.rf.refiner.p, tiles, patches, img, args.size)
    rd_delta = ref_rd["rd_score"] - plain_rd["rd_score"]
    iso = rd_delta >= -0.05
    d_flops = refine_flops(dss)
    d_refine_tflops = d_flops * args.refine_steps / (dbd["refine_ms"] * 1e-3) / 1e12 if dbd["refine_ms"] else 0.0
    d_init_tflops = dbd["work"][1] / (dbd["init_score_ms"] * 1e-3) / 1e12 if dbd["init_score_ms"] else 0.0
    n_cls = sum(1 for k in (8, 16, 32) if drf.fit.n_items[k])
    # moments, reset, prepare, begin, select, end, scoring (one per size class), refine start, one
    # launch for all refine steps, wire-grid snap (+ the pool generation, one launch per tile side,
    # in fit_total)
    ref_launches = 9 + n_cls
    # what the Adam steps add: RD of the same init round's picks without them
    init_rd = rd_of_params(dss, drf.rf.start, tiles, patches, img, args.size)

    pixels_h = pinned_copy(pixels, pin_keep)
    u8_h = pinned_copy(build_workload.u8, pin_keep)

    def refined_e2e():
        # the public call from the sRGB image: quadtree, tile extraction, pool generation, init
        # round, Adam steps and the wire-grid snap on the GPU; tiles and snapped rows come back
        from weft_b200.frontend import refine_image

        qt, rows, kinds = refine_image(u8_h, QUALITY, CAP, steps=args.refine_steps, lr=args.refine_lr, device=local)
        return int(u8_h.nbytes), int(qt.nbytes + rows.nbytes + kinds.nbytes + 4)

    def tiles_e2e():
        from weft_b200.pools import refine_tiles

        rows, kinds = refine_tiles(pixels_h, sizes, QUALITY, caps=caps, steps=args.refine_steps, lr=args.refine_lr,
                                   device=local)
        return int(pixels.nbytes + sizes.nbytes), int(rows.nbytes + kinds.nbytes)

    ref_e2e_val, (r_h2d, r_d2h) = timed_e2e(refined_e2e)
    tiles_e2e_val, _ = timed_e2e(tiles_e2e)
    # where the time of the same fit driven from Python goes: one call of the stepwise front end,
    # synchronised between its phases (untimed)
    from weft_b200.frontend import refine_image_steps

    e2e_phases: dict = {}
    refine_image_steps(u8_h, QUALITY, CAP, steps=args.refine_steps, lr=args.refine_lr, device=local,
                       timings=e2e_phases)

    diff = differentiable_fit(args, executor, local, stream) if args.diff_steps > 0 and rank == 0 else None
    ibatch = image_batch_fit(args, executor, local, stream) if args.batch_images and rank == 0 else None

    cpu = parity = None
    dec_cpu = ras_cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        if args.decode_iters > 0:
            dec_cpu, ras_cpu = cpu_decode_baselines(fit, tiles, patches, args.size, 3840, 2160)
        pick = cpu_sample(patches, pools, args.cpu_budget_s, executor)
        results: dict = {}
        v, wall, px = run_cpu(patches, pools, pick, executor, cores, schedule, results)
        cpu = {"value": v, "unit": "MPix/s", "cores": cores, "kind": "port", "cpu": cpu_model(),
               "sample": f"oracle greedy (plain fit) over {len(pick)} of {len(tiles)} tiles ({px / 1e6:.3f} MPix), "
                         f"{wall:.1f} s wall on {cores} processes"}
        parity = fit_parity(fit, results)
    if rank != 0:
        return
    # the raster branch is timed last, so that a failure in it leaves every number above intact
    raster_line = None
    if args.decode_iters > 0:
        try:
            raster_line = raster_bench(fit, tiles, patches, args.size, 3840, 2160, args.decode_iters, _hbm_peak())
        except Exception as e:  # reported in the line instead of ending the run
            raster_line = {"error": f"{type(e).__name__}: {e}"}
        if ras_cpu is not None:
            raster_line["cpu_baseline"] = ras_cpu
    if decode is not None and dec_cpu is not None:
        decode["cpu_baseline"] = dec_cpu
    score_roof = {"bound": "fp32", "achieved": achieved_tflops, "peak": peak_tflops, "unit": "TFLOP/s",
                  "frac": achieved_tflops / peak_tflops if peak_tflops else None, "traffic": None,
                  "kernel": "fit_score_queue_kernel (3 tile-size classes, all rounds), plain fit",
                  "peak_source": "measured FMA-loop probe on this GPU (weftk_measure_fp32_peak)",
                  "score_ms_per_step": score_ms.value / args.steps, "score_launches": n_score.value,
                  "candidate_pixels_per_step": cand_px // args.steps}
    fp32_src = "measured FMA-loop probe on this GPU (weftk_measure_fp32_peak)"
    refine_roof = {"bound": "fp32", "achieved": d_refine_tflops, "peak": peak_tflops, "unit": "TFLOP/s",
                   "frac": d_refine_tflops / peak_tflops if peak_tflops else None, "traffic": REFINE_TRAFFIC,
                   "traffic_source": TRAFFIC_SOURCE,
                   "kernel": "refine_tiles_kernel (loss + gradient + Adam; all steps of a fit in one launch)",
                   "peak_source": fp32_src, "ms": dbd["refine_ms"], "adam_steps_per_launch": args.refine_steps,
                   "flops_per_adam_step": d_flops}
    init_roof = {"bound": "fp32", "achieved": d_init_tflops, "peak": peak_tflops, "unit": "TFLOP/s",
                 "frac": d_init_tflops / peak_tflops if peak_tflops else None, "traffic": INIT_ROUND_TRAFFIC,
                 "traffic_source": TRAFFIC_SOURCE,
                 "kernel": "fit_score_queue_kernel, init round of the refined fit (three tile-size classes)", "ms": dbd["init_score_ms"],
                 "ms_samples": [round(v, 4) for v in dbd["init_score_samples"]],
                 "launches": dbd["init_score_launches"], "peak_source": fp32_src}
    n_cand = int(sum(len(p) for p in dev_cl))
    gen_bytes = 16 * n_px + 60 * n_cand + 4 * len(tiles)
    hbm_gbs, hbm_src = _hbm_peak()
    gen_gbs = gen_bytes / (dbd["gen_ms"] * 1e-3) / 1e9 if dbd["gen_ms"] else 0.0
    gen_roof = {"bound": "hbm", "achieved": gen_gbs, "peak": hbm_gbs, "unit": "GB/s", "frac": gen_gbs / hbm_gbs,
                "traffic": None, "kernel": "gen_pool_kernel (one launch per tile side)", "ms": dbd["gen_ms"],
                "algorithmic_bytes": gen_bytes, "candidates": n_cand, "peak_source": hbm_src,
                "note": "latency-bound: every mean is a sequential float32 sum in numpy's order"}
    # the dominant kernel of the timed step (pools resident: the init-round scoring or the refine
    # launch); the generator's roofline is in the details (it runs in fit_total's step only)
    parts = sorted([(dbd["init_score_ms"], init_roof), (dbd["refine_ms"], refine_roof)], key=lambda x: -x[0])
    dominant = parts[0][1]
    head_value, head_ms = (ref_value, ref_ms) if iso else (plain_value, plain_ms)
    grad_db = ref_rd["rd_score"] - init_rd["rd_score"]
    fit_desc = (f"refined batched fit over device-resident pools generated on the device (constant + linear, "
                f"{n_cand} candidates): one init round, {args.refine_steps} fused Adam steps (lr {args.refine_lr}) "
                f"and the wire-grid snap, one CUDA graph (with the generation in the graph: fit_total).  The speed-up "
                f"over the plain fit comes from the restricted pool's single init round; the Adam steps change RD by "
                f"{grad_db:+.4f} dB over that init round alone (iso_rd.adam_steps_db)" if iso else
                "plain greedy fit (the refined fit missed iso RD)")
    details = {
        "plain": {"value": plain_value, "ms_per_step": plain_ms, "tiles_per_s": len(tiles) * world / (plain_ms * 1e-3),
                  "e2e": plain_e2e_val, "e2e_bytes": [p_h2d, p_d2h], "roofline": score_roof,
                  "clocks": clocks, "gpu_launches": launches_per_step * args.steps,
                  "rounds_per_step": rounds[-1], "reseeds": fit.stats.reseeds, "graph_control": ctl,
                  "fit": "whole greedy (init, rounds, device re-seeds, wire-grid snap) replayed from one CUDA graph",
                  "cand_gen_s": cand_s, "prims_per_tile": prims_total / len(tiles), "psnr_prims_db": psnr_prims,
                  "prim_payload_bytes": prim_bytes,
                  "autotune": {str(k): {"variant": v[0], "cands_per_cta": v[1], "score_ms": v[2]}
                               for k, v in tuned_plain.items()}},
        "refined_device": {"ms": ref_ms, "breakdown": {k: v for k, v in dbd.items() if k != "work"},
                           "roofline_gen": gen_roof, "roofline_init": init_roof, "roofline_refine": refine_roof,
                           "autotune": {str(k): {"variant": v[0], "cands_per_cta": v[1], "score_ms": v[2]}
                                        for k, v in (drf.fit.tuning or {}).items()},
                           "pools_equal_host": [pools_equal, len(tiles)], "candidates": n_cand,
                           "e2e_from_tile_pixels": tiles_e2e_val,
                           "e2e": "frontend.refine_image from the sRGB u8 image in page-locked memory",
                           "e2e_steps": e2e_wall, "e2e_phases_ms": e2e_phases},
        "refined_host_pools": {"ms": host_ref_ms, "mpix_per_s": world * n_px / (host_ref_ms * 1e-3) / 1e6,
                               "rd": host_ref_rd, "candidates": int(len(frec)),
                               "score_ms": r_score_ms, "refine_ms_per_step": r_step_ms,
                               "refine_tflops": refine_tflops, "init_tflops": init_tflops,
                               "pools": "the reference's generators on the host (numpy arctan2), kind-filtered"},
        "iso_rd": {"plain": plain_rd, "refined": ref_rd, "init_round_only": init_rd},
        "decode": decode, "decode_with_residuals": decode_res, "decode_raster": raster_line,
        "differentiable_fit": diff, "image_batch": ibatch, "rd": rd, "parity": parity,
    }
    print(json.dumps({"bench_details": details}), file=sys.stderr, flush=True)

    def frac(d, key="frac"):
        return None if not d or key not in d else round(d[key], 4)

    line = {
        "metric": METRIC, "value": head_value, "unit": "MPix/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(args, len(tiles), int(sum(len(p) for p in pools))),
        "fit": fit_desc,
        "l2": "refined fit: 256 MiB written before each timed step; plain fit: per-step working set (pixels + "
              "pools) exceeds L2, no flush",
        "e2e": {"value": ref_e2e_val if iso else plain_e2e_val, "unit": "MPix/s",
                "h2d_bytes_per_step": r_h2d if iso else p_h2d, "d2h_bytes_per_step": r_d2h if iso else p_d2h},
        "roofline": dominant if iso else score_roof,
        "cpu_baseline": cpu,
        "clocks": clocks2 if iso else clocks,
        "gpu_launches": (ref_launches if iso else launches_per_step) * args.steps,
        "tiles_per_s": len(tiles) * world / (head_ms * 1e-3),
        "plain": {"value": plain_value, "ms_per_step": plain_ms, "e2e": plain_e2e_val,
                  "roofline_frac": frac(score_roof), "reseeds": fit.stats.reseeds},
        "iso_rd": {"plain_rd": plain_rd["rd_score"], "refined_rd": ref_rd["rd_score"], "delta_db": rd_delta,
                   "init_only_rd": init_rd["rd_score"], "adam_steps_db": grad_db, "tolerance_db": 0.05},
        "fit_total": {"refined_device_gen_mpix_per_s": world * n_px / (total_ms * 1e-3) / 1e6,
                      "refined_device_gen_ms": total_ms,
                      "refined_host_gen_mpix_per_s": world * n_px / (cl_gen_s + host_ref_ms * 1e-3) / 1e6,
                      "plain_host_gen_mpix_per_s": world * n_px / (gen_s + plain_ms * 1e-3) / 1e6,
                      "host_gen_s": {"constlin": cl_gen_s, "full": gen_s, "processes": cores},
                      "device_pools_equal_host": f"{pools_equal}/{len(tiles)} tiles"},
        "decode": {"frac": frac(decode), "frac_with_residuals": frac(decode_res),
                   "frac_back_to_back": frac((decode or {}).get("back_to_back")),
                   "frac_with_residuals_back_to_back": frac((decode_res or {}).get("back_to_back")),
                   "raster_resize_frac": frac((raster_line or {}).get("resize")),
                   "ms": None if not decode else round(decode["ms"], 4)},
        "parity": None if parity is None else {k: parity[k] for k in ("tiles", "equal_selections", "max_obj_rel")},
        "parity_2048": None if not diff or not diff.get("parity") else
        {k: diff["parity"][k] for k in ("tiles", "equal_selections", "max_obj_rel")},
        "image_batch": None if ibatch is None else {k: ibatch[k] for k in (
            "n_images", "mpix", "plain_mpix_per_s", "refined_mpix_per_s", "rd_delta_db_min", "rd_delta_db_mean",
            "images_within_0.05db")},
        "details": "the full record is the bench_details JSON line on stderr",
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
