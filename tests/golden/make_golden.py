"""Generate the golden fixtures in this folder by running the reference itself.

Run once, in a container where the reference source tree is available:

    python tests/golden/make_golden.py /path/to/reference/src [fixture ...]

or with the path in the environment variable ``WEFT_REFERENCE_SRC`` (the path
is required; there is no default).  The fixtures are small ``.npz`` files
committed next to this script; the tests read only those files, never the
reference.

What is captured (reference function -> fixture):
  * ``render.render_tile`` (src/weft/render.py:127) on random stacks of every
    primitive kind, tile sizes 8/16/32/64, with RES0 and scaled sampling
                                                           -> render_tiles.npz
  * ``render.render_scene_adaptive`` (src/weft/render.py:270) on a quadtree
    scene with RES0/RES1, native and scaled targets        -> render_scene.npz
  * ``encoder._tile_lambda`` / ``_PRIM_BYTE_SIZES_LUT`` / ``_estimate_bits``
    (src/weft/encoder.py:167-268)                           -> rate.npz
  * ``entropy.encode_bytes`` (src/weft/entropy.py:192) and
    ``prim_chunks.build_prim_chunks`` (src/weft/prim_chunks.py:23)
                                                           -> entropy.npz
  * ``encoder._quantize_primitive`` (src/weft/encoder.py:211),
    ``primitives.encode_tiles`` (src/weft/primitives.py:315) -> quant.npz
  * ``quadtree.decompose_quadtree`` / ``pack_qtree`` (src/weft/quadtree.py:42,111)
                                                           -> quadtree.npz
  * ``encoder._worker_gen_cands`` / ``_generate_residual_candidates``
    (src/weft/encoder.py:2490, :1255)                       -> candidates.npz
  * ``encoder.encode_image`` + ``decoder.decode_to_array`` of a small image, and the
    reference decoder reading this repo's re-encode of the same records
    (src/weft/encoder.py:3573, src/weft/decoder.py:650)     -> container.npz
  * ``encoder._fit_adaptive_state`` greedy (src/weft/encoder.py:2520-2831),
    driven by a CPU scorer that renders each eval with the reference's own
    ``render_tile`` at pixel centres (the reference GPU launcher
    ``gpu_render.gpu_batch_score_prepacked`` needs a GPU)
                               -> fit_small.npz (q=75), fit_hq.npz (q=92)
  * the same greedy inside ``encoder.encode_image`` on the 256x256 plain-method
    workload (40 primitives, seed 0, q=75, fixed 32-px tiles, at most 8
    primitives per tile, primitive-stack basis only), with the written file
    and ``decoder.decode_to_array`` at native size          -> fit_cfg256.npz
  * ``dct_residual.encode_tile_residuals`` / ``permute_tile_to_band`` /
    ``bitstream.pack_dct`` payloads (block versions 2-5, every chroma mode and
    layout, presence masks, per-tile scales) applied by the reference decoder's
    steps ``unpack_dct`` -> ``permute_band_to_tile`` -> ``apply_residual_to_image``, plus
    extremes (u8 scales 0 and 255; noise residuals up to std 0.6, ~40 % of pixels clipped;
    smooth residuals whose low-frequency coefficients reach ~800)
    (src/weft/decoder.py:477-507), and Pillow ``Image.resize(BILINEAR)`` of u8
    images (src/weft/decoder.py:514-518)                    -> dct.npz
  * the first three ``gpu_batch_score_prepacked`` calls of the reference's fit, arguments as
    passed, with the CPU stand-in's MSEs (src/weft/encoder.py:2698-2811)
                                                            -> launcher_calls.npz
  * ``encoder.encode_image`` with the DCT residual layer, decoded by
    ``decoder.decode_to_array`` at the encoded size and at up/down-scaled
    targets (the raster branch)                             -> container_dct.npz

Every primitive parameter handed to the reference is first rounded to float32,
so the fixtures are exact for kernels that consume float32 records.
"""

from __future__ import annotations

import os
import struct
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

GEOM_LEN = {0: 0, 1: 4, 2: 5, 3: 7, 4: 6, 5: 48}


def _f32(x: float) -> float:
    return float(np.float32(x))


def _rand_prim(rng, ref, kind: int, ts: int):
    Primitive = ref["Primitive"]
    lo, hi = -2.0, ts + 1.0
    if kind == 0:
        geom = ()
    elif kind == 1:
        geom = tuple(_f32(v) for v in rng.uniform(lo, hi, 4))
    elif kind == 2:
        geom = tuple(_f32(v) for v in rng.uniform(lo, hi, 4)) + (_f32(rng.uniform(0.0, 4.0)),)
    elif kind == 3:
        geom = tuple(_f32(v) for v in rng.uniform(lo, hi, 6)) + (_f32(rng.uniform(0.0, 4.0)),)
    elif kind == 4:
        geom = tuple(_f32(v) for v in rng.uniform(lo, hi, 6))
    else:
        geom = tuple(_f32(v) for v in rng.uniform(0.0, 1.0, 48))
    c0 = tuple(_f32(v) for v in rng.uniform(0.0, 1.0, 3))
    c1 = tuple(_f32(v) for v in rng.uniform(0.0, 1.0, 3)) if kind == 1 else None
    alpha = _f32(rng.uniform(0.05, 1.0))
    if kind == 5:
        c0, c1, alpha = (0.0, 0.0, 0.0), None, 1.0
    return Primitive(kind=kind, geom=geom, color0=c0, color1=c1, alpha=alpha)


def _pack_full(prims) -> dict:
    """Pack a primitive list into flat float64 arrays (geom padded to 48)."""
    n = len(prims)
    kind = np.zeros(n, np.int32)
    geom = np.zeros((n, 48), np.float64)
    c0 = np.zeros((n, 3), np.float64)
    c1 = np.zeros((n, 3), np.float64)
    has_c1 = np.zeros(n, np.int8)
    alpha = np.zeros(n, np.float64)
    for i, p in enumerate(prims):
        kind[i] = p.kind
        g = list(p.geom)
        geom[i, : len(g)] = g
        c0[i] = p.color0
        if p.color1 is not None:
            c1[i] = p.color1
            has_c1[i] = 1
        alpha[i] = p.alpha
    return {"kind": kind, "geom": geom, "c0": c0, "c1": c1, "has_c1": has_c1, "alpha": alpha}


def _concat_packs(packs: list[dict]) -> dict:
    out = {}
    for k in ("kind", "geom", "c0", "c1", "has_c1", "alpha"):
        arrs = [p[k] for p in packs]
        out[k] = np.concatenate(arrs) if arrs else np.zeros(0)
    counts = np.array([len(p["kind"]) for p in packs], np.int64)
    out["offsets"] = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    return out


def _save(name: str, **arrays) -> None:
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({os.path.getsize(path)} bytes)")


# ---------------------------------------------------------------------------
def gen_render_tiles(ref) -> None:
    render_tile = ref["render"].render_tile
    rng = np.random.default_rng(20260101)
    cases = []  # (prims, tile_size, source_size, residual)
    for ts in (8, 16, 32, 64):
        for kind in range(5):
            for _ in range(3):
                cases.append(([_rand_prim(rng, ref, kind, ts)], ts, None, None))
        for _ in range(2):
            cases.append(([_rand_prim(rng, ref, 5, ts)], ts, None, None))
        for n in (2, 5, 9, 16):
            kinds = rng.integers(0, 5, n)
            cases.append(([_rand_prim(rng, ref, int(k), ts) for k in kinds], ts, None, None))
        # const-only fast path, with residual
        cases.append(([_rand_prim(rng, ref, 0, ts) for _ in range(3)], ts, None,
                      tuple(int(v) for v in rng.integers(-127, 128, 3))))
        kinds = rng.integers(0, 5, 6)
        cases.append(([_rand_prim(rng, ref, int(k), ts) for k in kinds], ts, None,
                      tuple(int(v) for v in rng.integers(-127, 128, 3))))
        # kind 5 inside a multi-primitive stack is skipped by the renderer
        cases.append(([_rand_prim(rng, ref, 2, ts), _rand_prim(rng, ref, 5, ts)], ts, None, None))
    # edge cases on a 16-px tile
    P = ref["Primitive"]
    cases.append(([], 16, None, None))
    cases.append(([], 16, None, (10, -20, 127)))
    cases.append(([P(kind=2, geom=(5.0, 5.0, 5.0, 5.0, 1.0), color0=(0.9, 0.1, 0.2), alpha=0.8)], 16, None, None))
    cases.append(([P(kind=4, geom=(1.0, 1.0, 5.0, 5.0, 9.0, 9.0), color0=(0.9, 0.1, 0.2), alpha=0.8)], 16, None, None))
    cases.append(([P(kind=4, geom=(0.0, 0.0, 15.0, 0.0, 15.0, 15.0), color0=(0.3, 0.6, 0.2), alpha=1.0)], 16, None, None))
    cases.append(([P(kind=3, geom=(2.0, 2.0, 2.0, 2.0, 2.0, 2.0, 0.0), color0=(0.3, 0.6, 0.2), alpha=1.0)], 16, None, None))
    cases.append(([P(kind=1, geom=(3.0, 3.0, 3.0, 3.0), color0=(0.3, 0.6, 0.2), color1=(0.9, 0.9, 0.1), alpha=0.5)], 16, None, None))
    cases.append(([P(kind=0, geom=(), color0=(0.5, 0.25, 0.75), alpha=1.5),
                   P(kind=2, geom=(0.0, 3.0, 15.0, 9.0, 2.0), color0=(0.1, 0.2, 0.3), alpha=-0.25)], 16, None, None))
    # scaled sampling (decoder's scale-independent path)
    for ts, out in ((8, 16), (16, 40), (32, 48), (16, 12), (32, 5)):
        kinds = rng.integers(0, 5, 5)
        cases.append(([_rand_prim(rng, ref, int(k), ts) for k in kinds], out, ts,
                      tuple(int(v) for v in rng.integers(-40, 40, 3))))
    cases.append(([_rand_prim(rng, ref, 5, 16)], 24, 16, (3, -3, 0)))

    packs, ts_arr, src_arr, res_arr, has_res = [], [], [], [], []
    out_imgs, mses = [], []
    for prims, ts, src_size, res in cases:
        img = render_tile(prims, tile_size=ts, residual_rgb=res, source_size=src_size)
        assert img.dtype == np.float32 and img.shape == (ts, ts, 3)
        src = np.random.default_rng(1000 + len(ts_arr)).random((ts, ts, 3), dtype=np.float32)
        mses.append(float(np.mean((src - img) ** 2)))
        packs.append(_pack_full(prims))
        ts_arr.append(ts)
        src_arr.append(src_size if src_size is not None else ts)
        res_arr.append(res if res is not None else (0, 0, 0))
        has_res.append(res is not None)
        out_imgs.append(img.reshape(-1))
    pk = _concat_packs(packs)
    px_off = np.concatenate([[0], np.cumsum([t * t * 3 for t in ts_arr])]).astype(np.int64)
    _save(
        "render_tiles.npz",
        tile_size=np.array(ts_arr, np.int32),
        source_size=np.array(src_arr, np.int32),
        residual=np.array(res_arr, np.int32),
        has_residual=np.array(has_res, np.int8),
        px_offsets=px_off,
        image=np.concatenate(out_imgs).astype(np.float32),
        mse=np.array(mses, np.float64),
        **{"p_" + k: v for k, v in pk.items()},
    )


# ---------------------------------------------------------------------------
def gen_render_scene(ref) -> None:
    """Two scenes: 80x72 (pad/crop, native only) and 96x64 (native + scaled)."""
    from weft_b200.synth import make_image_linear

    render = ref["render"]
    quadtree = ref["quadtree"]
    TileRecord = ref["TileRecord"]
    rng = np.random.default_rng(424242)
    out = {}
    scenes = {
        "a": (80, 72, [(80, 72, True), (80, 72, False)]),
        # The reference's scaled walk needs the padded tile grid to fit inside the
        # target padded to 32, so scaled targets use an image that is a multiple of 32.
        # Anisotropic targets are run without RES1 (the reference raises there).
        "b": (96, 64, [(96, 64, True), (192, 128, True), (144, 96, True), (48, 32, True),
                       (120, 64, False), (96, 80, False)]),
    }
    for name, (width, height, targets) in scenes.items():
        image = make_image_linear(width, height, 12, 7)
        qts = quadtree.decompose_quadtree(image, split_threshold=0.08, min_tile=8, max_tile=32)
        records, packs, res1_maps = [], [], []
        for qt in qts:
            n = int(rng.integers(0, 5))
            if rng.random() < 0.1:
                prims = [_rand_prim(rng, ref, 5, qt.size)]
            else:
                prims = [_rand_prim(rng, ref, int(k), qt.size) for k in rng.integers(0, 5, n)]
            res = tuple(int(v) for v in rng.integers(-30, 31, 3))
            records.append(TileRecord(primitives=prims, residual_rgb=res))
            packs.append(_pack_full(prims))
            q = rng.integers(-127, 128, (4, 4, 3)).astype(np.int8)
            res1_maps.append(q.astype(np.float32) / 255.0)
        outs = []
        for tw, th, use_res1 in targets:
            img = render.render_scene_adaptive(
                records, qts, width, height,
                residual_maps=res1_maps if use_res1 else None, res1_grid_size=4,
                target_width=tw, target_height=th,
            )
            outs.append(img.astype(np.float32).reshape(-1))
        pk = _concat_packs(packs)
        out.update({
            f"{name}_dims": np.array([width, height], np.int32),
            f"{name}_qt": np.array([(q.x, q.y, q.size) for q in qts], np.int32),
            f"{name}_residual": np.array([r.residual_rgb for r in records], np.int32),
            f"{name}_res1": np.stack(res1_maps).astype(np.float32),
            f"{name}_targets": np.array([(t[0], t[1], int(t[2])) for t in targets], np.int32),
            f"{name}_images": np.concatenate(outs),
            **{f"{name}_p_" + k: v for k, v in pk.items()},
        })
    _save("render_scene.npz", **out)


# ---------------------------------------------------------------------------
def gen_rate(ref) -> None:
    enc = ref["encoder"]
    P = ref["Primitive"]
    lam = np.array([enc._tile_lambda(q) for q in range(-5, 106)], np.float64)
    rng = np.random.default_rng(5)
    stacks = []
    bits = []
    for _ in range(40):
        kinds = rng.integers(0, 6, int(rng.integers(0, 10)))
        prims = [P(kind=int(k), geom=(), color0=(0, 0, 0)) for k in kinds]
        inc_res = bool(rng.random() < 0.5)
        inc_res1 = bool(rng.random() < 0.5)
        g = int(rng.choice([2, 4, 8]))
        stacks.append((list(kinds), inc_res, inc_res1, g))
        bits.append(enc._estimate_bits(prims, inc_res, include_res1=inc_res1, res1_grid_size=g))
    flat = np.zeros((len(stacks), 16), np.int32) - 1
    meta = np.zeros((len(stacks), 3), np.int32)
    for i, (ks, a, b, g) in enumerate(stacks):
        flat[i, : len(ks)] = ks
        meta[i] = (int(a), int(b), g)
    _save("rate.npz", quality=np.arange(-5, 106, dtype=np.int32), lam=lam,
          lut=np.asarray(enc._PRIM_BYTE_SIZES_LUT, np.int32),
          stack_kinds=flat, stack_meta=meta, bits=np.array(bits, np.int64))


# ---------------------------------------------------------------------------
def gen_entropy(ref) -> None:
    ent = ref["entropy"]
    chunks = ref["prim_chunks"]
    rng = np.random.default_rng(99)
    payloads = [b"", b"\x00", b"\x07" * 100, bytes(range(256)), bytes(range(256)) * 3]
    for n in (10, 100, 1000, 5000):
        p = rng.dirichlet(np.full(256, 0.05))
        payloads.append(bytes(rng.choice(256, n, p=p).astype(np.uint8)))
    payloads.append(bytes(rng.integers(0, 256, 3000).astype(np.uint8)))
    payloads.append(bytes(rng.geometric(0.3, 4000).clip(0, 255).astype(np.uint8)))
    enc_out = [ent.encode_bytes(p) for p in payloads]
    # chunked PRIM payload from random quantized tiles
    prims_mod = ref["primitives"]
    enc = ref["encoder"]
    tiles = []
    for t in range(150):
        ps = [enc._quantize_primitive(_rand_prim(rng, ref, int(k), 16)) for k in rng.integers(0, 5, int(rng.integers(1, 6)))]
        tiles.append(ref["TileRecord"](primitives=ps))
    raw, toc = prims_mod.encode_tiles(tiles)
    coded64, entries64 = chunks.build_prim_chunks(raw, toc, 64)
    coded7, entries7 = chunks.build_prim_chunks(raw, toc, 7)

    def _ent(entries):
        return np.array([(e.start_tile, e.tile_count, e.raw_offset, e.raw_length, e.coded_offset, e.coded_length)
                         for e in entries], np.int64)

    def _cat(bs):
        off = np.concatenate([[0], np.cumsum([len(b) for b in bs])]).astype(np.int64)
        return np.frombuffer(b"".join(bs), np.uint8), off

    pay, pay_off = _cat(payloads)
    eo, eo_off = _cat(enc_out)
    _save("entropy.npz", payload=pay, payload_off=pay_off, encoded=eo, encoded_off=eo_off,
          prim_raw=np.frombuffer(raw, np.uint8), toc=np.array(toc, np.int64),
          coded64=np.frombuffer(coded64, np.uint8), entries64=_ent(entries64),
          coded7=np.frombuffer(coded7, np.uint8), entries7=_ent(entries7))


# ---------------------------------------------------------------------------
def gen_quant(ref) -> None:
    enc = ref["encoder"]
    prims_mod = ref["primitives"]
    rng = np.random.default_rng(1234)
    raw_prims, q_prims, tiles = [], [], []
    for t in range(60):
        ts = int(rng.choice([8, 16, 32]))
        ps = []
        for k in rng.integers(0, 6, int(rng.integers(0, 7))):
            p = _rand_prim(rng, ref, int(k), ts)
            if int(k) == 5:
                ps = [p]
                break
            ps.append(p)
        raw_prims.extend(ps)
        qs = [enc._quantize_primitive(p) if p.kind != 5 else p for p in ps]
        q_prims.extend(qs)
        tiles.append(ref["TileRecord"](primitives=ps))
    raw, toc = prims_mod.encode_tiles(tiles)
    counts = np.array([len(t.primitives) for t in tiles], np.int64)
    a = _pack_full(raw_prims)
    b = _pack_full(q_prims)
    _save("quant.npz", tile_counts=counts, tiles_raw=np.frombuffer(raw, np.uint8), toc=np.array(toc, np.int64),
          **{"in_" + k: v for k, v in a.items()}, **{"q_" + k: v for k, v in b.items()})


# ---------------------------------------------------------------------------
def gen_quadtree(ref) -> None:
    from weft_b200.synth import make_image_linear

    qt = ref["quadtree"]
    out = {}
    for name, (w, h, n, seed) in {"a": (256, 256, 40, 0), "b": (100, 70, 15, 3)}.items():
        img = make_image_linear(w, h, n, seed)
        for thr in (0.12, 0.08, 0.03):
            tiles = qt.decompose_quadtree(img, split_threshold=thr, min_tile=8, max_tile=32)
            key = f"{name}_{int(thr * 100):02d}"
            out[key] = np.array([(t.x, t.y, t.size) for t in tiles], np.int32)
            out[key + "_packed"] = np.frombuffer(qt.pack_qtree(tiles), np.uint8)
        out[name + "_dims"] = np.array([w, h, n, seed], np.int32)
    _save("quadtree.npz", **out)


# ---------------------------------------------------------------------------
def gen_candidates(ref) -> None:
    from weft_b200.synth import make_image_linear

    enc = ref["encoder"]
    qt = ref["quadtree"]
    img = make_image_linear(96, 96, 14, 11)
    tiles = qt.decompose_quadtree(img, split_threshold=0.08, min_tile=8, max_tile=32)
    patches = qt.extract_adaptive_tiles(img, tiles)
    rng = np.random.default_rng(77)
    pick = sorted(rng.choice(len(tiles), min(14, len(tiles)), replace=False).tolist())
    # make sure every tile size present gets at least one sample
    for s in (8, 16, 32):
        idx = [i for i, t in enumerate(tiles) if t.size == s]
        if idx and not any(tiles[i].size == s for i in pick):
            pick.append(idx[0])
    pick = sorted(set(pick))
    cand_packs, res_packs, patch_list, pred_list = [], [], [], []
    for i in pick:
        patch = patches[i]
        for q in (75,):
            cands, _ = enc._worker_gen_cands((patch, q))
            cand_packs.append(_pack_full(cands))
        pred = ref["render"].render_tile(cands[:2], tile_size=patch.shape[0])
        res = enc._generate_residual_candidates(patch, pred, 75)
        res_packs.append(_pack_full(res))
        patch_list.append(patch.reshape(-1))
        pred_list.append(pred.reshape(-1))
    sizes = np.array([tiles[i].size for i in pick], np.int32)
    px_off = np.concatenate([[0], np.cumsum(sizes.astype(np.int64) ** 2 * 3)])
    c = _concat_packs(cand_packs)
    r = _concat_packs(res_packs)
    _save("candidates.npz", sizes=sizes, px_offsets=px_off,
          patch=np.concatenate(patch_list), pred=np.concatenate(pred_list),
          **{"c_" + k: v for k, v in c.items()}, **{"r_" + k: v for k, v in r.items()})


# ---------------------------------------------------------------------------
def _cpu_score_prepacked(ref):
    """CPU stand-in for ``gpu_render.gpu_batch_score_prepacked`` (pixel centres)."""
    render_tile = ref["render"].render_tile
    P = ref["Primitive"]
    glen = {0: 0, 1: 4, 2: 5, 3: 7, 4: 6}
    stats = {"launches": 0, "evals": 0}

    def unpack(rec):
        k = int(rec["kind"])
        g = tuple(float(v) for v in rec["geom"][: glen.get(k, 7)])
        c0 = tuple(float(v) for v in rec["color0"])
        c1 = tuple(float(v) for v in rec["color1"]) if k == 1 else None
        return P(kind=k, geom=g, color0=c0, color1=c1, alpha=float(rec["alpha"]))

    def score(tile_pixels_flat, tile_pixel_offsets, tile_indices, tile_sizes, eval_prim_arrays, eval_prim_counts):
        stats["launches"] += 1
        out = []
        for j, ti in enumerate(tile_indices):
            ts = tile_sizes[j]
            off = tile_pixel_offsets[ti]
            src = tile_pixels_flat[off: off + ts * ts * 3].reshape(ts, ts, 3)
            arr = eval_prim_arrays[j]
            counts = eval_prim_counts[j]
            res = np.zeros(len(counts), np.float32)
            o = 0
            for k, nc in enumerate(counts):
                prims = [unpack(arr[o + m]) for m in range(int(nc))]
                o += int(nc)
                res[k] = np.float32(np.mean((src - render_tile(prims, tile_size=ts)) ** 2))
            stats["evals"] += len(counts)
            out.append(res)
        return out

    return score, stats


class _FitCapture:
    """Runs the reference's adaptive fit with the CPU scorer installed and records, per tile, the
    initial candidate pool, every re-seed batch and the fit state's selections.

    ``tile_size`` forces the quadtree to fixed tiles of that side and ``cap`` the per-tile primitive
    cap (the reference reads both from module globals: ``quadtree.decompose_quadtree`` is imported
    inside the fit, ``QuadTile.max_primitives`` reads ``MAX_PRIMITIVES_BY_TILE_SIZE``)."""

    def __init__(self, ref, tile_size: int | None = None, cap: int | None = None):
        self.ref, self.tile_size, self.cap = ref, tile_size, cap
        self.pools: dict[int, list] = {}
        self.reseeds: list[tuple[int, list]] = []
        self.patches = None
        self.state = None

    def __enter__(self):
        enc, gr, qt_mod = self.ref["encoder"], self.ref["gpu_render"], self.ref["quadtree"]
        score, self.stats = _cpu_score_prepacked(self.ref)
        orig_worker, orig_resid = enc._worker_gen_cands, enc._generate_residual_candidates
        orig_extract, orig_decomp, orig_fit = qt_mod.extract_adaptive_tiles, qt_mod.decompose_quadtree, \
            enc._fit_adaptive_state

        def extract(image, tiles):
            self.patches = orig_extract(image, tiles)
            return self.patches

        def decomp(image, **kw):
            if self.tile_size is not None:
                kw["min_tile"] = kw["max_tile"] = self.tile_size
            return orig_decomp(image, **kw)

        def worker(args):
            cands, packed = orig_worker(args)
            idx = next(i for i, p in enumerate(self.patches) if p is args[0])
            self.pools[idx] = list(cands)
            return cands, packed

        def resid(tile, pred, quality):
            out = orig_resid(tile, pred, quality)
            idx = next(i for i, p in enumerate(self.patches) if p is tile)
            self.reseeds.append((idx, list(out)))
            return out

        def fit(*a, **kw):
            self.state = orig_fit(*a, **kw)
            return self.state

        self.saved = (gr.gpu_batch_score_prepacked, enc._worker_gen_cands, enc._generate_residual_candidates,
                      qt_mod.extract_adaptive_tiles, qt_mod.decompose_quadtree, enc._get_persistent_worker_pool,
                      enc._fit_adaptive_state, qt_mod.MAX_PRIMITIVES_BY_TILE_SIZE)
        gr.gpu_batch_score_prepacked = score
        enc._worker_gen_cands = worker
        enc._generate_residual_candidates = resid
        qt_mod.extract_adaptive_tiles = extract
        qt_mod.decompose_quadtree = decomp
        enc._get_persistent_worker_pool = lambda: None
        enc._fit_adaptive_state = fit
        if self.cap is not None:
            qt_mod.MAX_PRIMITIVES_BY_TILE_SIZE = {s: self.cap for s in (8, 16, 32, 64)}
        return self

    def __exit__(self, *exc):
        enc, gr, qt_mod = self.ref["encoder"], self.ref["gpu_render"], self.ref["quadtree"]
        (gr.gpu_batch_score_prepacked, enc._worker_gen_cands, enc._generate_residual_candidates,
         qt_mod.extract_adaptive_tiles, qt_mod.decompose_quadtree, enc._get_persistent_worker_pool,
         enc._fit_adaptive_state, qt_mod.MAX_PRIMITIVES_BY_TILE_SIZE) = self.saved
        return False

    def arrays(self) -> dict:
        """Pools, re-seeds and selections (indices into each tile's extended pool) as arrays."""
        state = self.state
        n_tiles = len(state.quad_tiles)
        ext_pools = {i: list(self.pools[i]) for i in range(n_tiles)}
        for i, cands in self.reseeds:
            ext_pools[i].extend(cands)
        sel_idx = []
        for i in range(n_tiles):
            sel_idx.append([next(j for j, c in enumerate(ext_pools[i]) if c is p) for p in state.selected_per_tile[i]])
        init = _concat_packs([_pack_full(self.pools[i]) for i in range(n_tiles)])
        rs = _concat_packs([_pack_full(c) for _, c in self.reseeds])
        sel_flat = np.full((n_tiles, 32), -1, np.int32)
        for i, ids in enumerate(sel_idx):
            sel_flat[i, : len(ids)] = ids
        print(f"fit: {n_tiles} tiles, {self.stats['launches']} launches, {self.stats['evals']} evals, "
              f"{len(self.reseeds)} reseeds, prims/tile {np.mean([len(s) for s in sel_idx]):.2f}")
        return dict(image=state.image.astype(np.float32),
                    qt=np.array([(q.x, q.y, q.size) for q in state.quad_tiles], np.int32),
                    quality=np.int32(state.quality), lam=np.float64(state.lam), selected=sel_flat,
                    reseed_tile=np.array([i for i, _ in self.reseeds], np.int32),
                    **{"pool_" + k: v for k, v in init.items()}, **{"rs_" + k: v for k, v in rs.items()})


def gen_fit(ref, name: str = "fit_small.npz", size: int = 64, n_prims: int = 10, seed: int = 5,
            quality: int = 75) -> None:
    from PIL import Image
    from weft_b200.synth import make_image_u8

    img_u8 = make_image_u8(size, size, n_prims, seed)
    with _FitCapture(ref) as cap, tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "in.png")
        Image.fromarray(img_u8).save(path)
        ref["encoder"]._fit_adaptive_state(path, ref["EncodeConfig"](quality=quality))
    _save(name, image_u8=img_u8, **cap.arrays())


def gen_fit_cfg256(ref) -> None:
    """The plain-method workload at 256x256: 40 primitives, seed 0, q=75, fixed 32-px tiles, at
    most 8 primitives per tile, primitive-stack basis only (``encode_image`` with no feature
    flags), then the reference decoder at native size."""
    from PIL import Image
    from weft_b200.synth import make_image_u8

    enc, dec_mod, prim_chunks = ref["encoder"], ref["decoder"], ref["prim_chunks"]
    img_u8 = make_image_u8(256, 256, 40, 0)
    saved = dec_mod._decode_prim_payload
    dec_mod._decode_prim_payload = lambda weft: (
        prim_chunks.decode_prim_payload(weft.prim_payload, weft.toc, weft.chunk_index), "cpu")
    try:
        with _FitCapture(ref, tile_size=32, cap=8) as cap, tempfile.TemporaryDirectory() as td:
            src = os.path.join(td, "in.png")
            Image.fromarray(img_u8).save(src)
            out = os.path.join(td, "out.weft")
            enc.encode_image(src, out, ref["EncodeConfig"](quality=75))
            blob = open(out, "rb").read()
            decoded = dec_mod.decode_to_array(out)
    finally:
        dec_mod._decode_prim_payload = saved
    assert {int(q.size) for q in cap.state.quad_tiles} == {32}
    assert max(len(s) for s in cap.state.selected_per_tile) <= 8
    print(f"cfg256: file {len(blob)} B")
    _save("fit_cfg256.npz", image_u8=img_u8, weft_file=np.frombuffer(blob, np.uint8),
          decoded=decoded.astype(np.float32), **cap.arrays())


def gen_container(ref) -> None:
    """Reference encode -> file A (+ its decode); this repo's writer re-encodes A's
    records -> file B, which the reference decoder must read (+ its decode)."""
    from PIL import Image

    from weft_b200 import bitstream
    from weft_b200.candidates import Cand
    from weft_b200.synth import make_image_u8

    enc = ref["encoder"]
    gr = ref["gpu_render"]
    dec_mod = ref["decoder"]
    prim_chunks = ref["prim_chunks"]
    score, _ = _cpu_score_prepacked(ref)
    saved = (gr.gpu_batch_score_prepacked, enc._get_persistent_worker_pool, dec_mod._decode_prim_payload)
    gr.gpu_batch_score_prepacked = score
    enc._get_persistent_worker_pool = lambda: None
    dec_mod._decode_prim_payload = lambda weft: (
        prim_chunks.decode_prim_payload(weft.prim_payload, weft.toc, weft.chunk_index), "cpu")
    try:
        img_u8 = make_image_u8(64, 64, 8, 21)
        with tempfile.TemporaryDirectory() as td:
            src = os.path.join(td, "in.png")
            Image.fromarray(img_u8).save(src)
            fa = os.path.join(td, "a.weft")
            enc.encode_image(src, fa, ref["EncodeConfig"](quality=75))
            blob_a = open(fa, "rb").read()
            dec_a = dec_mod.decode_to_array(fa)
            wf = bitstream.decode_weft(blob_a)
            tiles = [type("QT", (), {"x": x, "y": y, "size": sz})() for x, y, sz in wf.qtree]
            stacks = [[Cand(k, g, c0, c1, a) for k, g, c0, c1, a in st]
                      for st in bitstream.decode_tiles(wf.prim_raw, wf.toc)]
            blob_b = bitstream.encode_weft(wf.width, wf.height, wf.quality, tiles, stacks, wf.residuals, wf.res1_maps)
            fb = os.path.join(td, "b.weft")
            open(fb, "wb").write(blob_b)
            dec_b = dec_mod.decode_to_array(fb)
            ra = ref["bitstream"].decode_weft(blob_a)
            rb = ref["bitstream"].decode_weft(blob_b)
            for attr in ("prim_payload", "res0_payload", "res1_payload", "qtree_payload", "cidx_payload"):
                assert getattr(ra, attr) == getattr(rb, attr), attr
            assert ra.toc == rb.toc
    finally:
        gr.gpu_batch_score_prepacked, enc._get_persistent_worker_pool, dec_mod._decode_prim_payload = saved
    print(f"container: reference file {len(blob_a)} B, re-encoded {len(blob_b)} B; payload blocks identical")
    _save("container.npz", image_u8=img_u8, file_a=np.frombuffer(blob_a, np.uint8), decoded_a=dec_a.astype(np.float32),
          file_b=np.frombuffer(blob_b, np.uint8), decoded_b=dec_b.astype(np.float32))


DCT_TILES = [(0, 0, 64), (64, 0, 32), (96, 0, 32), (64, 32, 16), (80, 32, 16), (64, 48, 8), (72, 48, 8),
             (64, 56, 8), (72, 56, 8), (80, 48, 16), (96, 32, 32), (0, 64, 32), (32, 64, 32), (0, 96, 32),
             (32, 96, 32), (64, 64, 64)]


def gen_dct(ref) -> None:
    """BLOCK_DCT payloads from the reference's encoder helpers, applied to a random recon by
    the reference decoder's own steps (src/weft/decoder.py:477-507); Pillow BILINEAR resizes."""
    from PIL import Image

    R = ref["dct_residual"]
    B = ref["bitstream"]

    class QT:
        def __init__(self, x, y, size):
            self.x, self.y, self.size = x, y, size

    rng = np.random.default_rng(20260416)
    H, W = 72, 100   # tiles cover 128 x 128: some cross the image edge, two lie outside it
    recon = rng.uniform(-0.05, 1.05, (H, W, 3)).astype(np.float32)
    out = {"recon": recon, "tiles": np.array(DCT_TILES, np.int32)}

    def case(i, chroma, alpha, scales, layout, version, p_present, std=0.06, smooth=False):
        """One block: ``scales`` None (uniform), "rng" (u8 scales drawn from 40..219) or u8 bytes;
        ``smooth`` adds a per-tile offset and ramp (large low-frequency coefficients)."""
        present = [bool(rng.random() < p_present) for _ in DCT_TILES]
        res = [rng.normal(0.0, std, (s, s, 3)).astype(np.float32) for (_, _, s), p in zip(DCT_TILES, present) if p]
        if smooth:
            for r in res:
                s = r.shape[0]
                ramp = np.linspace(-0.3, 0.3, s, dtype=np.float32)
                r += (ramp[:, None, None] + np.array([0.45, -0.35, 0.2], np.float32)).astype(np.float32)
        sizes = [s for (_, _, s), p in zip(DCT_TILES, present) if p]
        if scales == "rng":
            su8 = bytes(int(v) for v in rng.integers(40, 220, len(res)))
        else:
            su8 = bytes(scales[:len(res)]) if scales else b""
        sc = [R.decode_tile_scale_u8(b) for b in su8] if su8 else None
        coeffs, _ = R.encode_tile_residuals(res, quant_step=0.0135, freq_alpha=alpha, chroma_mode=chroma,
                                            per_tile_scales=sc)
        payload = R.permute_tile_to_band(coeffs, sizes, chroma) if layout else coeffs
        mask = R._present_indices_to_bitmask(present)
        if version == 5:
            blob = B.pack_dct(payload, 0.0135, 3, freq_alpha=alpha, chroma_mode=chroma, presence_bitmask=mask,
                              n_tiles=len(DCT_TILES), layout=layout, per_tile_scales_u8=su8)
        elif version == 4:
            blob = struct.pack("<BBBBffHII", 4, chroma, layout, 0, 0.0135, alpha, 3, len(DCT_TILES),
                               payload.size) + mask + payload.astype("<i2").tobytes()
        elif version == 3:
            blob = struct.pack("<BBffHII", 3, chroma, 0.0135, alpha, 3, len(DCT_TILES),
                               payload.size) + mask + payload.astype("<i2").tobytes()
        else:
            blob = struct.pack("<BBffHI", 2, chroma, 0.0135, alpha, 3, payload.size) + payload.astype("<i2").tobytes()
        c, step, channels, falpha, cmode, pmask, n_hdr, lay, su = B.unpack_dct(blob)
        if lay == 1:
            pr = R._bitmask_to_present_indices(pmask, n_hdr) if (n_hdr > 0 and len(pmask) > 0) else [True] * 16
            c = R.permute_band_to_tile(c, [s for (_, _, s), p in zip(DCT_TILES, pr) if p], cmode)
        pts = [R.decode_tile_scale_u8(b) for b in su] if su else None
        want = R.apply_residual_to_image(recon, c, [QT(*t) for t in DCT_TILES], quant_step=step, channels=channels,
                                         freq_alpha=falpha, chroma_mode=cmode, presence_bitmask=pmask,
                                         per_tile_scales=pts)
        out[f"blob_{i}"] = np.frombuffer(blob, np.uint8)
        out[f"out_{i}"] = want.astype(np.float32)

    # (chroma mode, freq alpha, per-tile scales, layout, block version, presence probability)
    cases = [(0, 0.0, None, 0, 5, 0.8), (1, 4.0, None, 1, 5, 0.8), (2, 4.0, "rng", 1, 5, 0.8),
             (2, 0.0, "rng", 0, 5, 1.0), (2, 4.0, None, 1, 4, 0.7), (1, 0.0, None, 0, 3, 0.7),
             (2, 4.0, None, 0, 2, 1.0), (0, 4.0, None, 1, 5, 0.0)]
    for i, cfg in enumerate(cases):
        case(i, *cfg)
    for j, ((h, w), (ow, oh)) in enumerate((((48, 64), (240, 135)), ((64, 96), (96, 200)), ((80, 100), (37, 29)),
                                            ((17, 33), (200, 100)), ((50, 70), (70, 50)), ((31, 29), (300, 7)))):
        u8 = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
        out[f"rs_in_{j}"] = u8
        out[f"rs_out_{j}"] = np.asarray(Image.fromarray(u8).resize((ow, oh), Image.BILINEAR))
    # extremes: the ends of the u8 scale range, and residuals large enough to clip ~40 % of pixels
    case(8, 2, 4.0, bytes([0, 255] * 8), 1, 5, 1.0)
    case(9, 0, 0.0, None, 0, 5, 0.9, std=0.6)
    case(10, 1, 4.0, bytes([255, 0, 128] * 6), 0, 5, 0.9, std=0.3)
    case(11, 2, 4.0, None, 1, 5, 1.0, std=0.02, smooth=True)
    _save("dct.npz", **out)


def gen_container_dct(ref) -> None:
    """Reference encodes with the DCT residual layer (default flags, and with per-tile adaptive
    quantization), decoded by the reference at the encoded size and at an up- and a
    down-scaled target (the raster branch, src/weft/decoder.py:446-518)."""
    from PIL import Image

    from weft_b200.synth import make_image_u8

    enc = ref["encoder"]
    gr = ref["gpu_render"]
    dec_mod = ref["decoder"]
    prim_chunks = ref["prim_chunks"]
    score, _ = _cpu_score_prepacked(ref)
    saved = (gr.gpu_batch_score_prepacked, enc._get_persistent_worker_pool, dec_mod._decode_prim_payload)
    gr.gpu_batch_score_prepacked = score
    enc._get_persistent_worker_pool = lambda: None
    dec_mod._decode_prim_payload = lambda weft: (
        prim_chunks.decode_prim_payload(weft.prim_payload, weft.toc, weft.chunk_index), "cpu")
    out = {}
    try:
        img_u8 = make_image_u8(96, 80, 10, 33)
        out["image_u8"] = img_u8
        for name, flags in (("a", {"dct_residual": True}),
                            ("b", {"dct_residual": True, "dct_residual_adaptive_quant": True})):
            with tempfile.TemporaryDirectory() as td:
                src = os.path.join(td, "in.png")
                Image.fromarray(img_u8).save(src)
                fa = os.path.join(td, "a.weft")
                enc.encode_image(src, fa, ref["EncodeConfig"](quality=75, feature_flags=flags))
                out[f"file_{name}"] = np.frombuffer(open(fa, "rb").read(), np.uint8)
                out[f"native_{name}"] = dec_mod.decode_to_array(fa).astype(np.float32)
                out[f"up_{name}"] = dec_mod.decode_to_array(fa, 200, 150).astype(np.float32)
                out[f"down_{name}"] = dec_mod.decode_to_array(fa, 50, 37).astype(np.float32)
    finally:
        gr.gpu_batch_score_prepacked, enc._get_persistent_worker_pool, dec_mod._decode_prim_payload = saved
    _save("container_dct.npz", **out)


def gen_bicubic(ref) -> None:
    """The per-tile bicubic R-D swap of ``_fit_adaptive_state`` (src/weft/encoder.py:2841-2873).

    (a) ``bicubic.fit_tile`` / ``eval_tile`` (src/weft/bicubic.py:65-110) on tiles of every size
    (noise, smooth, step edges, values beyond [0, 1] that the fit clips), with the control grid
    rounded to u8 steps as the swap does; (b) three fits whose state's ``bicubic_replaced_per_tile``
    gives the swap decisions: the selected stacks, the tile patches and lambda go in, the swapped
    flags and control grids come out."""
    from weft_b200.synth import make_image_u8

    bic = ref["bicubic"]
    rng = np.random.default_rng(17)
    tiles, cps, cpq, mse = [], [], [], []
    for ts in (8, 16, 32, 64):
        yy, xx = np.meshgrid(np.linspace(0, 1, ts), np.linspace(0, 1, ts), indexing="ij")
        cases = [rng.random((ts, ts, 3)),
                 np.stack([0.2 + 0.6 * xx, 0.1 + 0.5 * yy * xx, 0.9 - 0.7 * yy], -1),
                 np.where((xx + 0.3 * yy > 0.55)[..., None], [0.9, 0.2, 0.1], [0.05, 0.6, 0.95]),
                 np.clip(rng.normal(0.5, 0.6, (ts, ts, 3)), -0.2, 1.3)]
        for c in cases:
            t = np.ascontiguousarray(c, np.float32)
            cp = bic.fit_tile(t)
            q = np.round(np.clip(cp, 0.0, 1.0) * 255.0) / 255.0
            r = bic.eval_tile(q, ts)
            tiles.append(t.reshape(-1))
            cps.append(cp.reshape(-1))
            cpq.append(q.reshape(-1))
            mse.append(float(np.mean((t - r) ** 2)))
    sizes = np.repeat([8, 16, 32, 64], 4).astype(np.int32)
    out = dict(tile_sizes=sizes, tiles=np.concatenate(tiles), cp=np.stack(cps).astype(np.float32),
               cp_q=np.stack(cpq).astype(np.float32),
               mse=np.array(mse, np.float64))
    from PIL import Image

    for name, size, n_prims, seed, quality in (("a", 64, 10, 5, 75), ("b", 64, 30, 11, 92), ("c", 64, 40, 2, 97)):
        img_u8 = make_image_u8(size, size, n_prims, seed)
        with _FitCapture(ref) as cap, tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "in.png")
            Image.fromarray(img_u8).save(path)
            ref["encoder"]._fit_adaptive_state(path, ref["EncodeConfig"](quality=quality))
        st = cap.state
        sel = st.selected_per_tile
        swapped = np.array([len(b) == 1 and b[0].kind == 5 and not (len(s) == 1 and s[0] is b[0])
                            for s, b in zip(sel, st.bicubic_replaced_per_tile)], np.int8)
        grids = np.zeros((len(sel), 48), np.float32)
        for i, b in enumerate(st.bicubic_replaced_per_tile):
            if swapped[i]:
                grids[i] = np.asarray(b[0].geom, np.float32)
        packed = _concat_packs([_pack_full(s) for s in sel])
        print(f"bicubic {name}: q={quality}, {len(sel)} tiles, {int(swapped.sum())} swapped "
              f"(state says {st.n_bicubic_tiles})")
        assert int(swapped.sum()) == st.n_bicubic_tiles
        out.update({f"{name}_image": st.image.astype(np.float32),
                    f"{name}_qt": np.array([(q.x, q.y, q.size) for q in st.quad_tiles], np.int32),
                    f"{name}_lam": np.float64(st.lam), f"{name}_quality": np.int32(quality),
                    f"{name}_swapped": swapped, f"{name}_grids": grids,
                    **{f"{name}_sel_{k}": v for k, v in packed.items()}})
    _save("bicubic.npz", **out)


def gen_launcher_calls(ref) -> None:
    """The first three calls the reference's fit makes to ``gpu_batch_score_prepacked`` (the init
    round, the selected stacks' current objective and the first greedy round of the fit_small
    workload, src/weft/encoder.py:2698-2811),
    with their arguments exactly as the fit passes them and the MSEs of the CPU stand-in (the
    reference's ``render_tile`` at pixel centres)."""
    from PIL import Image
    from weft_b200.synth import make_image_u8

    calls = []
    img_u8 = make_image_u8(64, 64, 10, 5)
    with _FitCapture(ref) as cap, tempfile.TemporaryDirectory() as td:
        gr = ref["gpu_render"]
        inner = gr.gpu_batch_score_prepacked

        def recording(*args):
            out = inner(*args)
            if len(calls) < 3:
                calls.append((args, out))
            return out

        gr.gpu_batch_score_prepacked = recording
        path = os.path.join(td, "in.png")
        Image.fromarray(img_u8).save(path)
        ref["encoder"]._fit_adaptive_state(path, ref["EncodeConfig"](quality=75))
    out = {"quality": np.int32(75), "selected": cap.arrays()["selected"], "n_calls": np.int32(len(calls))}
    for i, (args, res) in enumerate(calls):
        flat, offsets, tidx, tsizes, prim_arrays, prim_counts = args
        keys = sorted(offsets)
        out[f"c{i}_pixels"] = np.asarray(flat, np.float32)
        out[f"c{i}_offset_keys"] = np.array(keys, np.int64)
        out[f"c{i}_offset_vals"] = np.array([offsets[k] for k in keys], np.int64)
        out[f"c{i}_tile_indices"] = np.array(tidx, np.int64)
        out[f"c{i}_tile_sizes"] = np.array(tsizes, np.int64)
        out[f"c{i}_prims"] = np.concatenate([np.ascontiguousarray(a).view(np.uint8) for a in prim_arrays])
        out[f"c{i}_prim_len"] = np.array([len(a) for a in prim_arrays], np.int64)
        out[f"c{i}_counts"] = np.concatenate([np.asarray(c, np.int32) for c in prim_counts])
        out[f"c{i}_count_len"] = np.array([len(c) for c in prim_counts], np.int64)
        out[f"c{i}_mse"] = np.concatenate([np.asarray(r, np.float32) for r in res])
        print(f"launcher call {i}: {len(tidx)} tiles, {len(out[f'c{i}_counts'])} evals, "
              f"{int(out[f'c{i}_prim_len'].sum())} records")
    _save("launcher_calls.npz", **out)


def main() -> None:
    args = sys.argv[1:]
    src = os.environ.get("WEFT_REFERENCE_SRC")
    if args and os.path.isdir(args[0]):
        src = args.pop(0)
    if not src:
        sys.exit("usage: make_golden.py REFERENCE_SRC [fixture ...]  (or set WEFT_REFERENCE_SRC)")
    sys.path.insert(0, src)
    import weft.bicubic as bicubic
    import weft.bitstream as bitstream_mod
    import weft.dct_residual as dct_residual
    import weft.decoder as decoder
    import weft.encoder as encoder
    import weft.entropy as entropy
    import weft.gpu_render as gpu_render
    import weft.prim_chunks as prim_chunks
    import weft.primitives as primitives
    import weft.quadtree as quadtree
    import weft.render as render
    from weft.types import EncodeConfig

    ref = {
        "encoder": encoder, "entropy": entropy, "gpu_render": gpu_render, "prim_chunks": prim_chunks,
        "primitives": primitives, "quadtree": quadtree, "render": render,
        "Primitive": primitives.Primitive, "TileRecord": primitives.TileRecord, "EncodeConfig": EncodeConfig,
        "decoder": decoder, "bitstream": bitstream_mod, "dct_residual": dct_residual, "bicubic": bicubic,
    }
    which = set(args) if args else None
    for name, fn in (("render_tiles", gen_render_tiles), ("render_scene", gen_render_scene), ("rate", gen_rate),
                     ("entropy", gen_entropy), ("quant", gen_quant), ("quadtree", gen_quadtree),
                     ("candidates", gen_candidates), ("fit", gen_fit),
                     ("fit_hq", lambda r: gen_fit(r, "fit_hq.npz", 40, 8, 3, 92)), ("fit_cfg256", gen_fit_cfg256),
                     ("container", gen_container),
                     ("dct", gen_dct), ("container_dct", gen_container_dct), ("bicubic", gen_bicubic),
                     ("launcher_calls", gen_launcher_calls)):
        if which is None or name in which:
            fn(ref)


if __name__ == "__main__":
    main()
