"""DCT residual layer and raster resize on the CPU: the oracle against the reference's own outputs
(golden fixtures), the host descriptor logic of ``weft_b200.raster`` against the oracle, and the
C-ABI argument checks (no GPU work)."""

from __future__ import annotations

import struct

import numpy as np
import pytest

from oracle import dct as odct
from weft_b200 import _lib, raster

N_CASES = 12
N_RESIZE = 6
RESIZE_TARGETS = [(240, 135), (96, 200), (37, 29), (200, 100), (70, 50), (300, 7)]


def _blob(g, i) -> bytes:
    return g[f"blob_{i}"].tobytes()


@pytest.mark.parametrize("i", range(N_CASES))
def test_oracle_apply_matches_reference(golden, i):
    g = golden("dct.npz")
    tiles = [tuple(int(v) for v in t) for t in g["tiles"]]
    got = odct.apply_dct_block(g["recon"], _blob(g, i), tiles)
    np.testing.assert_array_equal(got, g[f"out_{i}"])


@pytest.mark.parametrize("j", range(N_RESIZE))
def test_oracle_resize_matches_pillow(golden, j):
    g = golden("dct.npz")
    ow, oh = RESIZE_TARGETS[j]
    np.testing.assert_array_equal(odct.resize_bilinear_u8(g[f"rs_in_{j}"], ow, oh), g[f"rs_out_{j}"])


def test_oracle_raster_decode_matches_reference_files(golden):
    """Whole raster branch: oracle walk at the encoded size, DCT residual, u8 + BILINEAR resize,
    against the reference decoder's arrays for the same files."""
    from oracle import render as orender
    from weft_b200 import bitstream
    from weft_b200.candidates import Cand

    g = golden("container_dct.npz")

    class Rec:
        def __init__(self, p, r):
            self.primitives, self.residual_rgb = p, r

    class QT:
        def __init__(self, x, y, size):
            self.x, self.y, self.size = x, y, size

    for name in ("a", "b"):
        wf = bitstream.decode_weft(g[f"file_{name}"].tobytes())
        assert wf.dct_payload is not None
        stacks = bitstream.decode_tiles(wf.prim_raw, wf.toc)
        recs = [Rec([Cand(*p) for p in st], tuple(wf.residuals[i])) for i, st in enumerate(stacks)]
        maps = [m.astype(np.float32) / 255.0 for m in wf.res1_maps]
        img = orender.render_scene_adaptive(recs, [QT(*q) for q in wf.qtree], wf.width, wf.height, maps, 4)
        img = odct.apply_dct_block(img, wf.dct_payload, wf.qtree)
        np.testing.assert_array_equal(img, g[f"native_{name}"])
        np.testing.assert_array_equal(odct.raster_finish(img, 200, 150), g[f"up_{name}"])
        np.testing.assert_array_equal(odct.raster_finish(img, 50, 37), g[f"down_{name}"])
    assert len(odct.unpack_dct(wf.dct_payload)["scales_u8"]) == len(wf.qtree)  # file b: adaptive quant


def kernel_zigzag_pos(n: int) -> np.ndarray:
    """The closed form weftk_dct.cu uses for the zigzag position of row-major (u, v)."""
    out = np.zeros(n * n, np.int64)
    for u in range(n):
        for v in range(n):
            s = u + v
            before = s * (s + 1) // 2 if s < n else n * n - (2 * n - 1 - s) * (2 * n - s) // 2
            lo, hi = max(0, s - n + 1), min(s, n - 1)
            out[u * n + v] = before + (hi - u if s % 2 == 0 else u - lo)
    return out


@pytest.mark.parametrize("n", [2, 4, 8, 16, 32, 64])
def test_kernel_zigzag_closed_form(n):
    zz = odct.zigzag(n)
    inv = np.empty_like(zz)
    inv[zz] = np.arange(n * n)
    np.testing.assert_array_equal(kernel_zigzag_pos(n), inv)


def test_kernel_table_offsets():
    offs = [((1 << (2 * L)) - 4) // 3 for L in range(1, 8)]
    assert offs[:6] == [0, 4, 20, 84, 340, 1364] and offs[6] == 5460  # 5460 entries for n = 2..64


@pytest.mark.parametrize("i", range(N_CASES))
def test_tile_table_addresses_reproduce_tile_major_blocks(golden, i):
    """Gathering each descriptor's coefficients with the kernel's address rule gives the blocks of
    the oracle's band-to-tile permutation."""
    g = golden("dct.npz")
    tiles = [tuple(int(v) for v in t) for t in g["tiles"]]
    h, w = g["recon"].shape[:2]
    blob = _blob(g, i)
    block = raster.unpack_dct(blob)
    o = odct.unpack_dct(blob)
    pres = odct.presence(o["mask"], len(tiles)) if o["mask"] else [True] * len(tiles)
    present = [t for t, p in zip(tiles, pres) if p]
    coeffs = o["coeffs"]
    if o["layout"] == 1:
        coeffs = odct.permute_band_to_tile(coeffs, [s for _, _, s in present], o["chroma_mode"])
    want, cur = {}, 0
    for k, (x, y, s) in enumerate(present):
        blocks = []
        for n in odct.channel_sizes(s, o["chroma_mode"]):
            blocks.append(coeffs[cur:cur + n * n])
            cur += n * n
        scale = odct.tile_scale(o["scales_u8"][k]) if o["scales_u8"] else 1.0
        want[(x, y)] = (blocks, scale)
    descs = raster.tile_table(block, tiles, w, h)
    assert len(descs) == sum(1 for x, y, _ in present if x < w and y < h)
    assert np.all(np.diff(descs["size"]) >= 0)
    for d in descs:
        blocks, scale = want[(int(d["x"]), int(d["y"]))]
        assert d["step_scale"] == scale
        for c, ref_blk in enumerate(blocks):
            n = int(np.sqrt(ref_blk.size))
            pos = kernel_zigzag_pos(n) if block.layout == 1 else np.arange(n * n)
            addr = int(d["coef_base"][c]) + pos * int(d["coef_stride"][c])
            assert addr.min() >= 0 and addr.max() < block.coeffs.size
            np.testing.assert_array_equal(block.coeffs[addr], ref_blk)


@pytest.mark.parametrize("i", range(N_CASES))
def test_unpack_matches_oracle(golden, i):
    g = golden("dct.npz")
    b = raster.unpack_dct(_blob(g, i))
    o = odct.unpack_dct(_blob(g, i))
    np.testing.assert_array_equal(b.coeffs, o["coeffs"])
    assert (b.quant_step, b.channels, b.freq_alpha, b.chroma_mode, b.presence_bitmask, b.n_tiles, b.layout,
            b.scales_u8) == (o["quant_step"], o["channels"], o["freq_alpha"], o["chroma_mode"], o["mask"],
                             o["n_tiles"], o["layout"], o["scales_u8"])


def test_unpack_and_table_errors(golden):
    g = golden("dct.npz")
    blob = _blob(g, 2)  # v5, band layout, per-tile scales
    with pytest.raises(ValueError, match="truncated"):
        raster.unpack_dct(b"")
    with pytest.raises(ValueError, match="truncated"):
        raster.unpack_dct(blob[:10])
    with pytest.raises(ValueError, match="unsupported"):
        raster.unpack_dct(b"\x07" + blob[1:])
    with pytest.raises(ValueError, match="size mismatch"):
        raster.unpack_dct(blob + b"\x00\x00")
    tiles = [tuple(int(v) for v in t) for t in g["tiles"]]
    block = raster.unpack_dct(blob)
    short = raster.DctBlock(**{**block.__dict__, "coeffs": block.coeffs[:-1]})
    with pytest.raises(ValueError, match="size mismatch"):
        raster.tile_table(short, tiles, 100, 72)
    fewer = raster.DctBlock(**{**block.__dict__, "scales_u8": block.scales_u8[:-1]})
    with pytest.raises(ValueError, match="per_tile_scales"):
        raster.tile_table(fewer, tiles, 100, 72)
    odd = [(0, 0, 12)] + tiles[1:]
    every = raster.unpack_dct(_blob(g, 3))  # every tile present, tile-major
    with pytest.raises(ValueError, match="power-of-two"):
        raster.tile_table(every, odd, 100, 72)


def test_empty_presence_gives_no_descriptors(golden):
    g = golden("dct.npz")
    tiles = [tuple(int(v) for v in t) for t in g["tiles"]]
    block = raster.unpack_dct(_blob(g, 7))
    assert block.coeffs.size == 0 and not any(block.presence_bitmask)
    assert len(raster.tile_table(block, tiles, 100, 72)) == 0


def test_u8_probe_inputs_survive_the_float_path():
    """(u8 + 0.5) / 255 in float32, times 255 in float32, truncates back to u8 for every value: the
    GPU resize test feeds Pillow's u8 inputs through the decoder's float path this way."""
    u = np.arange(256, dtype=np.float32)
    f = (u + np.float32(0.5)) / np.float32(255.0)
    back = np.clip(f * np.float32(255.0), 0.0, 255.0).astype(np.uint8)
    np.testing.assert_array_equal(back, np.arange(256, dtype=np.uint8))


def test_entry_points_reject_bad_arguments_without_gpu_work():
    lib = _lib.load()
    img = np.zeros(3, np.float32)
    rc = lib.weftk_dct_apply(0, 0, 0, 0, 3, 0, 0.01, 0.0, 16, _lib.ptr(img), 1, 1, 0, 0)
    assert rc == -1 and "chroma_mode" in _lib.last_error()
    rc = lib.weftk_dct_apply(0, 0, 0, 0, 2, 0, 0.01, 0.0, 12, _lib.ptr(img), 1, 1, 0, 0)
    assert rc == -1 and "max_size" in _lib.last_error()
    rc = lib.weftk_dct_apply(0, 0, 0, 0, 2, 2, 0.01, 0.0, 16, _lib.ptr(img), 1, 1, 0, 0)
    assert rc == -1 and "layout" in _lib.last_error()
    rc = lib.weftk_raster_resize(0, 4, 4, 0, 8, 8, 0, 0)
    assert rc == -1 and "null" in _lib.last_error()
    rc = lib.weftk_raster_resize(_lib.ptr(img), 0, 4, _lib.ptr(img), 8, 8, _lib.ptr(img), 0)
    assert rc == -1 and "sizes" in _lib.last_error()


def test_legacy_block_versions_parse():
    coeffs = np.arange(-5, 5, dtype=np.int16)
    v2 = struct.pack("<BBffHI", 2, 1, 0.02, 4.0, 3, coeffs.size) + coeffs.tobytes()
    b = raster.unpack_dct(v2)
    assert (b.chroma_mode, b.layout, b.n_tiles, b.presence_bitmask, b.scales_u8) == (1, 0, 0, b"", b"")
    np.testing.assert_array_equal(b.coeffs, coeffs)
    v3 = struct.pack("<BBffHII", 3, 2, 0.02, 0.0, 3, 9, coeffs.size) + b"\xff\x01" + coeffs.tobytes()
    b = raster.unpack_dct(v3)
    assert (b.chroma_mode, b.layout, b.n_tiles, b.presence_bitmask) == (2, 0, 9, b"\xff\x01")


class _RecordingLib:
    """Stands in for libweftk: checks each call against the bound signature and records it."""

    def __init__(self):
        self.calls = []

    def __getattr__(self, name):
        def call(*args):
            sig = _lib.SIGNATURES[name]
            assert len(args) == len(sig), name
            for a, t in zip(args, sig):
                t.from_param(a)  # raises on a type ctypes would reject
            self.calls.append((name, args))
            return 0
        return call


def test_dct_launch_enqueues_one_launch_per_tile_side(golden):
    """Host marshalling of ``DctLaunch.run`` with host arrays in place of device buffers."""
    g = golden("dct.npz")
    tiles = [tuple(int(v) for v in t) for t in g["tiles"]]
    layer = object.__new__(raster.DctLaunch)
    layer.block = raster.unpack_dct(_blob(g, 1))
    layer.descs = raster.tile_table(layer.block, tiles, 100, 72)
    layer.width, layer.height = 100, 72
    layer.lib = _RecordingLib()
    layer.t_coeffs = layer.block.coeffs
    layer.t_descs = layer.descs.view(np.uint8)
    sizes = layer.descs["size"]
    layer.groups = [(int(v), int(np.searchsorted(sizes, v, "left")), int(np.searchsorted(sizes, v, "right")))
                    for v in np.unique(sizes)]
    img = np.zeros((72, 100, 3), np.float32)
    layer.run(img, 0)
    calls = layer.lib.calls
    assert len(calls) == layer.launches == len(np.unique(sizes)) + 1
    base = layer.t_descs.ctypes.data
    seen = 0
    for (name, a), (s, lo, hi) in zip(calls, layer.groups):
        assert name == "weftk_dct_apply"
        assert a[0] == base + 64 * lo and a[1] == hi - lo and a[8] == s and a[12] == 0
        assert np.all(layer.descs["size"][lo:hi] == s)
        seen += hi - lo
    assert seen == len(layer.descs)
    name, a = calls[-1]
    assert name == "weftk_dct_apply" and a[1] == 0 and a[12] == 1 and a[9] == img.ctypes.data
    n = raster._channel_sides(layer.descs["size"].astype(np.int64), layer.block.chroma_mode)
    assert layer.flops() == pytest.approx(float(np.sum(4.0 * n.astype(np.float64) ** 3)))


def test_resize_into_checks_scratch_and_marshals(monkeypatch):
    rec = _RecordingLib()
    monkeypatch.setattr(_lib, "lib_for_device", lambda device=0: rec)

    class _T:
        """Minimal tensor stand-in: shape, numel, device index and a data pointer."""

        def __init__(self, shape, n):
            self.shape, self._n = shape, n
            self.device = type("D", (), {"index": 0})()
            self.buf = np.zeros(max(n, 1), np.uint8)

        def numel(self):
            return self._n

        def data_ptr(self):
            return self.buf.ctypes.data

    src, out = _T((48, 64, 3), 48 * 64 * 3), _T((135, 240, 3), 135 * 240 * 3)
    with pytest.raises(ValueError, match="scratch"):
        raster.resize_into(src, out, _T((1,), 48 * 240 * 3 - 1), 0)
    raster.resize_into(src, out, _T((1,), 48 * 240 * 3), 0)
    name, a = rec.calls[-1]
    assert name == "weftk_raster_resize" and a[1:3] == (64, 48) and a[4:6] == (240, 135)


def test_bench_synthetic_dct_block_is_a_valid_block():
    """The bench's raster-branch payload parses, covers every tile and decodes with the oracle."""
    import bench
    from weft_b200 import quadtree
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(128, 128, 30, 3)
    img = srgb_u8_to_linear(u8)
    tiles = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    blob = bench.synthetic_dct_block(tiles, 75)
    block = raster.unpack_dct(blob)
    assert (block.chroma_mode, block.layout, block.freq_alpha, block.n_tiles) == (2, 0, 4.0, len(tiles))
    assert block.quant_step == pytest.approx(0.01352, rel=1e-6)
    qt = [(t.x, t.y, t.size) for t in tiles]
    descs = raster.tile_table(block, qt, 128, 128)
    assert len(descs) == len(tiles)
    out = odct.apply_dct_block(img, blob, qt)
    assert out.shape == img.shape and 0.0 <= out.min() and out.max() <= 1.0
    assert 0.0 < float(np.sqrt(np.mean((out - np.clip(img, 0, 1)) ** 2))) < 0.2


def test_bench_cpu_decode_baselines_run_on_a_small_scene():
    """The bench's CPU decode baselines on a 128² scene with a stand-in fit (tile-mean constants)."""
    import bench
    from oracle import render as orender
    from weft_b200 import quadtree
    from weft_b200.candidates import Cand
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(128, 128, 30, 4)
    img = srgb_u8_to_linear(u8)
    tiles = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, tiles, 64)

    class Fit:
        def selected(self):
            return [[Cand(0, (), tuple(float(v) for v in p.reshape(-1, 3).mean(0)), None, 1.0)] for p in patches]

        def recon_tiles(self):
            return [orender.render_tile(s, p.shape[0]) for s, p in zip(self.selected(), patches)]

    walk, ras = bench.cpu_decode_baselines(Fit(), tiles, patches, 128, 480, 270)
    for d in (walk, ras):
        assert d["value"] > 0 and d["unit"] == "MPix/s" and d["cores"] == 1 and d["kind"] == "port"


def test_tile_table_with_float_scales_matches_u8_scales(golden):
    """The drop-in path passes the reference's float ``per_tile_scales``; the descriptors equal those
    built from the block's u8 scales."""
    g = golden("dct.npz")
    tiles = [tuple(int(v) for v in t) for t in g["tiles"]]
    block = raster.unpack_dct(_blob(g, 2))
    assert block.scales_u8
    a = raster.tile_table(block, tiles, 100, 72)
    b = raster.tile_table(raster.DctBlock(**{**block.__dict__, "scales_u8": b""}), tiles, 100, 72,
                          scales=[odct.tile_scale(u) for u in block.scales_u8])
    np.testing.assert_array_equal(a, b)
    with pytest.raises(ValueError, match="per_tile_scales"):
        raster.tile_table(block, tiles, 100, 72, scales=[1.0])


def test_install_raster_into_swaps_the_reference_entry():
    import types

    import weft_b200

    mod = types.SimpleNamespace(apply_residual_to_image=None)
    weft_b200.install_raster_into(mod)
    assert mod.apply_residual_to_image is raster.apply_residual_to_image
