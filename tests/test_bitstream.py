"""The product's WEFT writer/reader against the reference's bytes (golden fixtures)."""

from __future__ import annotations

import numpy as np

from oracle.primitives import prims_from_pack
from tests.test_oracle_golden import _pack
from weft_b200 import bitstream
from weft_b200.candidates import Cand


def test_rans_and_chunks_bit_exact(golden):
    g = golden("entropy.npz")
    pay, po, enc, eo = g["payload"], g["payload_off"], g["encoded"], g["encoded_off"]
    for i in range(len(po) - 1):
        data = pay[po[i]:po[i + 1]].tobytes()
        want = enc[eo[i]:eo[i + 1]].tobytes()
        assert bitstream.encode_bytes(data) == want, f"payload {i}"
        assert bitstream.decode_bytes(want) == data
    raw = g["prim_raw"].tobytes()
    toc = [int(v) for v in g["toc"]]
    for n, key in ((64, "64"), (7, "7")):
        coded, entries = bitstream.build_prim_chunks(raw, toc, n)
        assert coded == g["coded" + key].tobytes()
        assert entries == [tuple(int(v) for v in e) for e in g["entries" + key]]


def test_tile_payloads_bit_exact(golden):
    g = golden("quant.npz")
    a = _pack(g, "in_")
    prims = prims_from_pack(a, 0, len(a["kind"]))
    stacks, k = [], 0
    for c in g["tile_counts"]:
        stacks.append(prims[k:k + int(c)])
        k += int(c)
    blob, toc = bitstream.encode_tiles(stacks)
    assert blob == g["tiles_raw"].tobytes()
    assert toc == [int(v) for v in g["toc"]]
    back = bitstream.decode_tiles(blob, toc)
    assert [len(t) for t in back] == [len(s) for s in stacks]


def test_reader_parses_reference_file_and_writer_reproduces_its_payloads(golden):
    g = golden("container.npz")
    blob_a = g["file_a"].tobytes()
    wf = bitstream.decode_weft(blob_a)
    tiles = [type("QT", (), {"x": x, "y": y, "size": s})() for x, y, s in wf.qtree]
    stacks = [[Cand(k, gg, c0, c1, al) for k, gg, c0, c1, al in st] for st in bitstream.decode_tiles(wf.prim_raw, wf.toc)]
    blob = bitstream.encode_weft(wf.width, wf.height, wf.quality, tiles, stacks, wf.residuals, wf.res1_maps)
    assert blob == g["file_b"].tobytes()  # the file the reference decoder was shown to read
    wb = bitstream.decode_weft(blob)
    assert wb.prim_raw == wf.prim_raw and wb.toc == wf.toc and wb.residuals == wf.residuals
    assert all(np.array_equal(x, y) for x, y in zip(wb.res1_maps, wf.res1_maps))


def test_edge_cases_round_trip():
    """Empty stacks, empty files, one tile, the longest stacks and values at the wire grid's
    limits write and read back (host coder)."""
    class QT:
        def __init__(self, x, y, s):
            self.x, self.y, self.size = x, y, s

    rng = np.random.default_rng(5)
    # every tile empty
    tiles = [QT(0, 0, 64), QT(64, 0, 64)]
    blob = bitstream.encode_weft(128, 64, 75, tiles, [[], []])
    wf = bitstream.decode_weft(blob)
    assert [len(t) for t in bitstream.decode_tiles(wf.prim_raw, wf.toc)] == [0, 0]
    # one tile with a long stack of every kind, geometry and colours at the grid's limits
    kinds = [0, 1, 2, 3, 4] * 9
    stack = []
    for k in kinds:
        glen = {0: 0, 1: 4, 2: 5, 3: 7, 4: 6}[k]
        g = tuple(float(v) for v in rng.choice([0.0, 15.0, 7.5], glen))
        if k in (2, 3):
            g = g[:-1] + (float(rng.choice([0.0, 4.0])),)
        c1 = (1.0, 0.0, 1.0) if k == 1 else None
        stack.append(Cand(k, g, (0.0, 1.0, 0.5), c1, float(rng.choice([0.0, 1.0]))))
    blob = bitstream.encode_weft(64, 64, 92, [QT(0, 0, 64)], [stack])
    wf = bitstream.decode_weft(blob)
    back = bitstream.decode_tiles(wf.prim_raw, wf.toc)[0]
    assert [b[0] for b in back] == kinds
    for b, c in zip(back, stack):
        assert np.allclose(b[1], c.geom, atol=1e-3) and np.allclose(b[2], c.color0, atol=1 / 255)
        assert abs(b[4] - c.alpha) < 1e-4


def test_entropy_round_trip_small_payloads():
    """The reference's own small-payload cases (tests/test_entropy.py): empty, one byte, one
    repeated byte, 64 distinct bytes, a periodic pattern and 1 KiB of random bytes (seeded here).
    The host coder's bytes equal the oracle restatement's and decode back."""
    from oracle import entropy as oent

    payloads = [b"", b"a", b"aaaaaa", bytes(range(64)), bytes([7, 3, 7, 3, 7, 3]) * 20,
                np.random.default_rng(11).integers(0, 256, 1024, dtype=np.uint8).tobytes()]
    for payload in payloads:
        coded = bitstream.encode_bytes(payload)
        assert coded == oent.encode_bytes(payload)
        assert bitstream.decode_bytes(coded) == payload
        assert oent.decode_bytes(coded) == payload


def _valid_file() -> bytes:
    class QT:
        def __init__(self, x, y, s):
            self.x, self.y, self.size = x, y, s

    stack = [Cand(0, (), (0.25, 0.5, 0.75), None, 1.0)]
    return bitstream.encode_weft(32, 16, 75, [QT(0, 0, 16), QT(16, 0, 16)], [stack, []])


def _block(blob: bytes, tag: bytes) -> tuple[int, int, int]:
    """(directory entry offset, block offset, block length) of ``tag``."""
    import struct

    n = struct.unpack_from("<H", blob, 6)[0]
    for i in range(n):
        t, off, ln = struct.unpack_from("<4sQQ", blob, 12 + 20 * i)
        if t == tag:
            return 12 + 20 * i, off, ln
    raise KeyError(tag)


def test_reader_rejects_malformed_files():
    """The reference's rejections (tests/test_bitstream.py: bad magic, truncated header, truncated
    directory) and its HEAD / TOC / required-block checks raise BitstreamError, a ValueError."""
    import struct

    import pytest

    assert issubclass(bitstream.BitstreamError, ValueError)
    with pytest.raises(bitstream.BitstreamError):
        bitstream.decode_weft(b"NOPE\x01\x00\x00\x00")
    with pytest.raises(bitstream.BitstreamError, match="truncated file header"):
        bitstream.decode_weft(b"WEFT")
    with pytest.raises(bitstream.BitstreamError, match="truncated block directory"):
        bitstream.decode_weft(b"WEFT" + bytes([1, 0]) + (1).to_bytes(2, "little") + (0).to_bytes(4, "little"))

    good = _valid_file()
    wf = bitstream.decode_weft(good)
    assert (wf.width, wf.height) == (32, 16)
    with pytest.raises(bitstream.BitstreamError, match="invalid magic"):
        bitstream.decode_weft(b"WEFX" + good[4:])
    with pytest.raises(bitstream.BitstreamError, match="unsupported major version"):
        bitstream.decode_weft(good[:4] + bytes([2]) + good[5:])
    # a block past the end of the file
    d, off, ln = _block(good, b"PRIM")
    bad = bytearray(good)
    struct.pack_into("<Q", bad, d + 12, len(good))
    with pytest.raises(bitstream.BitstreamError, match="block extends past EOF"):
        bitstream.decode_weft(bytes(bad))
    # a required block renamed away
    d, off, ln = _block(good, b"META")
    bad = bytearray(good)
    bad[d:d + 4] = b"XXXX"
    with pytest.raises(bitstream.BitstreamError, match="missing required block: META"):
        bitstream.decode_weft(bytes(bad))
    # HEAD fields out of range: width 0, tile size 0, max primitives 0
    d, off, ln = _block(good, b"HEAD")
    for field_off, fmt, msg in ((0, "<I", "invalid dimensions"), (8, "<H", "invalid tile size"),
                                (10, "<H", "invalid max primitives")):
        bad = bytearray(good)
        struct.pack_into(fmt, bad, off + field_off, 0)
        with pytest.raises(bitstream.BitstreamError, match=msg):
            bitstream.decode_weft(bytes(bad))
    # TOC: a count that does not match the block length, then offsets out of order
    d, off, ln = _block(good, b"TOC ")
    bad = bytearray(good)
    struct.pack_into("<I", bad, off, 7)
    with pytest.raises(bitstream.BitstreamError, match="invalid TOC length"):
        bitstream.decode_weft(bytes(bad))
    n_toc = struct.unpack_from("<I", good, off)[0]
    assert n_toc >= 2
    bad = bytearray(good)
    struct.pack_into("<I", bad, off + 4, 1 << 20)
    with pytest.raises(bitstream.BitstreamError, match="TOC offsets must be monotonic"):
        bitstream.decode_weft(bytes(bad))
