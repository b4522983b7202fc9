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
