"""Primitive records, wire quantization and tile serialization (test oracle).

Restates ``src/weft/primitives.py`` (Primitive/TileRecord :27-40, the per-kind
payloads of ``encode_primitive`` :102-177 and ``decode_primitive`` :180-288,
``encode_tiles`` / ``decode_tiles`` :315-340) and ``_quantize_primitive``
(``src/weft/encoder.py:211-237``).  Rounding is Python's ``round`` (half to
even), as in the reference.
"""

from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

GEOM_LEN = {0: 0, 1: 4, 2: 5, 3: 7, 4: 6, 5: 48}
MAX_PRIMS_PER_TILE = 48


@dataclass
class Prim:
    kind: int
    geom: tuple = ()
    color0: tuple = (0.0, 0.0, 0.0)
    color1: tuple | None = None
    alpha: float = 1.0


@dataclass
class Record:
    primitives: list = field(default_factory=list)
    residual_rgb: tuple = (0, 0, 0)


def prims_from_pack(pack: dict, lo: int, hi: int) -> list[Prim]:
    """Rebuild Prim objects from the flat float64 fixture layout."""
    out = []
    for i in range(lo, hi):
        k = int(pack["kind"][i])
        g = tuple(float(v) for v in pack["geom"][i][: GEOM_LEN[k]])
        c1 = tuple(float(v) for v in pack["c1"][i]) if int(pack["has_c1"][i]) else None
        out.append(Prim(k, g, tuple(float(v) for v in pack["c0"][i]), c1, float(pack["alpha"][i])))
    return out


def _unit(v: float, lo: float, hi: float) -> float:
    x = (v - lo) / (hi - lo)
    return 0.0 if x < 0.0 else 1.0 if x > 1.0 else x


def q_u8(v: float, lo: float = 0.0, hi: float = 1.0) -> int:
    return 0 if hi <= lo else int(round(_unit(v, lo, hi) * 255.0))


def q_u16(v: float, lo: float, hi: float) -> int:
    return 0 if hi <= lo else int(round(_unit(v, lo, hi) * 65535.0))


def dq_u8(q: int, lo: float = 0.0, hi: float = 1.0) -> float:
    return lo + (q / 255.0) * (hi - lo)


def dq_u16(q: int, lo: float, hi: float) -> float:
    return lo + (q / 65535.0) * (hi - lo)


def quantize_primitive(p: Prim) -> Prim:
    """Snap to the wire grid without serializing (src/weft/encoder.py:211-237)."""
    def snap_c(c):
        return tuple(round(max(0, min(1, v)) * 255) / 255.0 for v in c)

    def s15(v):
        return round(max(0, min(1, v / 15)) * 65535) / 65535.0 * 15

    def s4(v):
        return round(max(0, min(1, v / 4)) * 65535) / 65535.0 * 4

    g = p.geom
    if p.kind == 0:
        geom = g
    elif p.kind == 2:
        geom = (s15(g[0]), s15(g[1]), s15(g[2]), s15(g[3]), s4(g[4]))
    elif p.kind == 3:
        geom = tuple(s15(v) for v in g[:6]) + (s4(g[6]),)
    else:
        geom = tuple(s15(v) for v in g)
    alpha = round(max(0, min(1, p.alpha)) * 65535) / 65535.0
    return Prim(p.kind, geom, snap_c(p.color0), snap_c(p.color1) if p.color1 is not None else None, alpha)


# wire layout per kind: (geom fields as (lo, hi) ranges, has color1)
_WIRE = {
    0: ((), False),
    1: (((0.0, 15.0),) * 4, True),
    2: (((0.0, 15.0),) * 4 + ((0.0, 4.0),), False),
    3: (((0.0, 15.0),) * 6 + ((0.0, 4.0),), False),
    4: (((0.0, 15.0),) * 6, False),
}


def encode_primitive(p: Prim) -> bytes:
    """``<kind u8><len u8><payload>`` (src/weft/primitives.py:102-177)."""
    k = p.kind
    if k == 5:
        if len(p.geom) != 48:
            raise ValueError("bicubic needs 48 control values")
        payload = bytes(max(0, min(255, int(round(v * 255.0)))) for v in p.geom)
    elif k in _WIRE:
        ranges, has_c1 = _WIRE[k]
        if len(p.geom) != len(ranges) or (has_c1 and p.color1 is None):
            raise ValueError(f"bad geometry for kind {k}")
        payload = b"".join(struct.pack("<H", q_u16(v, lo, hi)) for v, (lo, hi) in zip(p.geom, ranges))
        payload += bytes(q_u8(c) for c in p.color0)
        if has_c1:
            payload += bytes(q_u8(c) for c in p.color1)
        payload += struct.pack("<H", q_u16(p.alpha, 0.0, 1.0))
    else:
        raise ValueError(f"unsupported kind {k}")
    return struct.pack("<BB", k, len(payload)) + payload


def decode_primitive(blob: bytes, off: int) -> tuple[Prim, int]:
    """Inverse of ``encode_primitive`` (src/weft/primitives.py:180-288)."""
    k, n = struct.unpack_from("<BB", blob, off)
    off += 2
    payload = blob[off: off + n]
    if len(payload) != n:
        raise ValueError("truncated primitive")
    if k == 5:
        if n != 48:
            raise ValueError("invalid bicubic payload")
        return Prim(5, tuple(b / 255.0 for b in payload), (0.0, 0.0, 0.0), None, 1.0), off + n
    if k not in _WIRE:
        raise ValueError(f"unsupported kind {k}")
    ranges, has_c1 = _WIRE[k]
    expect = 2 * len(ranges) + 3 + (3 if has_c1 else 0) + 2
    if n != expect:
        raise ValueError("invalid payload length")
    geom = tuple(dq_u16(struct.unpack_from("<H", payload, 2 * j)[0], lo, hi) for j, (lo, hi) in enumerate(ranges))
    pos = 2 * len(ranges)
    c0 = tuple(dq_u8(b) for b in payload[pos: pos + 3])
    pos += 3
    c1 = None
    if has_c1:
        c1 = tuple(dq_u8(b) for b in payload[pos: pos + 3])
        pos += 3
    alpha = dq_u16(struct.unpack_from("<H", payload, pos)[0], 0.0, 1.0)
    return Prim(k, geom, c0, c1, alpha), off + n


def encode_tiles(records) -> tuple[bytes, list[int]]:
    """Concatenate ``<count u8><prims...>`` per tile; TOC of cumulative offsets (src/weft/primitives.py:315-324)."""
    out, toc = bytearray(), [0]
    for r in records:
        if len(r.primitives) > MAX_PRIMS_PER_TILE:
            raise ValueError("too many primitives")
        out += bytes([len(r.primitives)])
        for p in r.primitives:
            out += encode_primitive(p)
        toc.append(len(out))
    return bytes(out), toc


def decode_tiles(blob: bytes, toc: list[int]) -> list[Record]:
    """Inverse of ``encode_tiles`` (src/weft/primitives.py:327-340)."""
    recs = []
    for a, b in zip(toc[:-1], toc[1:]):
        part = blob[a:b]
        n = part[0]
        off = 1
        prims = []
        for _ in range(n):
            p, off = decode_primitive(part, off)
            prims.append(p)
        if off != len(part):
            raise ValueError("tile parse did not consume all bytes")
        recs.append(Record(prims))
    return recs


PRIM_DTYPE = np.dtype([("kind", np.int32), ("geom", np.float32, 7), ("color0", np.float32, 3),
                       ("color1", np.float32, 3), ("alpha", np.float32)])


def pack_prims(prims) -> np.ndarray:
    """Reference 60-byte PrimData records (src/weft/gpu_render.py:241-308)."""
    arr = np.zeros(max(1, len(prims)), PRIM_DTYPE)
    for i, p in enumerate(prims):
        arr[i]["kind"] = p.kind
        g = list(p.geom)[:7]
        arr[i]["geom"][: len(g)] = g
        arr[i]["color0"] = p.color0
        if p.color1 is not None:
            arr[i]["color1"] = p.color1
        arr[i]["alpha"] = p.alpha
    return arr
