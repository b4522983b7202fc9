"""WEFT v1.4 container for primitive-stack encodes (host side).

Writes and reads the blocks the adaptive primitive encoder produces, byte for
byte as the reference does, so files are interchangeable:

* primitive payloads per tile (src/weft/primitives.py:102-177, :315-340) with
  the wire quantization (u16 geometry over [0, 15], thickness over [0, 4], u8
  colours, u16 alpha; Python ``round`` = half to even);
* chunked order-0 rANS of the PRIM payload, 64 tiles per chunk, raw when rANS
  is not smaller (src/weft/entropy.py:30-217, src/weft/prim_chunks.py:23-77);
* HEAD / TOC / CIDX / RES0 / RES1 / QTRE / META blocks, 64-byte alignment,
  SHA-256 in META (src/weft/bitstream.py:150-330, :724-818, :839-967).

Blocks are written uncompressed: the reference compresses with zstd only when
the optional ``zstandard`` module is importable (src/weft/bitstream.py:55-71),
which its own lock file does not provide; its decoder accepts both.
"""

from __future__ import annotations

import hashlib
import json
import struct
from dataclasses import dataclass, field

import numpy as np

MAGIC = b"WEFT"
MAJOR, MINOR = 1, 4


class BitstreamError(ValueError):
    """A malformed WEFT file (the reference's ``weft.bitstream.BitstreamError``,
    src/weft/bitstream.py:44; the same checks in the same order as its ``decode_weft``,
    :839-870, ``_unpack_head`` :177-200 and ``_unpack_toc`` :222-233)."""
FLAG_DETERMINISTIC, FLAG_HAS_RES0, FLAG_HAS_RES1, FLAG_CHUNKED_PRIM = 1, 2, 4, 8
FLAG_HAS_DCT = 1 << 9
PROB_BITS = 12
TOTFREQ = 1 << PROB_BITS
RANS_L = 1 << 23
GEOM_RANGES = {0: (), 1: ((0.0, 15.0),) * 4, 2: ((0.0, 15.0),) * 4 + ((0.0, 4.0),),
               3: ((0.0, 15.0),) * 6 + ((0.0, 4.0),), 4: ((0.0, 15.0),) * 6}


# ------------------------------------------------------------------ primitive payloads
def _unit(v, lo, hi):
    x = (v - lo) / (hi - lo)
    return 0.0 if x < 0.0 else 1.0 if x > 1.0 else x


def _qu8(v) -> int:
    return int(round(_unit(float(v), 0.0, 1.0) * 255.0))


def _qu16(v, lo, hi) -> int:
    return int(round(_unit(float(v), lo, hi) * 65535.0))


def encode_primitive(kind: int, geom, color0, color1, alpha) -> bytes:
    """``<kind u8><len u8><payload>`` for one primitive."""
    if kind == 5:
        payload = bytes(max(0, min(255, int(round(float(v) * 255.0)))) for v in geom[:48])
    elif kind in GEOM_RANGES:
        rng = GEOM_RANGES[kind]
        payload = b"".join(struct.pack("<H", _qu16(v, lo, hi)) for v, (lo, hi) in zip(geom, rng))
        payload += bytes(_qu8(c) for c in color0[:3])
        if kind == 1:
            payload += bytes(_qu8(c) for c in color1[:3])
        payload += struct.pack("<H", _qu16(alpha, 0.0, 1.0))
    else:
        raise ValueError(f"unsupported primitive kind {kind}")
    return struct.pack("<BB", kind, len(payload)) + payload


def encode_tiles(stacks) -> tuple[bytes, list[int]]:
    """Tile payloads back to back (``<count u8>`` + primitives) and the TOC."""
    out, toc = bytearray(), [0]
    for prims in stacks:
        if len(prims) > 48:
            raise ValueError("tile has too many primitives")
        out.append(len(prims))
        for p in prims:
            out += encode_primitive(p.kind, tuple(p.geom), tuple(p.color0),
                                    tuple(p.color1) if p.color1 is not None else (0.0, 0.0, 0.0), p.alpha)
        toc.append(len(out))
    return bytes(out), toc


# ------------------------------------------------------------------ rANS
def _freqs(data: bytes) -> list[int]:
    counts = np.bincount(np.frombuffer(data, np.uint8), minlength=256).tolist()
    total = len(data)
    f = [max(1, int(round((c / total) * TOTFREQ))) if c > 0 else 0 for c in counts]
    if sum(f) == 0:
        f[0] = TOTFREQ
    diff = TOTFREQ - sum(f)
    order = sorted(range(256), key=lambda i: counts[i], reverse=True)  # stable
    k = 0
    while diff != 0 and k < 100000:
        idx = order[k % 256]
        if counts[idx] == 0:
            idx = 0
        if diff > 0:
            f[idx] += 1
            diff -= 1
        elif f[idx] > 1:
            f[idx] -= 1
            diff += 1
        k += 1
    if sum(f) != TOTFREQ:
        f[0] += TOTFREQ - sum(f)
    return f


def rans_encode(data: bytes) -> bytes:
    if not data:
        return struct.pack("<BI", 0, 0)
    f = _freqs(data)
    cum = np.concatenate([[0], np.cumsum(f)]).tolist()
    x = RANS_L
    em = bytearray()
    for s in reversed(data):
        fs = f[s]
        xm = ((RANS_L >> PROB_BITS) << 8) * fs
        while x >= xm:
            em.append(x & 0xFF)
            x >>= 8
        x = ((x // fs) << PROB_BITS) + (x % fs) + cum[s]
    pairs = [(s, f[s]) for s in range(256) if f[s] > 0]
    hdr = struct.pack("<BIH", 1, len(data), len(pairs)) + b"".join(struct.pack("<BH", s, v) for s, v in pairs)
    return hdr + struct.pack("<II", x, len(em)) + bytes(em)


def encode_bytes(data: bytes) -> bytes:
    """rANS if smaller than the raw form, else raw (``<0 u8><len u32><bytes>``)."""
    raw = struct.pack("<BI", 0, len(data)) + data
    if not data:
        return raw
    r = rans_encode(data)
    return r if len(r) < len(raw) else raw


def decode_bytes(payload: bytes) -> bytes:
    if not payload:
        return b""
    if payload[0] == 0:
        n = struct.unpack_from("<I", payload, 1)[0]
        if 5 + n != len(payload):
            raise ValueError("raw length mismatch")
        return payload[5:]
    if payload[0] != 1:
        raise ValueError("unknown entropy mode")
    n, ns = struct.unpack_from("<IH", payload, 1)
    off = 7
    f = [0] * 256
    for _ in range(ns):
        s, v = struct.unpack_from("<BH", payload, off)
        f[s] = v
        off += 3
    cum = np.concatenate([[0], np.cumsum(f)]).tolist()
    if cum[256] != TOTFREQ:
        raise ValueError("bad frequency sum")
    lookup = np.repeat(np.arange(256), f).tolist()
    x, m = struct.unpack_from("<II", payload, off)
    off += 8
    if off + m != len(payload):
        raise ValueError("emitted length mismatch")
    em = payload[off:]
    ptr = m - 1
    out = bytearray(n)
    for i in range(n):
        slot = x & (TOTFREQ - 1)
        s = lookup[slot]
        out[i] = s
        x = f[s] * (x >> PROB_BITS) + slot - cum[s]
        while x < RANS_L and ptr >= 0:
            x = (x << 8) | em[ptr]
            ptr -= 1
    return bytes(out)


def build_prim_chunks(prim_raw: bytes, toc: list[int], chunk_tiles: int = 64):
    n = len(toc) - 1
    coded, entries, pos = [], [], 0
    for st in range(0, n, chunk_tiles):
        en = min(n, st + chunk_tiles)
        c = encode_bytes(prim_raw[toc[st]:toc[en]])
        entries.append((st, en - st, toc[st], toc[en] - toc[st], pos, len(c)))
        coded.append(c)
        pos += len(c)
    return b"".join(coded), entries


# ------------------------------------------------------------------ container
@dataclass
class WeftFile:
    width: int
    height: int
    quality: int
    toc: list
    prim_raw: bytes
    residuals: list | None
    res1_maps: list | None       # per tile (4, 4, 3) int8
    qtree: list                  # (x, y, size)
    meta: dict = field(default_factory=dict)
    dct_payload: bytes | None = None   # BLOCK_DCT body (per-tile DCT residual layer)


def _align(v: int, a: int) -> int:
    return v if v % a == 0 else v + (a - v % a)


def encode_weft(width: int, height: int, quality: int, tiles, stacks, residuals=None, res1_maps=None,
                chunk_tiles: int = 64, encode_size=None, extra_meta=None) -> bytes:
    """Container bytes for an adaptive primitive-stack encode.

    ``tiles``: quad tiles (x, y, size); ``stacks``: per-tile primitives;
    ``residuals``: per-tile RES0 (r, g, b) ints or None; ``res1_maps``: per-tile
    (4, 4, 3) int8 arrays or None.
    """
    prim_raw, toc = encode_tiles(stacks)
    prim_payload, entries = build_prim_chunks(prim_raw, toc, chunk_tiles)
    flags = FLAG_DETERMINISTIC | FLAG_CHUNKED_PRIM
    if residuals is not None:
        flags |= FLAG_HAS_RES0
    if res1_maps is not None:
        flags |= FLAG_HAS_RES1
    caps = {8: 24, 16: 48, 32: 96}
    head = struct.pack("<IIHHBBHIIBBH", width, height, 16, max(caps.get(t.size, 48) for t in tiles), 1, 2, flags,
                       0, 0, quality, 2, 0)
    toc_b = struct.pack("<I", len(toc)) + np.asarray(toc, "<u4").tobytes()
    cidx = struct.pack("<I", len(entries)) + b"".join(struct.pack("<IIIIII", *e) for e in entries)
    res0 = None
    if residuals is not None:
        r = np.asarray(residuals, np.int64)
        if r.size and (r.min() < -127 or r.max() > 127):
            raise ValueError("residual out of range")
        res0 = struct.pack("<I", len(residuals)) + r.astype("<i1").tobytes()
    res1 = None
    if res1_maps is not None:
        res1 = struct.pack("<IBBH", len(res1_maps), 4, 4, 0) + b"".join(
            np.asarray(m, np.int8).reshape(48).tobytes() for m in res1_maps)
    qtree = struct.pack("<I", len(tiles)) + b"".join(struct.pack("<HHB", t.x, t.y, t.size) for t in tiles)
    ew, eh = encode_size if encode_size is not None else (width, height)
    meta = {"quality": quality, "entropy": "chunked-rans", "chunk_tiles": chunk_tiles, "chunked_prim": True,
            "prim_chunks": len(entries), "head_flags": flags, "res1_grid_size": 4 if res1 is not None else 0,
            "adaptive_tiling": True, "tile_count": len(tiles), "encode_scale": 1.0, "source_width": width,
            "source_height": height, "encode_width": ew, "encode_height": eh, "deterministic": True,
            "decompose_lighting": False, "lighting_grid_h": 0, "lighting_grid_w": 0, "dct_residual": False,
            "qtree_payload_bytes": len(qtree), "encoder": "weft-b200"}
    if extra_meta:
        meta.update(extra_meta)
    checksum = hashlib.sha256(head + toc_b + prim_payload + (res0 or b"") + (res1 or b"") + cidx + qtree).hexdigest()
    body = json.dumps({**meta, "sha256": checksum, "block_alignment": 64}, sort_keys=True,
                      separators=(",", ":")).encode()
    meta_b = struct.pack("<I", len(body)) + body
    blocks = [(b"HEAD", head), (b"TOC ", toc_b), (b"PRIM", prim_payload), (b"CIDX", cidx)]
    if res0 is not None:
        blocks.append((b"RES0", res0))
    if res1 is not None:
        blocks.append((b"RES1", res1))
    blocks += [(b"QTRE", qtree), (b"META", meta_b)]
    header = struct.pack("<4sBBHI", MAGIC, MAJOR, MINOR, len(blocks), 0)
    dir_size = len(blocks) * 20
    first = _align(len(header) + dir_size, 64)
    directory, payload = bytearray(), bytearray(b"\x00" * (first - len(header) - dir_size))
    running = len(payload)
    for tag, body_ in blocks:
        pad = _align(running, 64) - running
        payload += b"\x00" * pad
        running += pad
        directory += struct.pack("<4sQQ", tag, len(header) + dir_size + running, len(body_))
        payload += body_
        running += len(body_)
    return bytes(header + directory + payload)


def decode_prim_chunks_gpu(prim: bytes, entries, out_len: int, device: int = 0) -> bytes:
    """The PRIM payload's chunks decoded on the GPU (``weftk_rans_decode_chunks``, one warp per
    chunk); ``entries`` are CIDX rows (start_tile, tile_count, raw_off, raw_len, coded_off, coded_len)."""
    import torch

    from . import _lib

    lib = _lib.lib_for_device(device)
    d = torch.device("cuda", device)
    ent = np.array([(e[4], e[5], e[2], e[3]) for e in entries], np.int64).reshape(-1, 4)
    t_pay = torch.from_numpy(np.frombuffer(prim, np.uint8).copy()).to(d) if len(prim) else \
        torch.zeros(1, dtype=torch.uint8, device=d)
    t_ent = torch.from_numpy(ent).to(d)
    t_out = torch.zeros(max(out_len, 1), dtype=torch.uint8, device=d)
    status = ctypes_int()
    lib.weftk_device_status(ctypes_addr_of(status))  # clear any earlier report
    rc = lib.weftk_rans_decode_chunks(_lib.ptr(t_pay), len(prim), _lib.ptr(t_ent), len(ent), _lib.ptr(t_out),
                                      out_len, torch.cuda.current_stream(d).cuda_stream)
    _lib.check(rc, "weftk_rans_decode_chunks")
    out = t_out[:out_len].cpu().numpy().tobytes()
    _lib.check(lib.weftk_device_status(ctypes_addr_of(status)), "weftk_device_status")
    if status.value:
        raise ValueError("a PRIM chunk does not parse")
    return out


def ctypes_int():
    import ctypes

    return ctypes.c_int(0)


def ctypes_addr_of(v) -> int:
    import ctypes

    return ctypes.addressof(v)


def decode_weft(blob: bytes, device: int | None = None) -> WeftFile:
    """Parse a WEFT file; with ``device`` the PRIM chunks are entropy-decoded on that GPU.
    A malformed file raises ``BitstreamError``."""
    if len(blob) < 12:
        raise BitstreamError("truncated file header")
    magic, major, minor, n_blocks, _ = struct.unpack_from("<4sBBHI", blob, 0)
    if magic != MAGIC:
        raise BitstreamError("invalid magic")
    if major != MAJOR:
        raise BitstreamError(f"unsupported major version: {major}")
    if 12 + 20 * n_blocks > len(blob):
        raise BitstreamError("truncated block directory")
    blocks = {}
    off = 12
    for _ in range(n_blocks):
        tag, b_off, b_len = struct.unpack_from("<4sQQ", blob, off)
        off += 20
        if b_off + b_len > len(blob):
            raise BitstreamError("block extends past EOF")
        blocks[tag] = blob[b_off:b_off + b_len]
    for tag in (b"HEAD", b"TOC ", b"PRIM", b"META", b"QTRE"):
        if tag not in blocks:
            raise BitstreamError(f"missing required block: {tag.decode('ascii').strip()}")
    for tag in blocks:
        if blocks[tag][:4] == b"\x28\xb5\x2f\xfd":
            raise BitstreamError("zstd-compressed blocks are not supported")
    if len(blocks[b"HEAD"]) != struct.calcsize("<IIHHBBHIIBBH"):
        raise BitstreamError("invalid HEAD size")
    w, h, ts, mp, _cs, _qm, flags, _tc, _tr, quality, _pid, _ = struct.unpack("<IIHHBBHIIBBH", blocks[b"HEAD"])
    if w <= 0 or h <= 0:
        raise BitstreamError("invalid dimensions")
    if ts <= 0 or ts > 64:
        raise BitstreamError("invalid tile size")
    if mp <= 0 or mp > 255:
        raise BitstreamError("invalid max primitives")
    toc_b = blocks[b"TOC "]
    if len(toc_b) < 4:
        raise BitstreamError("truncated TOC")
    n_toc = struct.unpack_from("<I", toc_b, 0)[0]
    if len(toc_b) != 4 + 4 * n_toc:
        raise BitstreamError("invalid TOC length")
    toc = list(np.frombuffer(toc_b, "<u4", n_toc, 4).astype(np.int64))
    if any(b < a for a, b in zip(toc, toc[1:])):
        raise BitstreamError("TOC offsets must be monotonic")
    prim = blocks[b"PRIM"]
    if b"CIDX" in blocks and device is not None:
        nc = struct.unpack_from("<I", blocks[b"CIDX"], 0)[0]
        entries = [struct.unpack_from("<IIIIII", blocks[b"CIDX"], 4 + 24 * i) for i in range(nc)]
        prim_raw = decode_prim_chunks_gpu(prim, entries, int(toc[-1]) if toc else 0, device)
    elif b"CIDX" in blocks:
        nc = struct.unpack_from("<I", blocks[b"CIDX"], 0)[0]
        raw = bytearray(toc[-1] if toc else 0)
        for i in range(nc):
            _st, _tc2, ro, rl, co, cl = struct.unpack_from("<IIIIII", blocks[b"CIDX"], 4 + 24 * i)
            part = decode_bytes(prim[co:co + cl])
            if len(part) != rl:
                raise BitstreamError("chunk length mismatch")
            raw[ro:ro + rl] = part
        prim_raw = bytes(raw)
    else:
        prim_raw = decode_bytes(prim)
    residuals = None
    if b"RES0" in blocks:
        n = struct.unpack_from("<I", blocks[b"RES0"], 0)[0]
        residuals = [tuple(int(v) for v in r) for r in np.frombuffer(blocks[b"RES0"], np.int8, 3 * n, 4).reshape(n, 3)]
    res1 = None
    if b"RES1" in blocks:
        n, gw, gh, _ = struct.unpack_from("<IBBH", blocks[b"RES1"], 0)
        res1 = list(np.frombuffer(blocks[b"RES1"], np.int8, n * gw * gh * 3, 8).reshape(n, gh, gw, 3))
    qn = struct.unpack_from("<I", blocks[b"QTRE"], 0)[0]
    qtree = [struct.unpack_from("<HHB", blocks[b"QTRE"], 4 + 5 * i) for i in range(qn)]
    meta = json.loads(blocks[b"META"][4:].decode())
    if (flags & FLAG_HAS_DCT) and b"DCT " not in blocks:
        raise BitstreamError("HEAD indicates DCT but DCT block is missing")
    return WeftFile(w, h, quality, toc, prim_raw, residuals, res1, qtree, meta, blocks.get(b"DCT "))


def decode_tiles(prim_raw: bytes, toc) -> list[list[tuple]]:
    """Per-tile lists of (kind, geom, color0, color1, alpha) with dequantized values."""
    out = []
    for a, b in zip(toc[:-1], toc[1:]):
        part = prim_raw[a:b]
        n = part[0]
        off = 1
        prims = []
        for _ in range(n):
            k, ln = part[off], part[off + 1]
            pl = part[off + 2: off + 2 + ln]
            off += 2 + ln
            if k == 5:
                prims.append((5, tuple(v / 255.0 for v in pl), (0.0, 0.0, 0.0), None, 1.0))
                continue
            rng = GEOM_RANGES[k]
            g = tuple(lo + (struct.unpack_from("<H", pl, 2 * j)[0] / 65535.0) * (hi - lo)
                      for j, (lo, hi) in enumerate(rng))
            pos = 2 * len(rng)
            c0 = tuple(v / 255.0 for v in pl[pos:pos + 3])
            pos += 3
            c1 = None
            if k == 1:
                c1 = tuple(v / 255.0 for v in pl[pos:pos + 3])
                pos += 3
            a_ = struct.unpack_from("<H", pl, pos)[0] / 65535.0
            prims.append((k, g, c0, c1, a_))
        if off != len(part):
            raise ValueError("tile parse did not consume all bytes")
        out.append(prims)
    return out
