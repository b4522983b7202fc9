"""Order-0 static rANS and chunked PRIM payloads (test oracle).

Restates ``src/weft/entropy.py`` (model build :30-84, encoder :87-118,
decoder :121-189, raw/rANS selection :192-217) and ``src/weft/prim_chunks.py``
(``build_prim_chunks`` :23-77, ``decode_prim_payload`` :80-125).

Bit-exactness hinges on two details of the model build: the per-symbol
frequency is ``max(1, round(count / total * 4096))`` with Python's
half-to-even ``round`` on the float64 product, and the correction loop walks
symbols in a stable descending-count order.
"""

from __future__ import annotations

import struct

PROB_BITS = 12
TOTFREQ = 1 << PROB_BITS
RANS_L = 1 << 23
MODE_RAW, MODE_RANS = 0, 1


def build_freqs(data: bytes) -> list[int]:
    counts = [0] * 256
    for b in data:
        counts[b] += 1
    total = sum(counts)
    if total <= 0:
        f = [0] * 256
        f[0] = TOTFREQ
        return f
    f = [max(1, int(round((c / total) * TOTFREQ))) if c > 0 else 0 for c in counts]
    if sum(f) == 0:
        f[0] = TOTFREQ
    diff = TOTFREQ - sum(f)
    order = sorted(range(256), key=lambda i: counts[i], reverse=True)
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


def _cum(freqs: list[int]) -> list[int]:
    cum, run = [0] * 257, 0
    for i, v in enumerate(freqs):
        cum[i] = run
        run += v
    cum[256] = run
    return cum


def encode_rans(data: bytes) -> bytes:
    if not data:
        return struct.pack("<BI", MODE_RAW, 0)
    freqs = build_freqs(data)
    cum = _cum(freqs)
    x = RANS_L
    out = bytearray()
    for s in reversed(data):
        f = freqs[s]
        x_max = ((RANS_L >> PROB_BITS) << 8) * f
        while x >= x_max:
            out.append(x & 0xFF)
            x >>= 8
        x = ((x // f) << PROB_BITS) + (x % f) + cum[s]
    pairs = [(s, freqs[s]) for s in range(256) if freqs[s] > 0]
    hdr = struct.pack("<BIH", MODE_RANS, len(data), len(pairs))
    hdr += b"".join(struct.pack("<BH", s, f) for s, f in pairs)
    return hdr + struct.pack("<II", x, len(out)) + bytes(out)


def decode_rans(payload: bytes) -> bytes:
    mode = payload[0]
    if mode == MODE_RAW:
        n = struct.unpack_from("<I", payload, 1)[0]
        if 5 + n != len(payload):
            raise ValueError("raw length mismatch")
        return payload[5:]
    if mode != MODE_RANS:
        raise ValueError("unknown mode")
    n, n_sym = struct.unpack_from("<IH", payload, 1)
    off = 7
    freqs = [0] * 256
    for _ in range(n_sym):
        s, f = struct.unpack_from("<BH", payload, off)
        freqs[s] = f
        off += 3
    cum = _cum(freqs)
    if cum[256] != TOTFREQ:
        raise ValueError("bad frequency sum")
    lookup = [0] * TOTFREQ
    for s in range(256):
        lookup[cum[s]:cum[s] + freqs[s]] = [s] * freqs[s]
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
        x = freqs[s] * (x >> PROB_BITS) + (slot - cum[s])
        while x < RANS_L and ptr >= 0:
            x = (x << 8) | em[ptr]
            ptr -= 1
    return bytes(out)


def encode_bytes(data: bytes) -> bytes:
    raw = struct.pack("<BI", MODE_RAW, len(data)) + data
    if not data:
        return raw
    r = encode_rans(data)
    return r if len(r) < len(raw) else raw


def decode_bytes(payload: bytes) -> bytes:
    return b"" if not payload else decode_rans(payload)


def build_prim_chunks(prim_raw: bytes, toc: list[int], chunk_tiles: int):
    """Code each run of ``chunk_tiles`` tiles separately; returns (payload, entries).

    Entries are (start_tile, tile_count, raw_offset, raw_length, coded_offset, coded_length).
    """
    if chunk_tiles <= 0:
        raise ValueError("chunk_tiles must be > 0")
    if not toc:
        return b"", []
    n = len(toc) - 1
    coded, entries, pos = [], [], 0
    for start in range(0, n, chunk_tiles):
        end = min(n, start + chunk_tiles)
        c = encode_bytes(prim_raw[toc[start]:toc[end]])
        entries.append((start, end - start, toc[start], toc[end] - toc[start], pos, len(c)))
        coded.append(c)
        pos += len(c)
    return b"".join(coded), entries


def decode_prim_payload(payload: bytes, toc: list[int], entries) -> bytes:
    if not entries:
        return decode_bytes(payload)
    out = bytearray(toc[-1] if toc else 0)
    for (_st, _tc, ro, rl, co, cl) in entries:
        raw = decode_bytes(payload[co:co + cl])
        if len(raw) != rl:
            raise ValueError("chunk raw length mismatch")
        out[ro:ro + rl] = raw
    return bytes(out)
