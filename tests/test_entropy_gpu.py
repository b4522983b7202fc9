"""GPU chunked rANS decode of PRIM payloads, bit-exact against the oracle's coder.

Payloads are built by the oracle's restatement of the reference encoder (order-0 static rANS,
raw fallback, chunks of tiles with a CIDX table), over random bytes of several distributions
and lengths, over a real fitted PRIM stream, and a WEFT file read back with the GPU stage.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import entropy as oe

pytestmark = pytest.mark.gpu


def _payload(rng, n, kind):
    if kind == "skewed":
        return bytes(rng.choice(8, n, p=[0.5, 0.2, 0.1, 0.08, 0.05, 0.04, 0.02, 0.01]).astype(np.uint8))
    if kind == "uniform":
        return bytes(rng.integers(0, 256, n, dtype=np.uint8))
    if kind == "single":
        return bytes([7]) * n
    return bytes(rng.integers(0, 4, n, dtype=np.uint8))


@pytest.mark.parametrize("kind", ["skewed", "uniform", "single", "small"])
def test_random_chunks_decode_bit_exact(kind):
    from weft_b200.bitstream import decode_prim_chunks_gpu

    rng = np.random.default_rng(11)
    for n_tiles in (1, 7, 64, 200):
        lens = rng.integers(0, 40, n_tiles)
        toc = [0] + list(np.cumsum(lens))
        raw = _payload(rng, int(toc[-1]), kind)
        for chunk_tiles in (1, 16, 64):
            payload, entries = oe.build_prim_chunks(raw, toc, chunk_tiles)
            assert oe.decode_prim_payload(payload, toc, entries) == raw
            got = decode_prim_chunks_gpu(payload, entries, len(raw))
            assert got == raw


def test_fitted_prim_stream_and_file_round_trip():
    from weft_b200 import bitstream, candidates, quadtree
    from weft_b200.encode import encode_fit
    from weft_b200.fit import BatchedFit
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(256, 256, 40, 0)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, qts, 64)
    pools = [candidates.tile_candidates(p, 75) for p in patches]
    fit = BatchedFit(patches, pools, 75, caps=[16] * len(qts)).run()
    blob = encode_fit(256, 256, 75, qts, patches, fit.selected(), fit.recon_tiles())
    host = bitstream.decode_weft(blob)
    gpu = bitstream.decode_weft(blob, device=0)
    assert gpu.prim_raw == host.prim_raw and gpu.toc == host.toc


def test_malformed_chunk_is_reported_not_written():
    from weft_b200.bitstream import decode_prim_chunks_gpu

    raw = bytes(range(50)) * 4
    payload, entries = oe.build_prim_chunks(raw, [0, len(raw)], 64)
    bad = bytearray(payload)
    bad[1] ^= 0x01  # the chunk's raw length no longer matches its CIDX entry
    with pytest.raises(ValueError):
        decode_prim_chunks_gpu(bytes(bad), entries, len(raw))
    # and the decoder stays usable
    assert decode_prim_chunks_gpu(payload, entries, len(raw)) == raw
