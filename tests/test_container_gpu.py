"""GPU decode of WEFT files: a reference-written file and this repo's re-encode of it."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", ["a", "b"])
def test_gpu_decode_matches_reference_decoder(golden, which):
    from weft_b200.encode import decode_file

    g = golden("container.npz")
    img = decode_file(g[f"file_{which}"].tobytes())
    want = g[f"decoded_{which}"]
    assert img.shape == want.shape
    assert float(np.max(np.abs(img - want))) <= 1.0 / 255.0


def test_fit_encode_decode_roundtrip_rd():
    from weft_b200 import candidates, quadtree
    from weft_b200.encode import encode_fit, rd_score
    from weft_b200.fit import BatchedFit
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(128, 128, 12, 5)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="gradvar", threshold=0.08, min_tile=8, max_tile=32)
    patches = quadtree.extract_tiles(img, qts)
    fit = BatchedFit(patches, [candidates.tile_candidates(p, 75) for p in patches], 75).run()
    blob = encode_fit(128, 128, 75, qts, patches, fit.selected(), fit.recon_tiles())
    r = rd_score(img, blob, 75)
    assert r["psnr_db"] > 20 and 0 < r["bpp"] < 8
    assert r["rd_score"] == pytest.approx(r["psnr_db"] - 4.0 * r["bpp"])
