"""The decoder's raster branch on the GPU: ``weftk_dct_apply`` and ``weftk_raster_resize`` against
the reference's outputs (golden fixtures made by the reference and Pillow), and whole-file decodes
of reference-written files that carry the DCT residual layer."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RESIZE_TARGETS = [(240, 135), (96, 200), (37, 29), (200, 100), (70, 50), (300, 7)]
# float64 transform with fused multiply-adds against scipy's FFT: the float32 results may differ
# in the last place
APPLY_TOL = 2.5e-7


@pytest.mark.parametrize("i", range(12))
def test_dct_apply_matches_reference(golden, i):
    import torch

    from weft_b200 import raster

    g = golden("dct.npz")
    tiles = [tuple(int(v) for v in t) for t in g["tiles"]]
    img = torch.from_numpy(g["recon"].copy()).cuda()
    out = raster.apply_dct(img, g[f"blob_{i}"].tobytes(), tiles).cpu().numpy()
    want = g[f"out_{i}"]
    assert float(np.max(np.abs(out - want))) <= APPLY_TOL
    assert float(out.min()) >= 0.0 and float(out.max()) <= 1.0


@pytest.mark.parametrize("j", range(len(RESIZE_TARGETS)))
def test_raster_resize_matches_pillow(golden, j):
    import torch

    from weft_b200 import raster

    g = golden("dct.npz")
    u8 = g[f"rs_in_{j}"]
    src = torch.from_numpy((u8.astype(np.float32) + np.float32(0.5)) / np.float32(255.0)).cuda()
    tw, th = RESIZE_TARGETS[j]
    # the kernels themselves, also for the unchanged-size case (identity taps; raster.resize skips it)
    out = torch.empty((th, tw, 3), dtype=torch.float32, device=src.device)
    tmp = torch.empty(u8.shape[0] * tw * 3, dtype=torch.uint8, device=src.device)
    raster.resize_into(src, out, tmp, torch.cuda.current_stream().cuda_stream)
    np.testing.assert_array_equal(out.cpu().numpy(), g[f"rs_out_{j}"].astype(np.float32) / np.float32(255.0))


@pytest.mark.parametrize("which", ["a", "b"])
def test_decode_file_raster_branch_matches_reference_decoder(golden, which):
    from weft_b200.encode import decode_file

    g = golden("container_dct.npz")
    blob = g[f"file_{which}"].tobytes()
    for key, size in (("native", (None, None)), ("up", (200, 150)), ("down", (50, 37))):
        got = decode_file(blob, *size)
        want = g[f"{key}_{which}"]
        assert got.shape == want.shape, key
        # primitive walk parity is 1/255; after u8 truncation a walk difference moves a value by at
        # most one step, and the resize keeps that bound
        assert float(np.max(np.abs(got - want))) <= 1.0 / 255.0 + 1e-6, key


@pytest.mark.parametrize("i", range(12))
def test_drop_in_apply_residual_to_image(golden, i):
    """The reference decoder's own steps (unpack, undo the band layout, decode the u8 scales) feeding
    the drop-in ``apply_residual_to_image``."""
    from oracle import dct as odct
    from weft_b200 import raster

    g = golden("dct.npz")
    tiles = [tuple(int(v) for v in t) for t in g["tiles"]]
    d = odct.unpack_dct(g[f"blob_{i}"].tobytes())
    coeffs = d["coeffs"]
    if d["layout"] == 1:
        pres = odct.presence(d["mask"], d["n_tiles"]) if (d["n_tiles"] and d["mask"]) else [True] * len(tiles)
        coeffs = odct.permute_band_to_tile(coeffs, [s for (_, _, s), p in zip(tiles, pres) if p], d["chroma_mode"])
    scales = [odct.tile_scale(u) for u in d["scales_u8"]] if d["scales_u8"] else None

    class QT:
        def __init__(self, x, y, size):
            self.x, self.y, self.size = x, y, size

    out = raster.apply_residual_to_image(g["recon"], coeffs, [QT(*t) for t in tiles], quant_step=d["quant_step"],
                                         channels=d["channels"], freq_alpha=d["freq_alpha"],
                                         chroma_mode=d["chroma_mode"], presence_bitmask=d["mask"],
                                         per_tile_scales=scales)
    assert out.dtype == np.float32
    assert float(np.max(np.abs(out - g[f"out_{i}"]))) <= APPLY_TOL
