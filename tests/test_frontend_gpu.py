"""The fit's front end on the device against the host restatement of the reference's: the
variance-rule quadtree (the same tiles in the same order), tile extraction with the sRGB decode
(bit-equal pixels, edge padding included), and the whole refined fit from the u8 image."""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,h,n,seed", [(256, 256, 40, 0), (200, 130, 25, 3), (1024, 1024, 600, 0), (72, 264, 9, 5)])
def test_device_quadtree_and_extraction_equal_host(w, h, n, seed):
    from weft_b200 import frontend, quadtree
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(w, h, n, seed)
    img = srgb_u8_to_linear(u8)
    want = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    dimg = torch.from_numpy(u8).to("cuda:0")
    tiles, count = frontend.decompose_device(dimg, 100.0)
    got = tiles.cpu().numpy()
    assert count == len(want)
    assert [tuple(int(v) for v in r) for r in got] == [(t.x, t.y, t.size) for t in want]
    sizes = got[:, 2].copy()
    src4, _ = frontend.extract_device(dimg, tiles, sizes)
    host = np.concatenate([p.reshape(-1, 3) for p in quadtree.extract_tiles(img, want, 64)])
    np.testing.assert_array_equal(src4[:, :3].cpu().numpy(), host)
    assert float(src4[:, 3].abs().max()) == 0.0


def test_refine_image_equals_the_fit_over_host_tiles():
    from weft_b200 import frontend, quadtree
    from weft_b200.pools import refine_tiles
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(192, 160, 20, 7)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, qts, 64)
    sizes = np.array([p.shape[0] for p in patches], np.int32)
    rows_h, kinds_h = refine_tiles(np.concatenate([p.reshape(-1, 3) for p in patches]), sizes, 75,
                                   caps=[16] * len(sizes), steps=5)
    tiles, rows, kinds = frontend.refine_image(u8, 75, 16, steps=5)
    assert [tuple(r) for r in tiles.tolist()] == [(t.x, t.y, t.size) for t in qts]
    np.testing.assert_array_equal(rows, rows_h)
    np.testing.assert_array_equal(kinds, kinds_h)


def test_refine_image_steps_releases_its_device_memory_at_return():
    """No reference cycle holds the fit's buffers after the call (the caching allocator gets
    them back at once, with the cycle collector off)."""
    import gc

    from weft_b200 import frontend
    from weft_b200.synth import make_image_u8

    u8 = make_image_u8(256, 256, 30, 2)
    frontend.refine_image_steps(u8, 75, 16, steps=3)  # tables, lookup tables, streams
    torch.cuda.synchronize()
    gc.collect()
    base = torch.cuda.memory_allocated()
    gc.disable()
    try:
        for _ in range(3):
            frontend.refine_image_steps(u8, 75, 16, steps=3)
        torch.cuda.synchronize()
        assert torch.cuda.memory_allocated() == base
    finally:
        gc.enable()


def test_native_pipeline_equals_the_stepwise_calls_across_image_sizes():
    """``weftk_refine_image`` (one native call, a workspace kept and grown between images) against
    the same steps driven one entry point at a time: equal tiles, rows and kinds, bit for bit, on
    a sequence of images whose sizes grow and shrink."""
    from weft_b200 import frontend
    from weft_b200.synth import make_image_u8

    r = frontend.Refiner(75, 16, steps=5)
    for w, h, n, seed in [(256, 256, 30, 1), (520, 392, 70, 2), (72, 264, 9, 5), (256, 256, 30, 1), (130, 200, 20, 3)]:
        u8 = make_image_u8(w, h, n, seed)
        tiles, rows, kinds = r(u8)
        t2, r2, k2 = frontend.refine_image_steps(u8, 75, 16, steps=5)
        np.testing.assert_array_equal(tiles, t2)
        np.testing.assert_array_equal(kinds, k2)
        np.testing.assert_array_equal(rows, r2)
        assert (kinds >= 0).all()
    r.close()


def test_native_pipeline_reports_too_many_tiles():
    import ctypes

    from weft_b200 import frontend
    from weft_b200.synth import make_image_u8

    r = frontend.Refiner(75, 16, steps=2)
    u8 = make_image_u8(128, 128, 30, 4)
    tiles = np.empty((1, 3), np.int32)
    rows = np.empty((1, 16), np.float32)
    kinds = np.empty(1, np.int32)
    n = ctypes.c_int(0)
    rc = r.lib.weftk_refine_image(r.handle, u8.ctypes.data, 128, 128, tiles.ctypes.data, rows.ctypes.data,
                                  kinds.ctypes.data, 1, ctypes.addressof(n), torch.cuda.current_stream().cuda_stream)
    assert rc == -3  # WEFTK_E_RANGE: more tiles than max_tiles, the count reported
    assert n.value > 1
    r.close()
