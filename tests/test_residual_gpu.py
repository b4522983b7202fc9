"""GPU RES0/RES1 build: byte-identical to the host build (numpy float32, the reference's
build phase) on a fitted image and on random tiles of every side."""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_fit_residuals_identical_to_host_build():
    from weft_b200 import candidates, quadtree
    from weft_b200.encode import residuals_from_fit_gpu, residuals_from_recon
    from weft_b200.fit import BatchedFit
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(256, 256, 40, 2)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, qts, 64)
    pools = [candidates.tile_candidates(p, 75) for p in patches]
    fit = BatchedFit(patches, pools, 75, caps=[16] * len(qts)).run()
    want0, want1 = residuals_from_recon(patches, fit.recon_tiles())
    got0, got1 = residuals_from_fit_gpu(fit)
    assert got0 == want0
    assert all(np.array_equal(a, b) for a, b in zip(got1, want1))


@pytest.mark.parametrize("ts", [8, 16, 32, 64])
def test_random_tiles_identical_to_host_build(ts):
    from weft_b200 import _lib
    from weft_b200.encode import residuals_from_recon

    rng = np.random.default_rng(ts)
    n = 50
    patches = [rng.random((ts, ts, 3), dtype=np.float32) for _ in range(n)]
    # composites outside [0, 1] too (the kernel clips, as the host build's input is clipped)
    comps = [(rng.random((ts, ts, 3), dtype=np.float32) * np.float32(1.4) - np.float32(0.2)) for _ in range(n)]
    want0, want1 = residuals_from_recon(patches, [np.clip(c, 0.0, 1.0) for c in comps])
    d = torch.device("cuda", 0)
    lib = _lib.lib_for_device(0)

    def f4(arrs):
        a = np.zeros((n * ts * ts, 4), np.float32)
        a[:, :3] = np.concatenate([x.reshape(-1, 3) for x in arrs])
        return torch.from_numpy(a).to(d)

    src, rec = f4(patches), f4(comps)
    px_off = torch.arange(n, dtype=torch.int32, device=d) * (ts * ts)
    size = torch.full((n,), ts, dtype=torch.int32, device=d)
    r0 = torch.zeros((n, 3), dtype=torch.int8, device=d)
    r1 = torch.zeros((n, 4, 4, 3), dtype=torch.int8, device=d)
    _lib.check(lib.weftk_build_residuals(_lib.ptr(src), _lib.ptr(rec), 1, _lib.ptr(px_off), _lib.ptr(size), n,
                                         _lib.ptr(r0), _lib.ptr(r1), torch.cuda.current_stream().cuda_stream),
               "weftk_build_residuals")
    assert [tuple(int(v) for v in row) for row in r0.cpu().numpy()] == want0
    assert np.array_equal(r1.cpu().numpy(), np.stack(want1))
