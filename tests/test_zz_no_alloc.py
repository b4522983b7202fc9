"""weftk_fit_round_static: the fit round for callers that cannot allocate device memory.

Some callers must not call cudaMalloc while they run (hosts that give the library
a fixed device budget, services that cannot afford cudaMalloc's implicit device
synchronisation).  The static entry point keeps its scoring scratch in a fixed
device array instead.  It must give the same results as weftk_fit_round, call
after call.  This file is collected last on purpose.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

OBJ_RTOL = 1e-5  # the fit tests' tolerance on objectives


def _fit_pair():
    from weft_b200 import candidates, quadtree
    from weft_b200.fit import BatchedFit
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(128, 64, 3, 3)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, qts, 64)
    pools = [candidates.tile_candidates(p, 92) for p in patches]
    return BatchedFit(patches, pools, 92, caps=[16] * len(qts)), BatchedFit(patches, pools, 92, caps=[16] * len(qts))


def _call(fit, fn, mode):
    lib = fit.lib
    ti = fit.t_items
    from weft_b200 import _lib

    rc = getattr(lib, fn)(ctypes.addressof(fit.st), mode, fit.lam, fit.thr, _lib.ptr(fit.t_perm), _lib.ptr(ti[8]),
                          fit.n_items[8], _lib.ptr(ti[16]), fit.n_items[16], _lib.ptr(ti[32]), fit.n_items[32],
                          torch.cuda.current_stream().cuda_stream)
    _lib.check(rc, fn)
    torch.cuda.synchronize()


def test_static_round_matches_allocating_round_twice_in_a_row():
    ref, stat = _fit_pair()
    stat.st.partial = None  # the static entry point must not touch the caller's scratch pointer
    assert stat.n_slots * 4 <= 4 * 1024 * 1024
    for mode in (0, 1):  # init, then one greedy round: two calls in a row
        _call(ref, "weftk_fit_round", mode)
        _call(stat, "weftk_fit_round_static", mode)
        assert torch.equal(ref.t_status, stat.t_status)
        assert ref.selected_indices() == stat.selected_indices()
        np.testing.assert_allclose(stat.objectives(), ref.objectives(), rtol=OBJ_RTOL)
        assert torch.equal(ref.t_bg, stat.t_bg)


def test_static_round_rejects_oversized_fit_without_launching():
    from weft_b200 import _lib

    ref, _ = _fit_pair()
    big = _lib.WeftFitState.from_buffer_copy(ref.st)
    big.n_slots = 4 * 1024 * 1024  # 4x the slots the static scratch can hold
    rc = ref.lib.weftk_fit_round_static(ctypes.addressof(big), 1, ref.lam, ref.thr, _lib.ptr(ref.t_perm), 0, 0, 0, 0,
                                        0, 0, torch.cuda.current_stream().cuda_stream)
    assert rc == -3 and "static scratch" in _lib.last_error()
