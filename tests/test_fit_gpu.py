"""GPU parity of the device-resident greedy fit.

The fit must pick the same candidates as the reference's greedy given the same
pools and re-seeds.  MSEs agree with the oracle to ~1e-7 relative, so a
different pick is only legitimate on an exact objective tie; the tests below
require identical selections.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import fit as ofit
from oracle import quadtree as oq
from oracle import rate as orate
from oracle.primitives import prims_from_pack
from tests.test_oracle_golden import _fit_inputs, _pack

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["fit_small.npz", "fit_hq.npz"])
def test_device_fit_matches_reference_greedy(golden, name):
    from weft_b200.fit import BatchedFit

    g = golden(name)
    tiles, patches, pools, reseeds = _fit_inputs(g)
    queue = {k: list(v) for k, v in reseeds.items()}
    fit = BatchedFit(patches, pools, int(g["quality"]))
    fit.run(reseed=lambda i, patch, pred: queue[i].pop(0))
    want = [[int(v) for v in row if v >= 0] for row in g["selected"]]
    assert fit.selected_indices() == want
    assert all(len(v) == 0 for v in queue.values())


def _oracle_objective(patch, prims, lam):
    return orate.tile_objective(patch, [ofit.as_f32(p) for p in prims], (0, 0, 0), lam)[0]


def test_device_fit_matches_oracle_on_all_tile_sizes():
    """8/16/32/64-px tiles (64 exercises the 4-block split) at q=92 for 2 rounds."""
    from weft_b200 import candidates, quadtree
    from weft_b200.fit import BatchedFit
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(128, 64, 3, 3)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    assert {q.size for q in qts} == {8, 16, 32, 64}
    patches = quadtree.extract_tiles(img, qts, 64)
    pools = [candidates.tile_candidates(p, 92) for p in patches]
    caps = [16] * len(qts)
    fixed = [candidates.residual_candidates(p, np.zeros_like(p), 92) for p in patches]
    fit = BatchedFit(patches, pools, 92, caps=caps)
    fit.run(reseed=lambda i, patch, pred: list(fixed[i]), max_rounds=2)
    sel, cur, _ = ofit.greedy_fit(patches, [q.size for q in qts], pools, 92,
                                  reseed=lambda i, patch, pred: list(fixed[i]), caps=caps, max_rounds=2)
    assert fit.selected_indices() == sel
    np.testing.assert_allclose(fit.objectives(), cur, rtol=1e-5)
    lam = orate.tile_lambda(92)
    for t, p in enumerate(patches):
        assert fit.objectives()[t] == pytest.approx(_oracle_objective(p, fit.selected()[t], lam), rel=1e-5)


def test_device_fit_is_deterministic():
    from weft_b200 import candidates, quadtree
    from weft_b200.fit import BatchedFit
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(96, 96, 12, 9)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="gradvar", threshold=0.08, min_tile=8, max_tile=32)
    patches = quadtree.extract_tiles(img, qts)
    pools = [candidates.tile_candidates(p, 90) for p in patches]
    a = BatchedFit(patches, pools, 90).run()
    b = BatchedFit(patches, pools, 90).run()
    assert a.selected_indices() == b.selected_indices()
    assert np.array_equal(a.objectives(), b.objectives())
    # the cached composite equals a full re-render of the selected stacks
    from weft_b200 import render

    for t in range(0, len(patches), 7):
        full = render.render_tile(a.selected()[t], int(qts[t].size))
        assert np.array_equal(full, a.recon_tiles()[t])


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_every_scoring_variant_matches_oracle(variant):
    """Each autotuner choice (kernel shape per size class, candidates per CTA) picks the same
    candidates as the oracle greedy on 8/16/32/64-px tiles."""
    from weft_b200 import candidates, quadtree
    from weft_b200.fit import BatchedFit
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(128, 64, 3, 3)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, qts, 64)
    pools = [candidates.tile_candidates(p, 92) for p in patches]
    caps = [16] * len(qts)
    fixed = [candidates.residual_candidates(p, np.zeros_like(p), 92) for p in patches]
    fit = BatchedFit(patches, pools, 92, caps=caps)
    chunk = (32, 64, 128)[variant]
    fit.configure(variants={8: variant, 16: variant, 32: variant}, chunks={8: chunk, 16: chunk, 32: chunk})
    fit.run(reseed=lambda i, patch, pred: list(fixed[i]), max_rounds=2)
    sel, cur, _ = ofit.greedy_fit(patches, [q.size for q in qts], pools, 92,
                                  reseed=lambda i, patch, pred: list(fixed[i]), caps=caps, max_rounds=2)
    assert fit.selected_indices() == sel
    np.testing.assert_allclose(fit.objectives(), cur, rtol=1e-5)


def test_autotune_keeps_the_reference_selection(golden):
    from weft_b200.fit import BatchedFit

    g = golden("fit_small.npz")
    tiles, patches, pools, reseeds = _fit_inputs(g)
    fit = BatchedFit(patches, pools, int(g["quality"]))
    tuned = fit.autotune(reps=1)
    assert tuned and all(0 <= v < 3 and c in (32, 64, 128) and ms >= 0 for v, c, ms in tuned.values())
    queue = {k: list(v) for k, v in reseeds.items()}
    fit.run(reseed=lambda i, patch, pred: queue[i].pop(0))
    assert fit.selected_indices() == [[int(v) for v in row if v >= 0] for row in g["selected"]]


def test_device_driven_fit_equals_host_loop_and_replays():
    """The whole fit enqueued without host synchronisation (and replayed from a CUDA graph)
    takes the host loop's decisions: same selections and objectives as run() with device
    re-seeding, on 8/16/32/64-px tiles at q=92 (re-seeds happen)."""
    from weft_b200 import candidates, quadtree
    from weft_b200.fit import BatchedFit
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(128, 64, 3, 3)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, qts, 64)
    pools = [candidates.tile_candidates(p, 92) for p in patches]
    fit = BatchedFit(patches, pools, 92, caps=[16] * len(qts))
    fit.run()
    want_sel, want_obj, want_rounds = fit.selected_indices(), fit.objectives(), fit.stats.rounds
    assert fit.stats.reseeds > 0
    fit.reset()
    fit.run_device()
    assert fit.selected_indices() == want_sel
    np.testing.assert_array_equal(fit.objectives(), want_obj)
    assert fit.control()["rounds"] == want_rounds
    g = fit.graph()
    for _ in range(2):
        g.replay()
        assert fit.selected_indices() == want_sel
        np.testing.assert_array_equal(fit.objectives(), want_obj)


def test_closed_form_init_matches_per_pixel_objectives():
    """Init-round objectives with constant candidates scored from tile moments agree with the
    per-pixel scores to float rounding; selections agree except on near ties."""
    from weft_b200 import candidates, quadtree
    from weft_b200.fit import BatchedFit
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(128, 64, 3, 3)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, qts, 64)
    pools = [[c for c in candidates.tile_candidates(p, 75) if c.kind in (0, 1)] for p in patches]
    fit = BatchedFit(patches, pools, 75, caps=[16] * len(qts))
    fit.run(max_rounds=0)
    want_sel, want_obj = fit.selected_indices(), fit.objectives()
    fit.use_closed_form_init(True)
    fit.reset()
    fit.run(max_rounds=0)
    np.testing.assert_allclose(fit.objectives(), want_obj, rtol=1e-5)
    same = sum(a == b for a, b in zip(fit.selected_indices(), want_sel))
    assert same >= 0.95 * len(want_sel)


def test_queue_driven_rounds_equal_per_item_launches():
    """Persistent scoring launches that pull the round's live items from a queue give the same
    fit as one CTA per item: selections, objectives and round decisions, host loop and graph."""
    from weft_b200 import candidates, quadtree
    from weft_b200.fit import BatchedFit
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(128, 64, 3, 3)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, qts, 64)
    pools = [candidates.tile_candidates(p, 92) for p in patches]
    a = BatchedFit(patches, pools, 92, caps=[16] * len(qts)).use_queue(False)
    b = BatchedFit(patches, pools, 92, caps=[16] * len(qts))
    a.run()
    b.run()
    assert a.stats.reseeds > 0
    assert a.selected_indices() == b.selected_indices()
    np.testing.assert_array_equal(a.objectives(), b.objectives())
    assert a.stats.per_round == b.stats.per_round
    b.reset()
    g = b.graph()
    g.replay()
    assert b.selected_indices() == a.selected_indices()
    np.testing.assert_array_equal(b.objectives(), a.objectives())


def test_init_only_fit_skips_the_composite_and_refuses_rounds():
    """A fit declared init-only (the refined fit) leaves the composite untouched, picks what the
    full fit's init round picks, and refuses a greedy round, which would need the composite."""
    from weft_b200 import candidates, quadtree
    from weft_b200._lib import WeftkError
    from weft_b200.fit import BatchedFit
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(128, 64, 3, 3)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, qts, 64)
    pools = [[c for c in candidates.tile_candidates(p, 75) if c.kind in (0, 1)] for p in patches]
    full = BatchedFit(patches, pools, 75, caps=[16] * len(qts)).use_closed_form_init(True)
    full.run_init_only()
    lean = BatchedFit(patches, pools, 75, caps=[16] * len(qts)).use_closed_form_init(True).init_only()
    lean.t_bg.fill_(0.25)
    lean.run_init_only()
    assert lean.selected_indices() == full.selected_indices()
    np.testing.assert_array_equal(lean.objectives(), full.objectives())
    assert bool((lean.t_bg == 0.25).all())
    with pytest.raises(WeftkError):
        lean.run(max_rounds=1)
