"""The fused refine path (one loss+gradient launch and one Adam+projection launch per
step) against the autograd + torch.optim.Adam path, and the graph-captured refined fit
against the same work launched eagerly.

Workload: a 256x256 synthetic image (40 primitives, seed 0), quadtree 8-64 px on u8
luminance variance > 100, q=75 candidate pools.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _fit(kinds_out=()):
    from weft_b200 import candidates, quadtree
    from weft_b200.fit import BatchedFit
    from weft_b200.synth import make_image_u8, srgb_u8_to_linear

    u8 = make_image_u8(256, 256, 40, 0)
    img = srgb_u8_to_linear(u8)
    qts = quadtree.decompose(img, rule="variance", threshold=100.0, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, qts, 64)
    pools = [[c for c in candidates.tile_candidates(p, 75) if c.kind not in kinds_out] for p in patches]
    return BatchedFit(patches, pools, 75, caps=[16] * len(qts))


@pytest.mark.parametrize("residual", [False, True])
def test_backward_loss_output_equals_forward(residual):
    from weft_b200.refine import FusedRefiner

    fit = _fit().run()
    ss, params = fit.stack_set()
    fr = FusedRefiner(ss, params, residual=residual)
    want = ss.loss(fr.p, residual=residual).cpu().numpy()
    fr.step()
    got = fr.loss.cpu().numpy()
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-9)


@pytest.mark.parametrize("residual", [False, True])
def test_fused_refiner_matches_torch_adam(residual):
    from weft_b200.refine import FusedRefiner, refine

    fit = _fit().run()
    ss, params = fit.stack_set()
    steps = 15
    want, hist = refine(ss, params, steps=steps, lr=1e-2, residual=residual)
    fr = FusedRefiner(ss, params, lr=1e-2, residual=residual)
    losses = []
    for _ in range(steps):
        fr.step()
        losses.append(float((fr.loss * ss.weights).sum()))
    got = fr.p
    # Same update rule; the bias corrections are computed in float32 on the device
    # versus double on the host, so trajectories agree to rounding, not bit for bit.
    assert float((got[:, :14] - want[:, :14]).abs().max()) < 2e-3
    np.testing.assert_allclose(losses, hist, rtol=1e-4)
    assert float(fr.m[:, 15].min()) == steps and float(fr.m[:, 15].max()) == steps  # per-row step counts


@pytest.mark.parametrize("use_graph,residual", [(False, False), (True, False), (True, True)])
def test_refined_fit_matches_unfused_pipeline(use_graph, residual):
    from weft_b200.refine import FusedRefiner, RefinedFit

    fit = _fit(kinds_out=(3,))
    rf = RefinedFit(fit, steps=10, lr=1e-2, use_graph=use_graph, residual=residual)
    got = rf.run().clone()
    got2 = rf.run().clone()  # replays start from the same state
    assert torch.equal(got, got2)

    fit.reset()
    fit.run(max_rounds=0)
    ss, params = fit.stack_set()
    assert np.array_equal(ss.prim_off_np, rf.ss.prim_off_np)
    assert torch.equal(ss.t_kind, rf.kinds)
    ss.st.kinds_mask = rf.ss.st.kinds_mask  # same kernel choice as the refined fit (the pool's kinds)
    fr = FusedRefiner(ss, params, lr=1e-2, residual=residual)
    fr.run(10)
    assert torch.equal(fr.p[:, :14], got[:, :14])


@pytest.mark.parametrize("residual", [False, True])
def test_single_launch_step_equals_two_launch_step(residual):
    from weft_b200.refine import FusedRefiner

    fit = _fit().run()
    ss, params = fit.stack_set()
    one = FusedRefiner(ss, params, lr=1e-2, residual=residual, single_launch=True)
    two = FusedRefiner(ss, params, lr=1e-2, residual=residual, single_launch=False)
    for _ in range(8):
        one.step()
        two.step()
        assert torch.equal(one.loss, two.loss)
    assert torch.equal(one.p[:, :14], two.p[:, :14])
    assert torch.equal(one.m[:, :14], two.m[:, :14]) and torch.equal(one.v[:, :14], two.v[:, :14])
    assert float(one.m[:, 15].min()) == 8.0 and float(one.m[:, 15].max()) == 8.0


@pytest.mark.parametrize("residual", [False, True])
def test_single_layer_register_path_matches_general_path(residual):
    """Stacks of one constant/linear layer take the register-only kernel (declared kinds mask
    {0, 1}); the general kernel (mask undeclared) must give the same loss and gradient."""
    from weft_b200.refine import FusedRefiner, RefinedFit, StackSet

    fit = _fit(kinds_out=(2, 3, 4, 5))
    rf = RefinedFit(fit, steps=0, use_graph=False)
    rf.run()
    assert rf.ss.st.kinds_mask in (1, 2, 3)
    gen = StackSet(rf.ss.src, rf.ss.px_off, rf.ss.sizes, rf.ss.prim_off_np, rf.kinds, kinds_mask=0)
    p = rf.start.clone()
    w = rf.ss.weights
    for a, b in ((rf.ss.loss(p, residual=residual), gen.loss(p, residual=residual)),
                 (rf.ss.loss_backward(p, w, residual=residual), gen.loss_backward(p, w, residual=residual))):
        scale = float(b.abs().max()) + 1e-30
        assert float((a - b).abs().max()) <= 1e-4 * scale
    # Adam normalises each gradient component, so components that are zero up to rounding
    # (summed in another order by the two kernels) may step differently; the objective may not.
    one = FusedRefiner(rf.ss, p, residual=residual)
    two = FusedRefiner(gen, p, residual=residual)
    for _ in range(10):
        one.step()
        two.step()
        l1, l2 = float((one.loss * w).sum()), float((two.loss * w).sum())
        assert l1 == pytest.approx(l2, rel=1e-4)


@pytest.mark.parametrize("residual", [False, True])
def test_multi_step_launch_equals_single_steps(residual):
    """weftk_refine_steps (all steps in one launch) = the same number of one-step launches."""
    from weft_b200.refine import FusedRefiner

    fit = _fit().run()
    ss, params = fit.stack_set()
    one = FusedRefiner(ss, params, lr=1e-2, residual=residual)
    many = FusedRefiner(ss, params, lr=1e-2, residual=residual)
    for _ in range(7):
        one.step()
    many.run(7)
    assert torch.equal(one.p[:, :14], many.p[:, :14])
    assert torch.equal(one.m[:, :14], many.m[:, :14]) and torch.equal(one.v[:, :14], many.v[:, :14])
    assert torch.equal(one.m[:, 15], many.m[:, 15])
    assert torch.equal(one.loss, many.loss)
