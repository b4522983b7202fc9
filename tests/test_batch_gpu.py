"""Several images in one batched fit: tiles never interact, so the batch selects exactly what
separate per-image fits select, and every image keeps its own file and RD score."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _images():
    from weft_b200.batch import prepare_image
    from weft_b200.synth import make_image_u8

    specs = [(64, 64, 12, 5), (128, 128, 30, 6), (128, 64, 20, 7)]
    return [prepare_image(make_image_u8(w, h, n, seed), 75) for w, h, n, seed in specs]


def test_batched_fit_equals_per_image_fits():
    from weft_b200.batch import ImageBatch

    images = _images()
    batch = ImageBatch(images)
    fit = batch.plain_fit(autotune=False).run()
    got = fit.selected_indices()
    for i, im in enumerate(images):
        alone = ImageBatch([im]).plain_fit(autotune=False).run().selected_indices()
        assert got[batch.tile_off[i]:batch.tile_off[i + 1]] == alone


def test_refined_batch_reports_rd_per_image():
    from weft_b200.batch import ImageBatch

    batch = ImageBatch(_images())
    plain = batch.plain_fit()
    plain.run()
    ss, p = plain.stack_set()
    plain_rd = batch.rd_per_image(ss.to_stacks(ss.quantize(p)))
    rf = batch.refined_fit(steps=5)
    rows = rf.run()
    ref_rd = batch.rd_per_image(rf.ss.to_stacks(rf.ss.quantize(rows)))
    assert len(plain_rd) == len(ref_rd) == 3
    for a, b in zip(plain_rd, ref_rd):
        assert np.isfinite(a["rd_score"]) and np.isfinite(b["rd_score"])
        assert a["bytes"] > 0 and b["bytes"] > 0
