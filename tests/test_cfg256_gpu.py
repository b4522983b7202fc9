"""The plain-method workload end to end on the GPU, against the reference's own encode.

256x256 synthetic image (40 primitives, seed 0), q=75, fixed 32-px tiles, at most 8
primitives per tile, primitive-stack basis only, decoded at native size.  The fixture was
made by the reference's ``encode_image`` (its greedy ``_fit_adaptive_state``,
src/weft/encoder.py:2520-2898, with the candidate pools and re-seeds recorded) and its
``decode_to_array``.  The device fit must pick the same candidates; its file must carry the
same primitive, residual and quadtree payloads as the reference's; the GPU decoder must read
the reference's file within 1/255.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import fit as ofit
from oracle import rate as orate
from tests.test_oracle_golden import _fit_inputs

pytestmark = pytest.mark.gpu

CAP = 8


def _device_fit(g):
    from weft_b200.fit import BatchedFit

    tiles, patches, pools, reseeds = _fit_inputs(g)
    queue = {k: list(v) for k, v in reseeds.items()}
    fit = BatchedFit(patches, pools, int(g["quality"]), caps=[CAP] * len(tiles))
    fit.run(reseed=lambda i, patch, pred: queue[i].pop(0))
    assert all(len(v) == 0 for v in queue.values())
    return tiles, patches, fit


def test_device_fit_matches_reference_selection_256(golden):
    g = golden("fit_cfg256.npz")
    tiles, patches, fit = _device_fit(g)
    assert fit.selected_indices() == [[int(v) for v in row if v >= 0] for row in g["selected"]]
    lam = orate.tile_lambda(int(g["quality"]))
    for t in range(len(tiles)):
        want = orate.tile_objective(patches[t], [ofit.as_f32(p) for p in fit.selected()[t]], (0, 0, 0), lam)[0]
        assert fit.objectives()[t] == pytest.approx(want, rel=1e-5)


def test_encode_of_device_fit_matches_reference_file_256(golden):
    from weft_b200 import bitstream
    from weft_b200.encode import encode_fit

    g = golden("fit_cfg256.npz")
    tiles, patches, fit = _device_fit(g)
    blob = encode_fit(256, 256, 75, tiles, patches, fit.selected(), fit.recon_tiles())
    ours, ref = bitstream.decode_weft(blob), bitstream.decode_weft(g["weft_file"].tobytes())
    assert ours.prim_raw == ref.prim_raw
    assert list(ours.toc) == list(ref.toc)
    assert [tuple(r) for r in ours.residuals] == [tuple(r) for r in ref.residuals]
    assert all(np.array_equal(a, b) for a, b in zip(ours.res1_maps, ref.res1_maps))
    assert [tuple(q) for q in ours.qtree] == [tuple(q) for q in ref.qtree]


def test_gpu_decode_of_reference_file_256(golden):
    from weft_b200.encode import decode_file

    g = golden("fit_cfg256.npz")
    img = decode_file(g["weft_file"].tobytes())
    assert img.shape == (256, 256, 3)
    assert float(np.max(np.abs(img - g["decoded"]))) <= 1.0 / 255.0


def test_quantized_selection_256(golden):
    """The device snap of the selected stacks equals the reference's quantisation rule
    (``refine.quantize_rows``) applied to the selected records."""
    import torch

    from weft_b200.refine import quantize_rows, records_to_rows

    g = golden("fit_cfg256.npz")
    _, _, fit = _device_fit(g)
    fit.quantize_selected()
    got = fit.quantized_stacks()
    for t, recs in enumerate(fit.selected_records()):
        want = quantize_rows(torch.from_numpy(records_to_rows(recs)), torch.from_numpy(recs["kind"].astype(np.int32)))
        assert np.array_equal(records_to_rows(got[t]), want.numpy())
        assert np.array_equal(got[t]["kind"], recs["kind"])
