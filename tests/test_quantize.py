"""Wire-grid quantisation of parameter rows (CPU): ``refine.quantize_rows`` against the
reference's ``_quantize_primitive`` outputs (src/weft/encoder.py:211-237) in the golden
fixture, every primitive kind 0-4 (bicubic rows carry their control grid outside the row)."""

from __future__ import annotations

import numpy as np
import torch

from tests.test_oracle_golden import _pack


def test_quantize_rows_matches_reference_golden(golden):
    from weft_b200.refine import quantize_rows

    g = golden("quant.npz")
    a, q = _pack(g, "in_"), _pack(g, "q_")
    keep = a["kind"] != 5
    n = int(keep.sum())
    assert n > 80
    rows = np.zeros((n, 16), np.float32)
    rows[:, 0:7] = a["geom"][keep, :7]
    rows[:, 7:10] = a["c0"][keep]
    rows[:, 10:13] = a["c1"][keep]
    rows[:, 13] = a["alpha"][keep]
    kinds = torch.from_numpy(a["kind"][keep].astype(np.int32))
    got = quantize_rows(torch.from_numpy(rows), kinds).numpy()
    want = np.zeros((n, 16), np.float32)
    want[:, 0:7] = q["geom"][keep, :7]
    want[:, 7:10] = q["c0"][keep]
    want[:, 10:13] = q["c1"][keep]
    want[:, 13] = q["alpha"][keep]
    np.testing.assert_array_equal(got, want)


def test_quantize_rows_edges():
    """Half-way values round to even; values outside the box clamp; rows without a layer keep
    their geometry."""
    from weft_b200.refine import quantize_rows

    rows = torch.zeros((4, 16), dtype=torch.float32)
    rows[0, 7] = 0.5 / 255.0 * 3.0  # 1.5 steps -> 2 (even)
    rows[0, 8] = 2.5 / 255.0        # 2.5 steps -> 2 (even)
    rows[0, 9] = -0.25
    rows[0, 13] = 1.75
    rows[1, 0:4] = torch.tensor([-1.0, 16.0, 7.5, 15.0])
    rows[2, 4] = 9.0                 # line thickness clamps to 4
    rows[3, 0:7] = 3.3               # kind -1: untouched geometry
    kinds = torch.tensor([0, 1, 2, -1], dtype=torch.int32)
    out = quantize_rows(rows, kinds).numpy()
    r = np.float64(rows[0, 7]) * 255.0
    assert out[0, 7] == np.float32(round(r) / 255.0)
    assert out[0, 8] == np.float32(round(np.float64(np.float32(2.5 / 255.0)) * 255.0) / 255.0)
    assert out[0, 9] == 0.0 and out[0, 13] == 1.0
    assert out[1, 0] == 0.0 and out[1, 1] == 15.0 and out[1, 3] == 15.0
    assert out[2, 4] == 4.0
    np.testing.assert_array_equal(out[3, 0:7], np.float32(3.3))
