"""Device wire-grid quantisation (``weftk_quantize_rows``) against the torch restatement of the
reference's rule (``refine.quantize_rows``, pinned to reference outputs on the CPU): bit-equal on
random rows of every kind, including values outside the box and exact half-steps."""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_device_quantize_rows_bit_equal_to_reference_rule():
    from weft_b200 import _lib
    from weft_b200.refine import quantize_rows

    rng = np.random.default_rng(7)
    n = 4096
    rows = np.zeros((n, 16), np.float32)
    rows[:, 0:7] = rng.uniform(-2.0, 17.0, (n, 7))
    rows[:, 7:14] = rng.uniform(-0.2, 1.2, (n, 7))
    rows[:, 14:16] = rng.uniform(-1, 1, (n, 2))
    # exact half-steps of every grid
    rows[:64, 7] = (np.arange(64) + 0.5) / 255.0
    rows[64:128, 13] = (np.arange(64) + 0.5) / 65535.0
    rows[128:192, 0] = (np.arange(64) + 0.5) / 65535.0 * 15.0
    kinds = rng.integers(-1, 6, n).astype(np.int32)
    dev = torch.device("cuda", 0)
    lib = _lib.lib_for_device(0)
    t_rows, t_kind = torch.from_numpy(rows).to(dev), torch.from_numpy(kinds).to(dev)
    out = torch.empty_like(t_rows)
    _lib.check(lib.weftk_quantize_rows(_lib.ptr(t_rows), _lib.ptr(t_kind), n, _lib.ptr(out),
                                       torch.cuda.current_stream().cuda_stream), "weftk_quantize_rows")
    want = quantize_rows(torch.from_numpy(rows), torch.from_numpy(kinds)).numpy()
    got = out.cpu().numpy()
    np.testing.assert_array_equal(got[:, :14], want[:, :14])
    np.testing.assert_array_equal(got[:, 14:], rows[:, 14:])
