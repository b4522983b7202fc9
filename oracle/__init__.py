"""CPU oracle for the primitive-stack hot path — TEST INFRASTRUCTURE ONLY.

This package restates, in plain numpy, the reference's CPU algorithms for the
path the CUDA library implements: the per-tile renderer, the per-tile
objective and rate model, the greedy candidate-scoring fit, the decoder's
scene walk and its raster branch (DCT residual layer, Pillow-compatible
BILINEAR resize), primitive quantization/serialization, the quadtree and the
order-0 rANS coder.  Every function cites the reference file:line it follows.

Parity is pinned: ``tests/test_oracle_golden.py`` and ``tests/test_dct_cpu.py`` check every function here
against golden vectors produced by running the reference itself
(``tests/golden/make_golden.py``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker or the timed CPU
baseline.  The product (``weft_b200``) never imports it and has no CPU
fallback.
"""
