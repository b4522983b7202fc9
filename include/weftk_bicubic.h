/*
 * weftk_bicubic.h — the per-tile bicubic R-D swap of the adaptive fit on the GPU (C ABI of
 * libweftk.so).
 *
 * Replaces the loop at the end of _fit_adaptive_state (src/weft/encoder.py:2841-2873) that
 * builds bicubic_replaced_per_tile: for every tile, the least-squares 4x4x3 Bezier control grid
 * (bicubic.fit_tile, src/weft/bicubic.py:65-86: pinv(B) @ tile @ pinv(B^T) per channel in
 * float64, rounded to float32, clipped to [0, 1]), rounded to u8 steps
 * (round(clip(grid) * 255) / 255 in float32, half to even), evaluated (bicubic.eval_tile,
 * src/weft/bicubic.py:106-115) and scored as mse + lam * 408 against the selected stack's
 * mse + lam * (8 + 8 * sum of its primitives' byte sizes); the tile is marked for replacement
 * when the bicubic score is lower.  Both MSEs are float32 squared errors summed in float64.
 */
#ifndef WEFTK_BICUBIC_H
#define WEFTK_BICUBIC_H

#include "weftk.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Bits of a tile replaced by one bicubic primitive: count, kind and length bytes + 48 control
 * bytes (src/weft/encoder.py:2844-2846). */
#define WEFTK_BICUBIC_BITS 408

/* Doubles of the basis table: for each tile side n of 8, 16, 32, 64 in that order, pinv(B)
 * (4 x n), pinv(B^T) (n x 4) and B (n x 4), each row-major, where B is the cubic Bernstein
 * basis at numpy.linspace(0, 1, n) (src/weft/bicubic.py:31-57; the reference takes both
 * pseudo-inverses from numpy.linalg.pinv).  The side-n block starts at 12 * (n - 8) doubles. */
#define WEFTK_BICUBIC_BASIS_DOUBLES 1440

/*
 *   d_pixels    float4 (r, g, b, -) per pixel, tile t's side x side pixels row-major from
 *               d_px_off[t]
 *   d_size      int32 [n_tiles] tile side: 8, 16, 32 or 64
 *   d_prims     the selected stacks, n_prims WeftPrim records; tile t's are
 *               [d_prim_off[t], d_prim_off[t + 1])
 *   d_basis     WEFTK_BICUBIC_BASIS_DOUBLES doubles (above)
 *   lam         the fit's lambda (encoder._tile_lambda)
 * Outputs:
 *   d_grid      float [n_tiles * 48]: the u8-rounded control grid, (4, 4, 3) row-major
 *   d_swap      int32 [n_tiles]: 1 where the bicubic primitive scores lower, else 0
 *   d_score     double [n_tiles * 2]: (bicubic score, stack score)
 * A tile of another side, a stack longer than 48 primitives or a record range outside
 * [0, n_prims) is reported through weftk_device_status (WEFTK_E_ARG) and left unwritten.
 * Asynchronous on `stream`.
 */
int weftk_bicubic_swap(const float* d_pixels, const int32_t* d_px_off, const int32_t* d_size, int n_tiles,
                       const WeftPrim* d_prims, int n_prims, const int32_t* d_prim_off, const double* d_basis, double lam,
                       float* d_grid, int32_t* d_swap, double* d_score, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WEFTK_BICUBIC_H */
