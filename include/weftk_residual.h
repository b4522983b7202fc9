/*
 * weftk_residual.h — per-tile residual build on the GPU (C ABI of libweftk.so).
 *
 * The encoder's build phase for the primitive-stack basis (src/weft/encoder.py:2986-3005,
 * :3248-3372): RES0 = the tile's mean error of the fitted render, x255, rounded half-to-even,
 * clipped to +-127; RES1 = the 4x4 grid of block means of the error left after RES0 (render +
 * RES0/255 clipped to [0, 1]), x255, rounded half-to-even, clipped to +-127.  The arithmetic
 * follows numpy's float32 evaluation of that code, including its summation order (sequential
 * over the pixels in row-major order for each output value), so the bytes are identical to the
 * host build's.
 */
#ifndef WEFTK_RESIDUAL_H
#define WEFTK_RESIDUAL_H

#include "weftk.h"

#ifdef __cplusplus
extern "C" {
#endif

/* d_src, d_recon: float4 (r, g, b, -) per pixel, tiles back to back (d_px_off), row-major inside
 * a tile of side d_size[t] (a multiple of 4, at most 64); clamp_recon != 0 clips the recon to
 * [0, 1] first (pass the fit's raw composite).  Outputs: d_res0 int8[n_tiles * 3], d_res1
 * int8[n_tiles * 48] as (4, 4, 3) row-major.  A tile of unsupported side is reported through
 * weftk_device_status (WEFTK_E_ARG) and left unwritten. */
int weftk_build_residuals(const float* d_src, const float* d_recon, int clamp_recon, const int32_t* d_px_off,
                          const int32_t* d_size, int n_tiles, int8_t* d_res0, int8_t* d_res1, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WEFTK_RESIDUAL_H */
