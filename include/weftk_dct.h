/*
 * weftk_dct.h — the decoder's raster branch on the GPU (C ABI of libweftk.so): the per-tile
 * DCT residual layer added on top of the primitive walk, and the u8 BILINEAR resize that
 * follows it when the target size differs from the encoded size.
 *
 * Replaces, with the same arithmetic:
 *   - apply_residual_to_image (src/weft/dct_residual.py:727-783) with decode_tile_residuals
 *     (:550-701), _batch_dequant_idct (:513-547) and permute_band_to_tile (:221-296) folded
 *     into one gather + dequantize + inverse DCT + colour transform + add + clip per tile;
 *   - the raster upscale of the decoder (src/weft/decoder.py:514-518): float -> u8 by
 *     truncation of clip(x * 255), Pillow Image.resize(BILINEAR) (22-bit fixed-point
 *     triangle filter, horizontal pass into an 8-bit intermediate, then vertical pass), / 255.
 */
#ifndef WEFTK_DCT_H
#define WEFTK_DCT_H

#include "weftk.h"

#ifdef __cplusplus
extern "C" {
#endif

#define WEFTK_DCT_MAX_TILE 64 /* largest tile side (Y block); chroma blocks go down to 2 */

/* One tile that carries DCT coefficients: 64 bytes.  Channel c's block is n x n with n = size,
 * or size / 2 for the Cb / Cr blocks of 4:2:0 (chroma_mode 2).  The quantized coefficient of
 * row-major position k (row u = k / n, column v = k % n) is
 *     coeffs[coef_base[c] + k * coef_stride[c]]               (tile-major layout 0)
 *     coeffs[coef_base[c] + zigzag_pos(n, k) * coef_stride[c]] (band-major layout 1)
 * where zigzag_pos is the position of k in the JPEG zigzag scan of an n x n block
 * (src/weft/dct_residual.py:91-123); for layout 1, coef_base = band start + the tile's rank
 * among the band's members and coef_stride = the band's member count. */
typedef struct WeftDctTile {
    int32_t x, y;          /* tile origin in the image, pixels */
    int32_t size;          /* tile side: 4, 8, 16, 32 or 64 */
    int32_t _pad;
    double step_scale;     /* per-tile quant-step factor (decoded u8 scale; 1.0 = uniform) */
    int64_t coef_base[3];
    int32_t coef_stride[3];
    int32_t _pad2;
} WeftDctTile;

/*
 * Add the dequantized inverse-DCT residual of every tile to d_image (height x width x 3 float32,
 * HWC) and clip the touched pixels to [0, 1]; pixels past the image edge are dropped.  Tiles
 * must not overlap (quadtree tiles never do): each tile's pixels are written by one CTA.
 *   chroma_mode  0 RGB, 1 YCbCr 4:4:4, 2 YCbCr 4:2:0 (BT.601 residual matrices; chroma step
 *                quant_step * 1.5; 4:2:0 chroma upsampled by pixel repetition)
 *   band_layout  0 tile-major, 1 band-major zigzag (see WeftDctTile)
 *   freq_alpha   > 0: coefficient (u, v) of an n x n block uses step * (1 + alpha (u + v) / (2 (n - 1)))
 *   max_size     largest d_tiles[i].size in this launch (sizes the shared-memory staging)
 *   clip_all     != 0: afterwards clip every pixel of the image to [0, 1], as the reference's
 *                whole-image np.clip does (a no-op when d_image is a primitive-walk output)
 * The dequantization and the transform run in float64 (the reference's scipy idctn is float64);
 * each channel's result is rounded to float32 before the colour transform, as the reference
 * does.  Coefficient indices outside [0, n_coeffs) and unsupported tile sizes are reported
 * through weftk_device_status and skipped.
 */
int weftk_dct_apply(const WeftDctTile* d_tiles, int n_tiles, const int16_t* d_coeffs, int64_t n_coeffs,
                    int chroma_mode, int band_layout, float quant_step, float freq_alpha, int max_size,
                    float* d_image, int width, int height, int clip_all, void* stream);

/*
 * Raster resize of the decoder: d_src (src_h x src_w x 3 float32) -> u8 = trunc(clip(x * 255,
 * 0, 255)) -> Pillow BILINEAR resize to dst_w x dst_h -> d_dst = u8 / 255 (float32, HWC).
 * d_tmp: caller scratch of src_h * dst_w * 3 bytes (the horizontal pass).  Sizes 1..65535.
 */
int weftk_raster_resize(const float* d_src, int src_w, int src_h, float* d_dst, int dst_w, int dst_h,
                        uint8_t* d_tmp, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WEFTK_DCT_H */
