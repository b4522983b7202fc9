/*
 * weftk_quadtree.h — quadtree tiling and tile extraction on the device (C ABI of libweftk.so).
 *
 * The fit's host front end (src/weft/quadtree.py:42-108: decompose_quadtree and
 * extract_adaptive_tiles) with the split rule of the batched workloads: a tile of side s
 * splits into its four quarters while s > min_tile and the variance of its sRGB-u8
 * luminance (0.2126 R + 0.7152 G + 0.0722 B on 0..255 values, float64, numpy's np.var:
 * mean of squared deviations from the mean) exceeds the threshold.  The image is
 * edge-padded to a multiple of max_tile; macro tiles are visited row-major and each is split
 * recursively in top-left, top-right, bottom-left, bottom-right order, so the tile list
 * comes out in the reference's order.
 */
#ifndef WEFTK_QUADTREE_H
#define WEFTK_QUADTREE_H

#include "weftk.h"

#ifdef __cplusplus
extern "C" {
#endif

/* *bytes = the device workspace weftk_quadtree_variance needs for an h x w image. */
int weftk_quadtree_work_bytes(int h, int w, int max_tile, int min_tile, int64_t* bytes);

/*
 * Quadtree of an h x w sRGB u8 image (HWC, row-major, device): writes *d_n_tiles and the tiles
 * as int32 triples (x, y, side) into d_tiles (capacity max_tiles; a larger count is reported
 * through weftk_device_status and truncated).  max_tile and min_tile are powers of two with
 * 8 <= min_tile <= max_tile <= 64.  d_work: weftk_quadtree_work_bytes bytes of device memory
 * the caller owns.  Two launches on `stream`, no host synchronisation.
 */
int weftk_quadtree_variance(const uint8_t* d_img, int h, int w, double threshold, int max_tile, int min_tile,
                            int32_t* d_tiles, int max_tiles, int32_t* d_n_tiles, void* d_work, void* stream);

/*
 * Tile pixels of an h x w sRGB u8 image, converted to linear by the 256-entry table d_lut
 * (the host's float32 sRGB decode of each u8 value, src/weft/image_io.py:9-24) and written as
 * float4 (r, g, b, 0) per pixel, tile-major, row-major inside a tile, starting at pixel
 * d_px_off[t] of d_src4 (the fit's pixel layout).  Pixels past the image edge repeat the last
 * row / column (the reference's edge padding).  d_tiles: int32 (x, y, side) triples.
 */
int weftk_extract_tiles(const uint8_t* d_img, int h, int w, const float* d_lut, const int32_t* d_tiles,
                        int n_tiles, const int32_t* d_px_off, float* d_src4, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WEFTK_QUADTREE_H */
