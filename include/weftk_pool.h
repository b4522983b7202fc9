/*
 * weftk_pool.h — initial candidate pools generated on the device (C ABI of libweftk.so).
 *
 * Replaces the host candidate generation of the reference's adaptive fit for the
 * constant (kind 0) and linear (kind 1) patches: the per-tile worker
 * _worker_gen_cands (src/weft/encoder.py:2490-2517) = generate_edge_driven_candidates
 * (src/weft/edge_analysis.py:139-315) followed by _generate_candidates
 * (src/weft/encoder.py:535-745), de-duplicated by _dedup_candidates (:447-528), run in a
 * process pool on the host.  Here one CTA generates one tile's pool, in the reference's
 * order and with its float32 arithmetic:
 *   edge pool      palette (tile mean, then the means of the luminance-sorted pixels cut
 *                  into 2, 3 and 4 equal runs, each kept unless within 0.002 squared RGB
 *                  distance of one kept before) x alphas 1, .7, .4, .2; quadrant means
 *                  x .5, .3; for each dominant orientation of the reference's Sobel
 *                  histogram (12 bins of magnitude by angle, peaks >= 0.2 of the largest)
 *                  a split through the centre (side means) x 1, .7, .4 and two offset
 *                  splits x .5;
 *   template pool  the palette plus the means of the pixels above the 75th / below the
 *                  25th luminance percentile and at or above the 75th percentile of the
 *                  np.gradient magnitude, x 1, .7, .4, .2; quadrant means x .5, .3; 4x4
 *                  block means x .25; n_ang centre splits x 1, .7, .4 and 36 offset splits
 *                  x .5 with batched side means;
 * then the reference's coarse de-duplication key (geometry x4, colours x64, alpha x32,
 * first occurrence kept).  Every mean is numpy's: a sequential float32 sum in the
 * reference's pixel order divided by the count in float32; percentiles are numpy's
 * float32 linear interpolation; the palette sorts by (luminance, pixel index).  The one
 * rule that is not the host's numpy: the Sobel angle is the float64 arctan2 rounded to
 * float32 (numpy's float32 arctan2 differs in the last bit between host CPUs, and the
 * reference's Sobel values sit on the histogram's bin edges).
 *
 * The geometry of the split lines depends only on the tile side and the quality (as
 * float64, exactly as the reference computes it in Python): the host builds it once into
 * WeftPoolTables.
 */
#ifndef WEFTK_POOL_H
#define WEFTK_POOL_H

#include "weftk.h"

#ifdef __cplusplus
extern "C" {
#endif

#define WEFTK_POOL_MAX_SPECS 52            /* template split lines: n_ang (<= 16) + 36 */
#define WEFTK_POOL_MAX_CONST_LINEAR 272    /* candidates per tile before de-duplication, bound */
#define WEFTK_POOL_SPLITS (16 + WEFTK_POOL_MAX_SPECS)  /* split lines per tile side: 16 orientations,
                                                          then the template lines */
/* side-bit words of all four tile sides: WEFTK_POOL_SPLITS x (8^2 + 16^2 + 32^2 + 64^2) / 32 */
#define WEFTK_POOL_SIDE_WORDS (WEFTK_POOL_SPLITS * 170)

/* Host-built tables (device pointers), per tile side 8, 16, 32, 64 (index 0..3). */
typedef struct WeftPoolTables {
    const double* spec_geom;   /* [4][WEFTK_POOL_MAX_SPECS][4] template split lines x0, y0, x1, y1 */
    const float* spec_mask;    /* [4][WEFTK_POOL_MAX_SPECS][4] side test coefficients: x0, y0,
                                  y1 - y0, x1 - x0 (float32; a pixel (x, y) is on side a when
                                  (x - x0) * c2 - (y - y0) * c3 >= 0 in float32) */
    const double* orient_geom; /* [4][16][3][4] edge splits per orientation: centre line, then the
                                  offset lines at 0.25 and 0.75; orientations 0..11 are the
                                  histogram's bin centres, 12..15 the fallback 0, pi/4, pi/2, 3pi/4 */
    const float* orient_mask;  /* [4][16][4] side test coefficients of the centre lines */
    const double* bin_edges;   /* [13] orientation histogram bin edges (np.linspace(0, pi, 13)) */
    const int32_t* cuts;       /* [4][3][5] palette run boundaries for 2, 3, 4 runs */
    const uint32_t* side_bits; /* the side test of every split line over its tile's pixel grid:
                                  per side (8, 16, 32, 64 in turn) WEFTK_POOL_SPLITS rows (the 16
                                  orientations' centre lines, then the template lines) of
                                  side^2 / 32 words, bit p % 32 of word p / 32 set when raster
                                  pixel p is on side a; filled by weftk_pool_side_bits */
    int32_t n_spec;            /* template split lines (n_ang + 36) */
    int32_t n_centre;          /* the first n_centre of them are centre lines */
} WeftPoolTables;

/* One generation job over tiles resident on the device. */
typedef struct WeftPoolJob {
    const float* src;          /* float4 (r, g, b, 0) per pixel, tile-major, row-major in a tile */
    const int32_t* px_off;     /* [tiles] first pixel of each tile */
    const int32_t* pool_off;   /* [tiles] first candidate slot of each tile */
    int32_t pool_cap;          /* slots per tile; >= WEFTK_POOL_MAX_CONST_LINEAR */
    int32_t kinds_mask;        /* bit 0: constant patches, bit 1: linear patches */
    WeftPrim* cand;            /* output: tile t's pool in slots [pool_off[t], pool_off[t] + pool_cnt[t]) */
    int32_t* pool_cnt;         /* output: [tiles] candidates written */
    const int32_t* tiles[4];   /* indices of the tiles of side 8, 16, 32, 64 */
    int32_t n_tiles[4];
} WeftPoolJob;

/* Fill d_bits (WEFTK_POOL_SIDE_WORDS words, device) with the side test of tables->spec_mask
 * and tables->orient_mask over each tile side's pixel grid (the layout of
 * WeftPoolTables.side_bits; tables->side_bits itself is not read).  Once per table, on `stream`. */
int weftk_pool_side_bits(const WeftPoolTables* tables, uint32_t* d_bits, void* stream);

/* Generate the constant and linear candidates of every listed tile (one launch per tile
 * side, asynchronous on `stream`).  A tile whose pool would not fit pool_cap is truncated and
 * reported through weftk_device_status. */
int weftk_gen_pools(const WeftPoolTables* tables, const WeftPoolJob* job, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WEFTK_POOL_H */
