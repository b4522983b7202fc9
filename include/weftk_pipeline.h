/*
 * weftk_pipeline.h — the refined fit of whole images, one native call per image (C ABI of
 * libweftk.so).
 *
 * The reference encodes an image by decomposing it into a quadtree of tiles
 * (src/weft/quadtree.py:42-108), generating each tile's candidate pool on the host
 * (src/weft/encoder.py:2490-2517) and running the greedy fit (:2520-2898).  A WeftRefiner does
 * the device counterpart of that front end plus the refined fit, for one image per call:
 *   sRGB u8 image -> device; the variance-rule quadtree (weftk_quadtree_variance); the tile
 *   list back to the host (the only read in between, which the tile layout needs); tile
 *   extraction with the sRGB decode (weftk_extract_tiles); the constant + linear pools
 *   (weftk_gen_pools, WEFTK_POOL_MAX_CONST_LINEAR slots per tile); the init round over them
 *   with constants scored in closed form (weftk_fit_moments, weftk_fit_reset,
 *   weftk_fit_prepare, weftk_fit_round); `steps` fused Adam steps on each tile's pick
 *   (weftk_refine_start, weftk_refine_steps); the snap to the wire grid (weftk_quantize_rows);
 *   tiles, rows and kinds back to the host.
 * The device workspace is kept between calls and grows to the largest image seen, so a call
 * allocates nothing once the sizes repeat.  Results equal the same steps driven one entry point
 * at a time (the package's Python front end) bit for bit.
 */
#ifndef WEFTK_PIPELINE_H
#define WEFTK_PIPELINE_H

#include "weftk.h"
#include "weftk_pool.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct WeftRefineParams {
    int32_t cap;               /* primitive cap per tile of the fit state (>= 1) */
    int32_t steps;             /* Adam steps (>= 0) */
    int32_t min_tile;          /* quadtree tile sides: powers of two, 8 <= min <= max <= 64 */
    int32_t max_tile;
    int32_t chunk[3];          /* candidates per scoring CTA for 8-, 16- and 32/64-px tiles */
    int32_t variant[3];        /* scoring kernel shape per class (weftk_fit_variant) */
    float lr;                  /* Adam: learning rate, betas, epsilon (PyTorch's update rule) */
    float beta1;
    float beta2;
    float eps;
    double threshold;          /* quadtree: split while the sRGB-u8 luminance variance exceeds it */
    double lambda;             /* rate weight of the tile objective at the pools' quality */
    double complex_threshold;  /* the tile complexity threshold at that quality */
    const WeftPoolTables* tables;  /* device tables of the quality (kept by pointer; the caller
                                      keeps them alive as long as the refiner) */
    const float* srgb_lut;     /* device: 256 floats, the float32 sRGB decode of each u8 value */
} WeftRefineParams;

typedef struct WeftRefiner WeftRefiner;

/* A refiner on the current device with its own copy of *params (tables and lut by pointer). */
int weftk_refiner_create(const WeftRefineParams* params, WeftRefiner** out);
int weftk_refiner_destroy(WeftRefiner* refiner);

/*
 * Refine one h x w x 3 sRGB u8 image (host memory, row-major; page-locked copies fastest).
 * On success *n_tiles tiles were written: h_tiles int32[n][3] (x, y, side) in the quadtree's
 * order, h_rows float32[n][16] the refined primitive of each tile on the wire grid
 * (weftk_refine.h row layout), h_kinds int32[n] its kind (-1: none); page-locked h_rows and
 * h_kinds come back by DMA, faster than pageable ones.  More than max_tiles
 * tiles: WEFTK_E_RANGE with *n_tiles set and nothing written.  Device work on `stream`;
 * returns after the results are on the host.
 */
int weftk_refine_image(WeftRefiner* refiner, const uint8_t* h_img, int h, int w, int32_t* h_tiles, float* h_rows,
                       int32_t* h_kinds, int max_tiles, int* n_tiles, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WEFTK_PIPELINE_H */
