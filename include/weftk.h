/*
 * weftk.h — C ABI of libweftk.so, the B200 (sm_100a) kernels for Weft's
 * primitive-stack hot path: per-tile analytic render, per-tile MSE scoring
 * for the greedy tile fit, the decoder's primitive walk, and the backward
 * pass used by gradient refinement.
 *
 * Conventions
 *   - Every entry point returns int status: 0 = OK, < 0 = error (see
 *     WEFTK_E_*); weftk_last_error() gives a message for the calling thread.
 *   - d_* arguments are device pointers owned by the caller; h_* are host
 *     pointers.  The library never frees caller memory.
 *   - stream is a cudaStream_t passed as void*; NULL means the legacy
 *     default stream.  Device-pointer entry points are asynchronous on that
 *     stream; *_host entry points are synchronous.
 *   - Structs are plain C, little-endian, no padding surprises (sizes are
 *     asserted in the implementation).
 */
#ifndef WEFTK_H
#define WEFTK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WEFTK_OK 0
#define WEFTK_E_ARG (-1)     /* bad argument (null pointer, bad size, bad enum) */
#define WEFTK_E_CUDA (-2)    /* a CUDA runtime call failed */
#define WEFTK_E_RANGE (-3)   /* a size is beyond a documented maximum */
#define WEFTK_E_DEVICE (-4)  /* a kernel reported an error status */

/* Flags for the scoring / render entry points. */
#define WEFTK_SAMPLE_CORNER 1 /* sample at integer pixel corners (reference GPU fit), not centres */

/* One primitive: 60 bytes, identical to the reference's PrimData / _PRIM_DTYPE
 * (src/weft/gpu_render.py:26-32, :241-247).  Kinds: 0 const patch, 1 linear
 * patch, 2 Gaussian line, 3 quadratic Bezier stroke, 4 triangle, 5 bicubic.
 * For kind 5, geom[0] holds the index (as a float) of the tile's 48-value
 * control grid in the cp48 side table of weftk_render_tiles. */
typedef struct WeftPrim {
    int32_t kind;
    float geom[7];
    float color0[3];
    float color1[3];
    float alpha;
} WeftPrim;

/* One evaluation (tile, primitive stack): 16 bytes, identical to the
 * reference's EvalDesc (src/weft/gpu_render.py:106-111). */
typedef struct WeftEval {
    int32_t prim_offset; /* first primitive of the stack in the prim array */
    int32_t prim_count;  /* stack length (0 = empty stack) */
    int32_t tile_offset; /* offset of the source tile in the pixel array, in floats */
    int32_t tile_size;   /* tile side in pixels (1..64) */
} WeftEval;

/* One decoded tile: 48 bytes, identical to the reference's TileDecodeDesc
 * (src/weft/gpu_render.py:179-192). */
typedef struct WeftTileDecodeDesc {
    int32_t prim_offset;
    int32_t prim_count;
    int32_t target_x0;
    int32_t target_y0;
    int32_t target_w;
    int32_t target_h;
    int32_t source_size; /* primitive coordinate space (encoded tile side) */
    int32_t res1_index;  /* RES1 grid index for this tile, -1 = none (reference: _pad) */
    float res0_r;        /* RES0 bias (int8 / 255) added after the composite */
    float res0_g;
    float res0_b;
    float _pad2;
} WeftTileDecodeDesc;

/* Library version (major * 10000 + minor * 100 + patch). */
int weftk_version(void);

/* Copy the calling thread's last error message into buf (always NUL-terminated).
 * Returns the full message length. */
int weftk_last_error(char* buf, size_t n);

/* Make `device` current for this thread and check it is an sm_100 part.
 * Must precede any other call on a thread that has not selected the device. */
int weftk_init(int device);

/* Read and clear the first error code a kernel reported on the current device
 * (0 = none).  Synchronizes with the device. */
int weftk_device_status(int* status);

/*
 * Score a batch of evaluations: for each eval, render the primitive stack over
 * its tile (over-composite from black, pixel centres unless
 * WEFTK_SAMPLE_CORNER) and write MSE = sum((clip(render) - src)^2) / (3 ts^2).
 * Replaces the reference kernel batch_tile_objective (src/weft/gpu_render.py:113-152)
 * behind gpu_batch_score_prepacked (:455-566); the MSE matches the reference's
 * CPU objective (src/weft/encoder.py:271-285 without residuals).
 *   d_evals  [n_evals]           d_prims [sum of stack lengths]
 *   d_tiles  float HWC pixels    d_mse   [n_evals] (output)
 */
int weftk_score_evals(const WeftEval* d_evals, int n_evals, const WeftPrim* d_prims, const float* d_tiles,
                      float* d_mse, int flags, void* stream);

/* Synchronous host-buffer form of weftk_score_evals: copies inputs to a
 * library-owned device arena, launches, copies the MSEs back.  This is the
 * call gpu_batch_score_prepacked makes (src/weft/gpu_render.py:523-558). */
int weftk_score_evals_host(const WeftEval* h_evals, int n_evals, const WeftPrim* h_prims, int n_prims,
                           const float* h_tiles, int64_t n_tile_floats, float* h_mse, int flags);

/*
 * Decoder primitive walk: render every tile's stack into its target rect of
 * an out_h x out_w x 3 float32 image (HWC), sampling the tile's
 * [0, source_size] coordinate space at the rect's pixel centres (a square
 * max(w, h) grid, cropped, as the reference CPU walk does), add RES0, clip,
 * add the bilinear RES1 grid if res1_index >= 0, clip.  Pixels no tile covers
 * are left untouched.  Replaces decode_tile_pixels (src/weft/gpu_render.py:179-237)
 * behind gpu_render_tiles_to_image (:594-690) with the semantics of
 * render_scene_adaptive (src/weft/render.py:270-358).
 *   d_items [n_items] work items (tile index, first row).  Each row of a tile's
 *                     target rect touches G = floor((x0 + w + 3) / 4) - floor(x0 / 4)
 *                     4-pixel groups aligned to output x multiples of 4; an item
 *                     covers R = max(1, WEFTK_DECODE_ITEM_GROUPS / G) consecutive rows
 *                     of its tile, i.e. tile t contributes items (t, r0), (t, r0 + R),
 *                     ... for the rows r0 <= r < r1 of its rect that lie inside the
 *                     image (r0 = max(0, -y0), r1 = min(h, out_h - y0)).  Rows of an
 *                     item outside the image are skipped.  Any order renders the same
 *                     image; in descending order of cost (pixels, times 4 for a tile
 *                     evaluated per pixel, i.e. anything but a lone constant layer
 *                     without a RES1 grid) the warps finish together.
 *   d_cp48  [n_cp48 * 48]  control grids for kind-5 tiles (may be NULL)
 *   d_res1  [n_res1 * 48]  RES1 grids, (4, 4, 3) row-major, float (may be NULL;
 *                          res1_index is ignored when n_res1 == 0)
 * Tiles with more than 48 primitives, a rect side outside 1..8192 or an
 * out-of-range grid index are skipped and reported through weftk_device_status.
 */
#define WEFTK_DECODE_ITEM_GROUPS 256
int weftk_render_tiles(const WeftTileDecodeDesc* d_descs, int n_tiles, const int32_t* d_items, int n_items,
                       const WeftPrim* d_prims, const float* d_cp48, int n_cp48, const float* d_res1, int n_res1,
                       float* d_out, int out_h, int out_w, int flags, void* stream);

/* Synchronous host-buffer form of weftk_render_tiles (gpu_render_tiles_to_image). */
int weftk_render_tiles_host(const WeftTileDecodeDesc* h_descs, int n_tiles, const WeftPrim* h_prims,
                            int n_prims, const float* h_cp48, int n_cp48, const float* h_res1, int n_res1,
                            float* h_out, int out_h, int out_w, int flags);

#ifdef __cplusplus
}
#endif

#endif /* WEFTK_H */
