/*
 * weftk_refine.h — per-tile stack loss and its hand-written backward (C ABI of libweftk.so).
 *
 * No counterpart in the reference renderer's interface: the reference has no
 * differentiable path (its refinement is discrete perturbation).  The forward is
 * the reference's objective without the rate term (src/weft/encoder.py:271-285):
 * loss[t] = mean over pixels and channels of (clip(render(stack_t)) - src)^2, with
 * render = the reference CPU renderer's over-composite at pixel centres
 * (src/weft/render.py:127-234).  The backward recomputes coverage per pixel (no
 * per-pixel state is stored in HBM) and returns d(sum_t g[t] * loss[t]) / d params.
 *
 * Parameter rows: float[16] per primitive
 *   [0..6]  geom (kind-specific, as WeftPrim.geom)   [7..9]  color0
 *   [10..12] color1 (linear patch)                   [13]    alpha     [14..15] unused
 * Gradients exist for geometry (positions, thickness), colours and opacity.
 * Triangle coverage is a step function; its geometry gradient uses a soft-edge
 * surrogate (product of logistic functions of the signed edge distances,
 * width 0.5 px) in the backward only.  WEFTK_SOFT_TRIANGLES makes the forward use
 * the same surrogate, which is what a finite-difference check of the surrogate
 * differentiates.  Bicubic (kind 5) rows are inert.
 */
#ifndef WEFTK_REFINE_H
#define WEFTK_REFINE_H

#include "weftk.h"

#ifdef __cplusplus
extern "C" {
#endif

#define WEFTK_SOFT_TRIANGLES 2
/* Loss of the decoded tile: the error left after the decoder adds back the 4x4
 * grid of block-mean errors with bilinear interpolation (the tile's RES1 map,
 * src/weft/encoder.py:3248-3372, src/weft/render.py:474-515), ignoring the grid's
 * 8-bit quantisation.  Tile sides must be 8, 16, 32 or 64. */
#define WEFTK_LOSS_RESIDUAL 4
#define WEFTK_REFINE_MAX_PRIMS 32 /* longest stack the refine kernels accept */

typedef struct WeftStackSet {
    int32_t n_tiles;
    int32_t max_prims;        /* longest stack (<= WEFTK_REFINE_MAX_PRIMS) */
    const float* src;         /* float4 (r, g, b, 0) per pixel, tile-major */
    const int32_t* px_off;    /* [n_tiles] first pixel of the tile */
    const int32_t* size;      /* [n_tiles] tile side (1..64) */
    const int32_t* prim_off;  /* [n_tiles + 1] tile t owns parameter rows [prim_off[t], prim_off[t+1]) */
    const int32_t* kind;      /* [n_prims] primitive kind of each row */
    /* Optional work split by tile side (NULL: four warps per tile): a permutation
     * of the tiles listing n_big tiles of side > 32 (eight warps each), then n_mid
     * of side 17..32 (four warps), then n_s16 of side 9..16 (two warps), then the
     * rest (one warp).  The split only affects speed; any valid split gives the
     * same results. */
    const int32_t* order;
    int32_t n_big;
    int32_t n_mid;
    int32_t n_s16;
    /* Kinds the rows may hold, bit k for kind k (0: not declared).  Sets of at most one layer
     * per tile whose mask is within {constant, linear} run a register-only kernel; a row of
     * another kind is then reported (WEFTK_E_ARG in the device status) and treated as absent. */
    int32_t kinds_mask;
    /* Optional (NULL: off): per-tile pixel sums, double[n_tiles * 6] = sum of src r, g, b and of
     * their squares (the fit's weftk_fit_moments).  With the register path, a tile whose stack is
     * one constant layer then runs as one thread: over black such a layer renders one colour q
     * per channel, so its loss n q^2 - 2 q S1 + S2 and its gradient n q - S1 per channel need no
     * pixel loop (no residual loss). */
    const double* moments;
} WeftStackSet;

/* loss[t] for every tile (float32). */
int weftk_stack_loss(const WeftStackSet* set, const float* d_params, float* d_loss, int flags, void* stream);

/* grad_params = sum_t grad_loss[t] * d loss[t] / d params (rows of untouched
 * tiles are written with zeros; rows are owned by one tile, so no atomics).
 * d_loss (may be NULL) receives loss[t] from the same pass (the backward
 * re-renders every pixel anyway). */
int weftk_stack_loss_backward(const WeftStackSet* set, const float* d_params, const float* d_grad_loss,
                              float* d_grad_params, float* d_loss, int flags, void* stream);

/* One Adam step (PyTorch's update rule, FP32 moments) on every row, fused with the
 * projection onto what the wire format carries: colours and alpha in [0, 1],
 * coordinates in [0, 15], thickness in [0, 4] (src/weft/primitives.py:102-177).
 * d_step holds the step count t-1 on entry and is incremented by the call, so a
 * captured sequence of calls replays correctly. */
int weftk_adam_step(float* d_params, const float* d_grads, float* d_m, float* d_v, const int32_t* d_kind,
                    int n_rows, float lr, float beta1, float beta2, float eps, int32_t* d_step, void* stream);

/* One refinement step in one launch: the loss and gradient of every tile (as
 * weftk_stack_loss_backward) followed, inside the same tile group, by the Adam
 * step and projection of weftk_adam_step on the tile's own rows.  d_params is
 * updated in place.  Each row's step count is kept in d_m[row * 16 + 15] (zero
 * it with the moments to restart).  d_loss and d_grad_params may be NULL. */
int weftk_refine_step(const WeftStackSet* set, float* d_params, float* d_m, float* d_v, const float* d_grad_loss,
                      float* d_loss, float* d_grad_params, float lr, float beta1, float beta2, float eps, int flags,
                      void* stream);

/* `steps` refinement steps in one launch: each tile group repeats weftk_refine_step's work on
 * its own rows (tiles never interact), keeping the rows and moments in shared memory between
 * steps.  The same results as `steps` calls of weftk_refine_step; d_loss receives the last
 * step's loss and d_grad_params (may be NULL) its gradient. */
int weftk_refine_steps(const WeftStackSet* set, int steps, float* d_params, float* d_m, float* d_v,
                       const float* d_grad_loss, float* d_loss, float* d_grad_params, float lr, float beta1,
                       float beta2, float eps, int flags, void* stream);

/* Start a refinement from a fit: row r = the first selected primitive of tile d_tiles[r] of the
 * fit state (weftk_fit.h), as a parameter row projected onto the wire box, its kind in
 * d_kind[r], and zero Adam moments and step count (d_m, d_v rows).  A tile without a selection
 * gets an all-zero row of kind -1 (no layer).  One launch. */
struct WeftFitState;
int weftk_refine_start(const struct WeftFitState* fit, const int32_t* d_tiles, int n_rows, float* d_params,
                       float* d_m, float* d_v, int32_t* d_kind, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WEFTK_REFINE_H */
