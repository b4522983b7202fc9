/*
 * weftk_fit.h — device-resident greedy candidate-scoring fit (C ABI of libweftk.so).
 *
 * Replaces the greedy loop of the reference's adaptive fit
 * (src/weft/encoder.py:2668-2831, _fit_adaptive_state), whose every round was a
 * host->device copy, a batch_tile_objective launch, a device->host copy and a
 * host argmin.  Here all tiles' pixels, candidate pools, selections and
 * objectives stay in device memory; one call runs one round for every tile.
 *
 * Memory is owned by the caller (all pointers below are device pointers) and
 * laid out tile-major:
 *   pixels     float4 (r, g, b, 0) per pixel, each tile's ts*ts pixels
 *              row-major starting at px_off[t];
 *   candidates tile t owns slots [pool_off[t], pool_off[t] + pool_cap[t]) of
 *              every candidate array; the first pool_cnt[t] are filled
 *              (original order = tie-break order, as in the reference).
 *
 * Round semantics (mode WEFTK_FIT_ROUND), per tile with flag COMPLEX, at least
 * one live candidate and fewer than cap[t] selected primitives:
 *   mse_k = mean over pixels and channels of (clip(cand_k over bg) - src)^2
 *   obj_k = mse_k + f32(lambda) * f32(sel_bits + 8 * bytes[kind_k])  (float32)
 *   k* = first argmin; accept if (double)obj_k* < cur_obj[t].
 * An accepted candidate is composited into bg, appended to sel, its slot marked
 * dead, sel_bits and cur_obj updated.  If any tile improved, COMPLEX becomes
 * "improved this round"; otherwise COMPLEX is unchanged (the caller re-seeds).
 * Mode WEFTK_FIT_INIT scores every live candidate alone over black, accepts
 * each tile's argmin unconditionally, sets cur_obj = (double)mse + lambda*bits
 * and COMPLEX = cur_obj > complex_threshold and a live candidate remains.
 */
#ifndef WEFTK_FIT_H
#define WEFTK_FIT_H

#include "weftk.h"

#ifdef __cplusplus
extern "C" {
#endif

#define WEFTK_FIT_INIT 0
#define WEFTK_FIT_ROUND 1

#define WEFTK_TILE_COMPLEX 1
#define WEFTK_TILE_EVAL 2
#define WEFTK_TILE_IMPROVED 4

/* Byte size of a candidate's kind on the wire; bits per primitive = 8 * this
 * (src/weft/encoder.py:242-256: 7, 18, 17, 21, 19, everything else 20). */
#define WEFTK_PRIM_BYTES {7, 18, 17, 21, 19, 20, 20, 20}

typedef struct WeftFitState {
    int32_t n_tiles;
    int32_t cap_max;         /* row stride of sel[] */
    int64_t n_slots;         /* candidate slots in total */
    /* tiles */
    const float* src;        /* float4 per pixel */
    float* bg;               /* float4 per pixel: composite of the selected stack; may be NULL for a
                                fit that runs only its init round (then nothing is composited; greedy
                                rounds and re-seeding refuse it) */
    const int32_t* px_off;   /* [n_tiles] pixel offset of the tile */
    const int32_t* size;     /* [n_tiles] tile side: 8, 16, 32 or 64 */
    const int32_t* cap;      /* [n_tiles] primitive cap */
    const int32_t* pool_off; /* [n_tiles] first slot */
    int32_t* pool_cnt;       /* [n_tiles] filled slots (grows with re-seeds) */
    const int32_t* pool_cap; /* [n_tiles] slots reserved for the tile */
    int32_t* n_alive;        /* [n_tiles] live candidates */
    int32_t* n_sel;          /* [n_tiles] selected primitives */
    int32_t* sel_bits;       /* [n_tiles] 8 + sum of 8 * bytes[kind] over the selection */
    int32_t* flags;          /* [n_tiles] WEFTK_TILE_* bits */
    double* cur_obj;         /* [n_tiles] current objective */
    int32_t* sel;            /* [n_tiles * cap_max] selected slot indices (pool-local) */
    /* candidates (slot-indexed) */
    const WeftPrim* cand;    /* [n_slots] candidate records */
    float* prep;             /* [n_slots * 16] prepared per-candidate terms (64 B each) */
    uint8_t* alive;          /* [n_slots] 1 = still in the pool */
    uint8_t* kind;           /* [n_slots] primitive kind of the slot (filled by prepare / re-seed) */
    float* partial;          /* [n_slots * 4] per-1024-pixel-block squared-error sums (scratch) */
    int32_t* status;         /* [4] round counters: evaluated tiles, improved tiles */
    unsigned long long* work; /* [2] running totals: candidate-pixels scored, algorithmic FP32 ops
                                 (per candidate-pixel: per-kind op count + 9 for the error); may be NULL */
    /* Scoring-kernel shape per tile-size class [8-px, 16-px, 32/64-px tiles], an index into
     * that class's table (0 = default; WEFTK_FIT_VARIANTS per class, see weftk_fit_variant):
     * pixels per lane x warps per candidate x CTAs per SM.  Chosen by the autotuner. */
    int32_t variant[3];
    int32_t _pad;
    /* Optional (NULL: off): per-tile pixel moments, double[n_tiles * 6] = sum of src r, g, b and
     * of their squares (weftk_fit_moments).  When set, the init round scores a constant
     * candidate in closed form — over an empty stack its render is one colour q per channel,
     * so its squared error is n q^2 - 2 q S1 + S2 — instead of per pixel (equal up to
     * rounding; a near tie may then pick differently from the per-pixel sum). */
    const double* moments;
    /* Optional (NULL: off): the round's work queue.  With both set, every round first lists the
     * scoring items whose tile is evaluated and whose slot run holds filled slots (per size class,
     * any order), and the scoring launches are persistent grids of about one wave that pull those
     * items, so late rounds with few live tiles and runs past a pool's filled slots cost no CTA
     * launches.  queue: int32[n_items8 + n_items16 + n_items32]; queue_ctl: int32[8] scratch. */
    int32_t* queue;
    int32_t* queue_ctl;
} WeftFitState;

/* Fill d_moments (double[n_tiles * 6]) from the fit's tile pixels. */
int weftk_fit_moments(const WeftFitState* st, double* d_moments, void* stream);

#define WEFTK_FIT_VARIANTS 3

/* Shape of scoring variant `variant` of size class `size_class` (8, 16 or 32): pixels per lane,
 * warps per candidate, resident CTAs per SM the register budget targets. */
int weftk_fit_variant(int size_class, int variant, int* pixels_per_lane, int* warps_per_candidate,
                      int* ctas_per_sm);

/* A unit of scoring work: tile, 1024-pixel block, and a run of candidate
 * slots (pool-local, into perm). */
typedef struct WeftFitItem {
    int32_t tile;
    int32_t block;
    int32_t first;
    int32_t count;
} WeftFitItem;

/* Prepare candidate slots [pool_off[t] + lo, pool_off[t] + pool_cnt[t]) of every
 * tile whose slot range changed: compute the prepared terms and mark them live.
 * first_new[t] = first pool-local slot to prepare (pass pool_cnt[t] to skip). */
int weftk_fit_prepare(const WeftFitState* st, const int32_t* d_first_new, void* stream);

/* The whole greedy fit, enqueued without any host synchronisation (so it can be captured in a
 * CUDA graph): the init round, then max_rounds greedy rounds whose kernels skip their work once
 * the fit is over, with the host loop's decisions taken on the device after every round
 * (src/weft/encoder.py:2745-2830: a round that evaluates no tile ends the fit; a round without
 * improvement is a stall; more than three stalls end it; otherwise a stall re-seeds the complex
 * tiles on the device).  d_ctl: int32[4] scratch (done, stalls, re-seed pending, rounds run),
 * readable after the stream completes.  Requires scoring timing off (weftk_fit_timing). */
int weftk_fit_run(const WeftFitState* st, int max_rounds, double lambda, double complex_threshold,
                  const int32_t* d_perm, const WeftFitItem* d_items8, int n_items8, const WeftFitItem* d_items16,
                  int n_items16, const WeftFitItem* d_items32, int n_items32, int32_t* d_ctl, void* stream);

/* Start the fit over: per tile, pool_cnt = d_init_cnt (the initial pools), no selection
 * (n_sel 0, sel -1, sel_bits 8, objective 0, flags 0), every slot dead and n_alive 0 (a
 * following weftk_fit_prepare with zero first_new revives the initial pools), the composite bg
 * zero; the work counters zero.  One launch; no host synchronisation. */
int weftk_fit_reset(const WeftFitState* st, const int32_t* d_init_cnt, void* stream);

/*
 * Run one fit round over all tiles.
 *   d_perm     [n_slots] pool-local scoring order of each tile's slots (any
 *              permutation; ties are broken by slot index, not by perm)
 *   d_items_*  scoring work for tiles of side 8, 16, and >= 32 (block-split)
 *   lambda     rate weight (_tile_lambda of the quality)
 * Counters are written to st->status; read them after the stream syncs.
 */
int weftk_fit_round(const WeftFitState* st, int mode, double lambda, double complex_threshold,
                    const int32_t* d_perm, const WeftFitItem* d_items8, int n_items8,
                    const WeftFitItem* d_items16, int n_items16, const WeftFitItem* d_items32, int n_items32,
                    void* stream);

/*
 * Re-seed every tile that has flag COMPLEX and room under its cap with
 * residual-targeted candidates, generated on the device from src and the
 * clipped composite bg (the reference's _generate_residual_candidates,
 * src/weft/encoder.py:1255-1366), de-duplicated, appended to the tile's pool,
 * prepared and marked live.  At most 117 candidates per tile per call; a tile
 * whose reserved slots would overflow is skipped and reported.
 */
int weftk_fit_reseed(const WeftFitState* st, int quality, void* stream);

/*
 * weftk_fit_round_static — weftk_fit_round for callers that cannot allocate device
 * memory.  No counterpart in the reference.  Some callers must not call
 * cudaMalloc while they run: hosts that hand the library a fixed device budget
 * up front (plugin and FFI hosts with their own pool), latency-sensitive
 * services for which cudaMalloc's implicit device synchronisation would stall
 * other streams, and callers in the middle of stream-ordered work that an
 * allocation would serialise.  This entry point takes the same state but
 * ignores st->partial: the per-candidate scoring scratch lives in a file-scope
 * __device__ array of WEFTK_FIT_STATIC_SCRATCH_FLOATS floats (16 MiB) that every
 * GPU loading the library holds until the process exits.  It calls no
 * cudaMalloc/cudaFree and no allocating library routine.
 *   - needs 4 * st->n_slots <= WEFTK_FIT_STATIC_SCRATCH_FLOATS, else WEFTK_E_RANGE;
 *   - the first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress) with that device current; make that first call
 *     before any stream capture;
 *   - all calls share the one array and it keeps the last call's contents; a
 *     round writes every scratch entry before it reads it, so nothing needs
 *     clearing, but calls whose work overlaps on the GPU (other streams, other
 *     threads) race on the array and must be serialised by the caller.
 */
#define WEFTK_FIT_STATIC_SCRATCH_FLOATS (4 * 1024 * 1024)
int weftk_fit_round_static(const WeftFitState* st, int mode, double lambda, double complex_threshold,
                           const int32_t* d_perm, const WeftFitItem* d_items8, int n_items8,
                           const WeftFitItem* d_items16, int n_items16, const WeftFitItem* d_items32,
                           int n_items32, void* stream);

/* Kernel timing for measurement: while enabled, weftk_fit_round brackets its
 * scoring launches with CUDA events.  *score_ms receives the summed device time
 * of the scoring launches since the previous query and *n_rounds how many
 * rounds that covers; both reset on read.  Call after the stream has synced. */
int weftk_fit_timing(int enable, double* score_ms, int* n_rounds);

/* Measured FP32 FMA throughput of the current GPU in GFLOP/s (2 ops per FMA):
 * a register-resident FMA loop on every SM, timed with CUDA events. */
int weftk_measure_fp32_peak(double* gflops);

#ifdef __cplusplus
}
#endif

#endif /* WEFTK_FIT_H */
