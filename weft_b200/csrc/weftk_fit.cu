// weftk_fit.cu — device-resident greedy candidate-scoring fit (see include/weftk_fit.h).
//
// Scoring exploits the greedy's structure: every eval of a round is "the tile's
// selected stack + one candidate on top", and the over-composite is evaluated
// back to front, so the selected stack's composite (bg) is kept per pixel in
// HBM and each eval composites ONE primitive over it.  The float operations are
// the same sequence a full re-render performs, so results are identical to
// rendering the whole stack (blend() is shared with the decode walk).
//
// Work mapping (all CTAs are 128 threads = 4 warps; a warp works on one
// candidate at a time, each lane owns PPL pixels held in registers):
//   8-px tiles   PPL=2, one warp covers the tile, 4 independent warps per CTA
//   16-px tiles  PPL=8, one warp covers the tile, 4 independent warps per CTA
//   32/64-px     PPL=8, four warps cover a 1024-pixel block; a CTA scores a run
//                of candidates on one block and combines the 4 warp sums in
//                shared memory in a fixed order.
// Per-candidate sums go to partial[slot*4 + block] (float32, fixed reduction
// order, so results are deterministic run to run).
#include <cuda_runtime.h>

#include <algorithm>

#include <climits>
#include <map>
#include <mutex>
#include <string>

#include "../../include/weftk_fit.h"
#include "weftk_common.cuh"
#include "weftk_prim.cuh"

namespace weftk {

extern __device__ int g_device_status;
__device__ __forceinline__ void fit_report(int code) { atomicCAS(&g_device_status, 0, code); }

__constant__ int c_prim_bytes[8] = WEFTK_PRIM_BYTES;

__device__ __forceinline__ int prim_bits(int kind) { return 8 * c_prim_bytes[(kind >= 0 && kind < 8) ? kind : 7]; }

// FP32 operations to evaluate and blend one primitive at one pixel (FMA = 2): const 10,
// linear 24, line 28, curve 31 segments x 16 + 13 = 509, triangle 26.
__constant__ int c_kind_ops[8] = {10, 24, 28, 509, 26, 0, 0, 0};
__device__ __forceinline__ int kind_ops(int kind) { return c_kind_ops[(kind >= 0 && kind < 8) ? kind : 7]; }

__device__ __forceinline__ Prep load_prep(const float* prep, long long slot) {
    const float4* p = reinterpret_cast<const float4*>(prep) + slot * 4;
    Prep r;
    float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
    r.kind = __float_as_int(a.x);
    r.a = a.y;
    r.cr = a.z;
    r.cg = a.w;
    r.cb = b.x;
    r.q[0] = b.y; r.q[1] = b.z; r.q[2] = b.w;
    r.q[3] = c.x; r.q[4] = c.y; r.q[5] = c.z; r.q[6] = c.w;
    r.q[7] = d.x; r.q[8] = d.y; r.q[9] = d.z; r.q[10] = d.w;
    return r;
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// ------------------------------------------------------------------ prepare
__global__ void fit_prepare_kernel(WeftFitState st, const int* __restrict__ first_new) {
    const int t = blockIdx.x;
    if (t >= st.n_tiles) return;
    const int lo = first_new[t], hi = st.pool_cnt[t];
    const long long off = st.pool_off[t];
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const long long slot = off + i;
        const WeftPrim& P = st.cand[slot];
        WeftPrim c;
        c.kind = P.kind;
#pragma unroll
        for (int k = 0; k < 7; ++k) c.geom[k] = P.geom[k];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            c.color0[k] = P.color0[k];
            c.color1[k] = P.color1[k];
        }
        c.alpha = P.alpha;
        Prep r = prep_prim(c);
        if (r.kind == K_BICUBIC) r.kind = K_SKIP;  // bicubic grids are never fit candidates
        float4* dst = reinterpret_cast<float4*>(st.prep) + slot * 4;
        dst[0] = make_float4(__int_as_float(r.kind), r.a, r.cr, r.cg);
        dst[1] = make_float4(r.cb, r.q[0], r.q[1], r.q[2]);
        dst[2] = make_float4(r.q[3], r.q[4], r.q[5], r.q[6]);
        dst[3] = make_float4(r.q[7], r.q[8], r.q[9], r.q[10]);
        st.alive[slot] = 1;
        st.kind[slot] = (uint8_t)(c.kind >= 0 && c.kind < 8 ? c.kind : 7);
    }
    if (threadIdx.x == 0 && hi > lo) st.n_alive[t] += hi - lo;
}

// ------------------------------------------------------------------ round begin / end
// ctl (device-driven fit, may be NULL): [0] done, [1] stalls, [2] re-seed pending, [3] rounds.
__global__ void fit_begin_kernel(WeftFitState st, int mode, int* ctl) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= st.n_tiles) return;
    const bool done = ctl != nullptr && ctl[0] != 0;
    if (ctl != nullptr && t == 0) ctl[2] = 0;  // the pending re-seed (if any) ran before this launch
    int f = st.flags[t] & ~(WEFTK_TILE_EVAL | WEFTK_TILE_IMPROVED);
    bool ev;
    if (done)
        ev = false;
    else if (mode == WEFTK_FIT_INIT)
        ev = st.n_alive[t] > 0;
    else
        ev = (f & WEFTK_TILE_COMPLEX) && st.n_alive[t] > 0 && st.n_sel[t] < st.cap[t];
    if (ev) {
        f |= WEFTK_TILE_EVAL;
        atomicAdd(&st.status[0], 1);
    }
    st.flags[t] = f;
}

// The host loop's decisions after a greedy round, on the device (src/weft/encoder.py:2745-2830):
// no evaluated tile ends the fit; a round without improvement is a stall, more than three
// stalls end it, otherwise a stall triggers a re-seed; an improving round resets the count.
__global__ void fit_control_kernel(const int* __restrict__ status, int* ctl) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || ctl[0]) return;
    if (status[0] == 0) {
        ctl[0] = 1;
        return;
    }
    ctl[3] += 1;
    if (status[1] == 0) {
        ctl[1] += 1;
        if (ctl[1] > 3)
            ctl[0] = 1;
        else
            ctl[2] = 1;
    } else {
        ctl[1] = 0;
    }
}

__global__ void fit_end_kernel(WeftFitState st, int mode, double complex_threshold) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= st.n_tiles) return;
    int f = st.flags[t];
    if (mode == WEFTK_FIT_INIT) {
        bool cx = st.cur_obj[t] > complex_threshold && st.n_alive[t] > 0;
        f = cx ? (f | WEFTK_TILE_COMPLEX) : (f & ~WEFTK_TILE_COMPLEX);
    } else if (*(volatile int*)&st.status[1] > 0) {
        f = (f & WEFTK_TILE_IMPROVED) ? (f | WEFTK_TILE_COMPLEX) : (f & ~WEFTK_TILE_COMPLEX);
    }
    st.flags[t] = f;
}

// ------------------------------------------------------------------ scoring
// A CTA first gathers the live candidates of its run into shared memory (prepared
// terms + slot), compacting out dead slots; warps then read their candidate's terms
// as warp-uniform shared-memory broadcasts.  A curve's 31 polyline segments are
// computed one per lane into the warp's segment table and read back the same way.
constexpr int MAX_ITEM = 128;

template <int WPC>
struct ScoreSmem {
    float4 prep[MAX_ITEM][4];
    int slot[MAX_ITEM];
    int wcount[4];
    float4 seg[4][32][2];
    float red[WPC > 1 ? MAX_ITEM : 1][WPC];
};

// One scoring work item (tile, 1024-pixel block, run of candidate slots) by the whole CTA.
// INIT: the init round, over empty stacks: the cached composite is black, so it is not read and the
// blend over it is the product s * a (the fused form over +0 differs only in the sign of a zero
// result, which the clamp removes), the same values as the general form.
template <int PPL, int WPC, bool INIT>
__device__ __forceinline__ void score_item(const WeftFitState& st, const int* __restrict__ perm, const WeftFitItem w,
                                           int expect_min, int expect_max, bool mode_init, ScoreSmem<WPC>& sm) {
    constexpr int GROUPS = 4 / WPC;
    float4(&s_prep)[MAX_ITEM][4] = sm.prep;
    int(&s_slot)[MAX_ITEM] = sm.slot;
    int(&s_wcount)[4] = sm.wcount;
    float4(&s_seg)[4][32][2] = sm.seg;
    auto& red = sm.red;
    const int t = w.tile;
    if (t < 0 || t >= st.n_tiles) {
        if (threadIdx.x == 0) fit_report(WEFTK_E_ARG);
        return;
    }
    if (!(st.flags[t] & WEFTK_TILE_EVAL)) return;
    const int ts = st.size[t];
    const bool closed_form = mode_init && st.moments != nullptr;
    // a slot range outside the state's slot arrays (a malformed caller-built pool table) is
    // rejected, never scored: the per-candidate scratch is indexed by slot
    if (ts < expect_min || ts > expect_max || w.count > MAX_ITEM || w.block * 1024 >= ts * ts || w.first < 0 ||
        w.first + w.count > st.pool_cap[t] || st.pool_off[t] < 0 ||
        (long long)st.pool_off[t] + w.first + w.count > st.n_slots) {
        if (threadIdx.x == 0) fit_report(WEFTK_E_ARG);
        return;
    }
    // items cover the tile's reserved slots; only the filled ones are scored
    const int count = min(w.count, st.pool_cnt[t] - w.first);
    if (count <= 0) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long off = st.pool_off[t];

    // stage live candidates (order-preserving compaction with warp ballots)
    long long my_slot = -1;
    bool live = false;
    if ((int)threadIdx.x < count) {
        my_slot = off + perm[off + w.first + threadIdx.x];
        live = st.alive[my_slot] != 0;
        if (live && closed_form && st.kind[my_slot] == K_CONST) {
            // Init round over an empty stack: a constant layer renders one colour q per channel,
            // so sum over pixels and channels of (q - s)^2 = sum_ch n q^2 - 2 q S1 + S2.
            const float4 head = __ldg(reinterpret_cast<const float4*>(st.prep) + my_slot * 4);
            const float4 head2 = __ldg(reinterpret_cast<const float4*>(st.prep) + my_slot * 4 + 1);
            const float a = head.y, col[3] = {head.z, head.w, head2.x};
            const double* mo = st.moments + (size_t)t * 6;
            const double npx = (double)(ts * ts);
            double e = 0.0;
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) {
                const double q = (double)clamp01(blend(col[ch], a, 0.0f));
                e += npx * q * q - 2.0 * q * mo[ch] + mo[3 + ch];
            }
            st.partial[my_slot * 4 + w.block] = w.block == 0 ? (float)e : 0.0f;
            live = false;  // not evaluated per pixel
        }
    }
    const unsigned bal = __ballot_sync(FULL, live);
    if (lane == 0) s_wcount[warp] = __popc(bal);
    __syncthreads();
    int base = 0;
    for (int k = 0; k < warp; ++k) base += s_wcount[k];
    const int m = s_wcount[0] + s_wcount[1] + s_wcount[2] + s_wcount[3];
    unsigned long long ops = 0;
    int my_curve = 0;
    if (live) {
        const int pos = base + __popc(bal & ((1u << lane) - 1u));
        const float4* src4 = reinterpret_cast<const float4*>(st.prep) + my_slot * 4;
        const float4 head = __ldg(src4);
        ops = (unsigned long long)(WPC * 32 * PPL) * (unsigned long long)(kind_ops(__float_as_int(head.x)) + 9);
        my_curve = __float_as_int(head.x) == K_CURVE;
        s_prep[pos][0] = head;
        s_prep[pos][1] = __ldg(src4 + 1);
        s_prep[pos][2] = __ldg(src4 + 2);
        s_prep[pos][3] = __ldg(src4 + 3);
        s_slot[pos] = (int)(my_slot - off);
    }
    const int any_curve = __syncthreads_or(my_curve);
    if (m == 0) return;
    // The closed-form init round of 8-px tiles without curves: half a warp per candidate, 4 pixels
    // per lane, so the candidate's terms and its reduction are shared by twice the pixels per lane.
    // Its pixel sums run in another order than the full-warp form's (equal to float rounding), so
    // it serves only the fit with closed-form constants, which has no reference summation to match.
    bool half_done = false;
    if constexpr (INIT && PPL == 2 && WPC == 1) {
        if (closed_form && !any_curve && ts == 8) {
            const int half = lane >> 4, sub = lane & 15;
            const float4* src = reinterpret_cast<const float4*>(st.src) + st.px_off[t];
            float hx[4], hy[4];
            float3 hs[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int p = j * 16 + sub;  // an 8-px tile's 64 pixels
                hx[j] = (float)(p & 7) + 0.5f;
                hy[j] = (float)(p >> 3) + 0.5f;
                const float4 a = src[p];
                hs[j] = make_float3(a.x, a.y, a.z);
            }
            for (int c0 = warp * 2; c0 < m; c0 += 8) {
                const int c = min(c0 + half, m - 1);
                Prep P;
                {
                    const float4 a = s_prep[c][0], b = s_prep[c][1], cc = s_prep[c][2], d = s_prep[c][3];
                    P.kind = __float_as_int(a.x);
                    P.a = a.y; P.cr = a.z; P.cg = a.w; P.cb = b.x;
                    P.q[0] = b.y; P.q[1] = b.z; P.q[2] = b.w;
                    P.q[3] = cc.x; P.q[4] = cc.y; P.q[5] = cc.z; P.q[6] = cc.w;
                    P.q[7] = d.x; P.q[8] = d.y; P.q[9] = d.z; P.q[10] = d.w;
                }
                float a[4], sr[4], sg[4], sb[4];
                prim_eval<4>(P, hx, hy, a, sr, sg, sb, lane);  // no curve: no shuffles inside
                float e = 0.0f;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float dr = clamp01(__fmul_rn(sr[j], a[j])) - hs[j].x;
                    const float dg = clamp01(__fmul_rn(sg[j], a[j])) - hs[j].y;
                    const float db = clamp01(__fmul_rn(sb[j], a[j])) - hs[j].z;
                    e = fmaf(dr, dr, fmaf(dg, dg, fmaf(db, db, e)));
                }
#pragma unroll
                for (int o = 8; o > 0; o >>= 1) e += __shfl_xor_sync(FULL, e, o);
                if (sub == 0 && c0 + half < m) st.partial[(off + s_slot[c]) * 4] = e;
            }
            half_done = true;
        }
    }

    const int group = warp / WPC, wig = warp % WPC;
    const float4* src = reinterpret_cast<const float4*>(st.src) + st.px_off[t];
    const float4* bg = reinterpret_cast<const float4*>(st.bg) + st.px_off[t];
    const int pbase = w.block * 1024 + wig * 32 * PPL;
    float fx[PPL], fy[PPL];
    float3 s[PPL], g[PPL];
#pragma unroll
    for (int j = 0; j < PPL; ++j) {
        const int p = pbase + j * 32 + lane;
        fx[j] = (float)(p % ts) + 0.5f;
        fy[j] = (float)(p / ts) + 0.5f;
        const float4 a = src[p];
        s[j] = make_float3(a.x, a.y, a.z);
        if (INIT) {
            g[j] = make_float3(0.0f, 0.0f, 0.0f);
        } else {
            const float4 b = bg[p];
            g[j] = make_float3(b.x, b.y, b.z);
        }
    }
    for (int c = group; !half_done && c < m; c += GROUPS) {
        Prep P;
        {
            const float4 a = s_prep[c][0], b = s_prep[c][1], cc = s_prep[c][2], d = s_prep[c][3];
            P.kind = __float_as_int(a.x);
            P.a = a.y; P.cr = a.z; P.cg = a.w; P.cb = b.x;
            P.q[0] = b.y; P.q[1] = b.z; P.q[2] = b.w;
            P.q[3] = cc.x; P.q[4] = cc.y; P.q[5] = cc.z; P.q[6] = cc.w;
            P.q[7] = d.x; P.q[8] = d.y; P.q[9] = d.z; P.q[10] = d.w;
        }
        float a[PPL], sr[PPL], sg[PPL], sb[PPL];
        if (P.kind == K_CURVE) {
            const Seg sg1 = lane_segment(P, lane);
            s_seg[warp][lane][0] = make_float4(sg1.ax, sg1.ay, sg1.vx, sg1.vy);
            s_seg[warp][lane][1] = make_float4(sg1.ux, sg1.uy, 0.0f, 0.0f);
            __syncwarp();
#pragma unroll
            for (int j = 0; j < PPL; ++j) {
                sr[j] = P.cr;
                sg[j] = P.cg;
                sb[j] = P.cb;
            }
            curve_alpha_smem<PPL>(P, s_seg[warp], fx, fy, a);
            __syncwarp();
        } else {
            prim_eval<PPL>(P, fx, fy, a, sr, sg, sb, lane);
        }
        float e = 0.0f;
#pragma unroll
        for (int j = 0; j < PPL; ++j) {
            const float dr = clamp01(INIT ? __fmul_rn(sr[j], a[j]) : blend(sr[j], a[j], g[j].x)) - s[j].x;
            const float dg = clamp01(INIT ? __fmul_rn(sg[j], a[j]) : blend(sg[j], a[j], g[j].y)) - s[j].y;
            const float db = clamp01(INIT ? __fmul_rn(sb[j], a[j]) : blend(sb[j], a[j], g[j].z)) - s[j].z;
            e = fmaf(dr, dr, fmaf(dg, dg, fmaf(db, db, e)));
        }
        e = warp_sum_f(e);
        if (WPC == 1) {
            if (lane == 0) st.partial[(off + s_slot[c]) * 4] = e;
        } else if (lane == 0) {
            red[c][wig] = e;
        }
    }
    if (st.work != nullptr) {
        // algorithmic ops of this CTA: every live candidate over the pixels it covers
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ops += __shfl_xor_sync(FULL, ops, o);
        if (lane == 0 && ops) atomicAdd(&st.work[1], ops);
    }
    if (WPC > 1) {
        __syncthreads();
        for (int c = threadIdx.x; c < m; c += blockDim.x) {
            float e = red[c][0];
#pragma unroll
            for (int k = 1; k < WPC; ++k) e += red[c][k];
            st.partial[(off + s_slot[c]) * 4 + w.block] = e;
        }
    }
    // candidate-pixels of this CTA: every live candidate over its 1024-pixel block or whole tile
    if (st.work != nullptr && threadIdx.x == 0)
        atomicAdd(&st.work[0], (unsigned long long)m * (unsigned long long)(WPC * 32 * PPL));
}

// One CTA per work item of the class (every item of the round's size class is launched; items of
// tiles that are not evaluated this round exit at once).
template <int PPL, int WPC, int MINB>
__global__ void __launch_bounds__(128, MINB) fit_score_kernel(WeftFitState st, const int* __restrict__ perm,
                                                        const WeftFitItem* __restrict__ items, int n_items,
                                                        int expect_min, int expect_max, bool mode_init) {
    __shared__ ScoreSmem<WPC> sm;
    if ((int)blockIdx.x >= n_items) return;
    if (mode_init)
        score_item<PPL, WPC, true>(st, perm, items[blockIdx.x], expect_min, expect_max, true, sm);
    else
        score_item<PPL, WPC, false>(st, perm, items[blockIdx.x], expect_min, expect_max, false, sm);
}

// Persistent form: a grid of about one wave of CTAs that pull the round's live items of the class
// from the work queue fit_queue_kernel built (q_items[0..q_len)), one item per pull.
template <int PPL, int WPC, int MINB>
__global__ void __launch_bounds__(128, MINB) fit_score_queue_kernel(WeftFitState st, const int* __restrict__ perm,
                                                              const WeftFitItem* __restrict__ items,
                                                              const int32_t* __restrict__ q_items,
                                                              const int32_t* q_len, int32_t* q_next, int expect_min,
                                                              int expect_max, bool mode_init) {
    __shared__ ScoreSmem<WPC> sm;
    __shared__ int s_i;
    if (threadIdx.x == 0) s_i = atomicAdd(q_next, 1);
    __syncthreads();
    const int len = *q_len;
    for (;;) {
        const int i = s_i;
        if (i >= len) break;
        // the next pull is issued now and its result consumed only after this item, so the
        // atomic's round trip overlaps the scoring
        int next = 0;
        if (threadIdx.x == 0) next = atomicAdd(q_next, 1);
        if (mode_init)
            score_item<PPL, WPC, true>(st, perm, items[q_items[i]], expect_min, expect_max, true, sm);
        else
            score_item<PPL, WPC, false>(st, perm, items[q_items[i]], expect_min, expect_max, false, sm);
        __syncthreads();  // every thread has read s_i and the item's shared buffers are free
        if (threadIdx.x == 0) s_i = next;
        __syncthreads();
    }
}

// The round's work queue: per size class, the items whose tile is evaluated this round and whose
// slot run starts inside the tile's filled slots (the others would exit at once), in any order
// (items write disjoint scratch).  ctl[c] counts class c's queue, ctl[3 + c] is its pull counter.
__global__ void fit_queue_kernel(WeftFitState st, const WeftFitItem* __restrict__ items8, int n8,
                                 const WeftFitItem* __restrict__ items16, int n16,
                                 const WeftFitItem* __restrict__ items32, int n32) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n8 + n16 + n32) return;
    const int c = i < n8 ? 0 : i < n8 + n16 ? 1 : 2;
    const int j = c == 0 ? i : c == 1 ? i - n8 : i - n8 - n16;
    const WeftFitItem w = (c == 0 ? items8 : c == 1 ? items16 : items32)[j];
    if (w.tile < 0 || w.tile >= st.n_tiles) {
        fit_report(WEFTK_E_ARG);
        return;
    }
    if (!(st.flags[w.tile] & WEFTK_TILE_EVAL) || w.first >= st.pool_cnt[w.tile]) return;
    const int base = c == 0 ? 0 : c == 1 ? n8 : n8 + n16;
    st.queue[base + atomicAdd(&st.queue_ctl[c], 1)] = j;
}

// ------------------------------------------------------------------ select / accept
__global__ void __launch_bounds__(128) fit_select_kernel(WeftFitState st, int mode, float lam_f, double lam_d) {
    const int t = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= st.n_tiles) return;
    if (!(st.flags[t] & WEFTK_TILE_EVAL)) return;
    const int ts = st.size[t], npix = ts * ts, nb = (npix + 1023) / 1024;
    const long long off = st.pool_off[t];
    const int cnt = st.pool_cnt[t];
    if (off < 0 || cnt < 0 || cnt > st.pool_cap[t] || off + cnt > st.n_slots) {
        if (lane == 0) fit_report(WEFTK_E_ARG);
        return;
    }
    const int base_bits = (mode == WEFTK_FIT_INIT) ? 8 : st.sel_bits[t];
    const float denom = (float)(3 * npix);
    float best = __int_as_float(0x7f800000);
    int bi = INT_MAX;
    for (int c = lane; c < cnt; c += 32) {
        const long long slot = off + c;
        if (!st.alive[slot]) continue;
        float sse = st.partial[slot * 4];
        for (int b = 1; b < nb; ++b) sse += st.partial[slot * 4 + b];
        const float mse = __fdiv_rn(sse, denom);
        const float obj = __fadd_rn(mse, __fmul_rn(lam_f, (float)(base_bits + prim_bits(st.kind[slot]))));
        if (obj < best || (obj == best && c < bi)) {
            best = obj;
            bi = c;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ob = __shfl_xor_sync(FULL, best, o);
        const int oi = __shfl_xor_sync(FULL, bi, o);
        if (ob < best || (ob == best && oi < bi)) {
            best = ob;
            bi = oi;
        }
    }
    if (bi == INT_MAX) return;
    const bool accept = (mode == WEFTK_FIT_INIT) || ((double)best < st.cur_obj[t]);
    if (!accept) return;
    const long long slot = off + bi;
    const int kind = st.kind[slot];
    if (lane == 0) {
        const int k = st.n_sel[t];
        if (k < st.cap_max) st.sel[(long long)t * st.cap_max + k] = bi;
        else fit_report(WEFTK_E_RANGE);
        st.n_sel[t] = k + 1;
        st.n_alive[t] -= 1;
        st.alive[slot] = 0;
        const int bits = base_bits + prim_bits(kind);
        st.sel_bits[t] = bits;
        if (mode == WEFTK_FIT_INIT) {
            float sse = st.partial[slot * 4];
            for (int b = 1; b < nb; ++b) sse += st.partial[slot * 4 + b];
            st.cur_obj[t] = (double)__fdiv_rn(sse, denom) + lam_d * (double)bits;
        } else {
            st.cur_obj[t] = (double)best;
        }
        st.flags[t] |= WEFTK_TILE_IMPROVED;
        atomicAdd(&st.status[1], 1);
    }
    // Composite the accepted candidate into the tile's bg (a fit without one runs no round
    // after its init round, so nothing would read it).
    if (st.bg == nullptr) return;
    const Prep P = load_prep(st.prep, slot);
    float4* bgp = reinterpret_cast<float4*>(st.bg) + st.px_off[t];
    constexpr int U = 4;
    for (int base = 0; base < npix; base += 32 * U) {
        float fx[U], fy[U], a[U], sr[U], sg[U], sb[U];
        float4 g[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const int p = min(base + j * 32 + lane, npix - 1);
            fx[j] = (float)(p % ts) + 0.5f;
            fy[j] = (float)(p / ts) + 0.5f;
            g[j] = bgp[p];
        }
        prim_eval<U>(P, fx, fy, a, sr, sg, sb, lane);
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const int p = base + j * 32 + lane;
            if (p < npix)
                bgp[p] = make_float4(blend(sr[j], a[j], g[j].x), blend(sg[j], a[j], g[j].y),
                                     blend(sb[j], a[j], g[j].z), 0.0f);
        }
    }
}

// Register-resident FMA loop for measuring the FP32 pipe: 8 independent chains per thread.
__global__ void __launch_bounds__(256) fp32_peak_kernel(float* out, int iters, float a, float b) {
    float v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = (float)(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = fmaf(v[k], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += v[k];
    if (s == 12345.678f) out[threadIdx.x] = s;  // keeps the loop live; practically never taken
}

struct FitTiming {
    bool enabled = false;
    bool pending = false;
    cudaEvent_t start = nullptr, stop = nullptr;
    double ms = 0.0;
    int rounds = 0;
};
static FitTiming g_timing;

static int timing_collect() {
    if (!g_timing.pending) return WEFTK_OK;
    WEFTK_CUDA(cudaEventSynchronize(g_timing.stop));
    float ms = 0.0f;
    WEFTK_CUDA(cudaEventElapsedTime(&ms, g_timing.start, g_timing.stop));
    g_timing.ms += ms;
    g_timing.rounds += 1;
    g_timing.pending = false;
    return WEFTK_OK;
}

}  // namespace weftk

using namespace weftk;

// ---------------------------------------------------------------- allocation-free round
// Scoring scratch for weftk_fit_round_static: a fixed array in device memory, so
// that entry point never allocates.  Host code must not use the symbol as a
// pointer (it is a host-side stand-in); the device address comes from
// cudaGetSymbolAddress, looked up once per device.
static __device__ __align__(256) float g_fit_static_scratch[WEFTK_FIT_STATIC_SCRATCH_FLOATS];
static std::mutex g_static_mu;
static float* g_static_ptr[64] = {nullptr};

static int static_scratch_for_current_device(float** out) {
    int dev = 0;
    WEFTK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(WEFTK_E_RANGE, "fit_round_static: device index beyond 63");
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_fit_static_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_fit_static_scratch)");
        g_static_ptr[dev] = static_cast<float*>(p);
    }
    *out = g_static_ptr[dev];
    return WEFTK_OK;
}

extern "C" int weftk_fit_timing(int enable, double* score_ms, int* n_rounds) {
    int rc = timing_collect();
    if (rc) return rc;
    if (enable && !g_timing.start) {
        WEFTK_CUDA(cudaEventCreate(&g_timing.start));
        WEFTK_CUDA(cudaEventCreate(&g_timing.stop));
    }
    g_timing.enabled = enable != 0;
    if (score_ms) *score_ms = g_timing.ms;
    if (n_rounds) *n_rounds = g_timing.rounds;
    g_timing.ms = 0.0;
    g_timing.rounds = 0;
    return WEFTK_OK;
}

extern "C" int weftk_measure_fp32_peak(double* gflops) {
    WEFTK_REQUIRE(gflops, "measure_fp32_peak: null pointer");
    int dev = 0, sms = 0;
    WEFTK_CUDA(cudaGetDevice(&dev));
    WEFTK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    float* out = nullptr;
    WEFTK_CUDA(cudaMalloc(&out, 256 * sizeof(float)));
    cudaEvent_t a, b;
    WEFTK_CUDA(cudaEventCreate(&a));
    WEFTK_CUDA(cudaEventCreate(&b));
    const int blocks = sms * 8, iters = 1 << 15;
    fp32_peak_kernel<<<blocks, 256>>>(out, 256, 1.0000001f, 1e-7f);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 5; ++r) {
        WEFTK_CUDA(cudaEventRecord(a));
        fp32_peak_kernel<<<blocks, 256>>>(out, iters, 1.0000001f, 1e-7f);
        WEFTK_CUDA(cudaEventRecord(b));
        WEFTK_CUDA(cudaEventSynchronize(b));
        float ms = 0.0f;
        WEFTK_CUDA(cudaEventElapsedTime(&ms, a, b));
        best = ms < best ? ms : best;
    }
    WEFTK_CUDA(cudaGetLastError());
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    *gflops = 2.0 * 8.0 * (double)iters * 256.0 * (double)blocks / (best * 1e-3) / 1e9;
    return WEFTK_OK;
}

// One CTA per tile: the tile's state, selection row, slots and composite pixels.
__global__ void fit_reset_kernel(WeftFitState st, const int* __restrict__ init_cnt) {
    const int t = blockIdx.x;
    if (t >= st.n_tiles) return;
    if (t == 0 && threadIdx.x == 0 && st.work != nullptr) {
        st.work[0] = 0;
        st.work[1] = 0;
    }
    if (threadIdx.x == 0) {
        st.pool_cnt[t] = init_cnt[t];
        st.n_alive[t] = 0;
        st.n_sel[t] = 0;
        st.sel_bits[t] = 8;
        st.flags[t] = 0;
        st.cur_obj[t] = 0.0;
    }
    for (int i = threadIdx.x; i < st.cap_max; i += blockDim.x) st.sel[(size_t)t * st.cap_max + i] = -1;
    const long long off = st.pool_off[t];
    for (int i = threadIdx.x; i < st.pool_cap[t]; i += blockDim.x) st.alive[off + i] = 0;
    const int ts = st.size[t];
    if (st.bg == nullptr) return;
    float4* bg = reinterpret_cast<float4*>(st.bg) + st.px_off[t];
    for (int i = threadIdx.x; i < ts * ts; i += blockDim.x) bg[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

__global__ void fit_moments_kernel(WeftFitState st, double* __restrict__ out) {
    __shared__ double red[6][4];
    const int t = blockIdx.x;
    if (t >= st.n_tiles) return;
    const int ts = st.size[t], n = ts * ts, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float4* src = reinterpret_cast<const float4*>(st.src) + st.px_off[t];
    double a[6] = {0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float4 v = src[i];
        a[0] += v.x;
        a[1] += v.y;
        a[2] += v.z;
        a[3] += (double)v.x * v.x;
        a[4] += (double)v.y * v.y;
        a[5] += (double)v.z * v.z;
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_xor_sync(FULL, a[k], o);
        if (lane == 0) red[k][warp] = a[k];
    }
    __syncthreads();
    if (threadIdx.x < 6) out[(size_t)t * 6 + threadIdx.x] = red[threadIdx.x][0] + red[threadIdx.x][1] +
                                                             red[threadIdx.x][2] + red[threadIdx.x][3];
}

extern "C" int weftk_fit_moments(const WeftFitState* st, double* d_moments, void* stream) {
    WEFTK_REQUIRE(st && d_moments, "fit_moments: null argument");
    if (st->n_tiles == 0) return WEFTK_OK;
    fit_moments_kernel<<<st->n_tiles, 128, 0, (cudaStream_t)stream>>>(*st, d_moments);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}

extern "C" int weftk_fit_reset(const WeftFitState* st, const int32_t* d_init_cnt, void* stream) {
    WEFTK_REQUIRE(st && d_init_cnt, "fit_reset: null argument");
    if (st->n_tiles == 0) return WEFTK_OK;
    fit_reset_kernel<<<st->n_tiles, 128, 0, (cudaStream_t)stream>>>(*st, d_init_cnt);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}

extern "C" int weftk_fit_prepare(const WeftFitState* st, const int32_t* d_first_new, void* stream) {
    WEFTK_REQUIRE(st && d_first_new, "fit_prepare: null argument");
    if (st->n_tiles == 0) return WEFTK_OK;
    fit_prepare_kernel<<<st->n_tiles, 128, 0, (cudaStream_t)stream>>>(*st, d_first_new);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}

extern "C" int weftk_fit_round_static(const WeftFitState* st, int mode, double lambda, double complex_threshold,
                                      const int32_t* d_perm, const WeftFitItem* d_items8, int n_items8,
                                      const WeftFitItem* d_items16, int n_items16, const WeftFitItem* d_items32,
                                      int n_items32, void* stream) {
    WEFTK_REQUIRE(st, "fit_round_static: null state");
    if (st->n_slots < 0 || st->n_slots > (long long)WEFTK_FIT_STATIC_SCRATCH_FLOATS / 4)
        return fail(WEFTK_E_RANGE, "fit_round_static: " + std::to_string((long long)st->n_slots) +
                                       " candidate slots need more than the " +
                                       std::to_string(WEFTK_FIT_STATIC_SCRATCH_FLOATS) +
                                       "-float static scratch (at most " +
                                       std::to_string(WEFTK_FIT_STATIC_SCRATCH_FLOATS / 4) + " slots)");
    float* scratch = nullptr;
    int rc = static_scratch_for_current_device(&scratch);
    if (rc) return rc;
    WeftFitState local = *st;
    local.partial = scratch;
    return weftk_fit_round(&local, mode, lambda, complex_threshold, d_perm, d_items8, n_items8, d_items16, n_items16,
                           d_items32, n_items32, stream);
}

// Scoring variants per size class.  A class's variants cover the same pixels per candidate pass
// (64 for 8-px tiles, 256 for 16-px tiles, one 1024-pixel block for 32/64-px tiles) with a
// different split over lanes and warps, or a different register budget.
static_assert(sizeof(WeftFitState) == 224, "WeftFitState layout is part of the C ABI");

struct ScoreShape {
    int ppl, wpc, minb;
};
static const ScoreShape kShapes[3][WEFTK_FIT_VARIANTS] = {
    {{2, 1, 7}, {2, 1, 8}, {1, 2, 8}},
    {{8, 1, 4}, {4, 2, 6}, {2, 4, 8}},
    {{8, 4, 4}, {8, 4, 3}, {8, 4, 5}},
};

// mode of the round being enqueued (the class launchers' extra argument)
static thread_local bool g_mode_init = false;

// queue of the class being launched (set while weftk_fit_round enqueues a queue-driven round)
static thread_local int g_queue_class = -1;
static thread_local int g_queue_base = 0;
static thread_local int g_sms = 148;

template <int PPL, int WPC, int MINB>
static void launch_score(const WeftFitState& st, const int* perm, const WeftFitItem* items, int n, int lo, int hi,
                         cudaStream_t s) {
    if (g_queue_class < 0) {
        fit_score_kernel<PPL, WPC, MINB><<<n, 128, 0, s>>>(st, perm, items, n, lo, hi, g_mode_init);
        return;
    }
    const int c = g_queue_class;
    const int grid = std::min(n, g_sms * MINB);
    fit_score_queue_kernel<PPL, WPC, MINB><<<grid, 128, 0, s>>>(st, perm, items, st.queue + g_queue_base,
                                                                 st.queue_ctl + c, st.queue_ctl + 3 + c, lo, hi,
                                                                 g_mode_init);
}

static void launch_score_class8(int v, const WeftFitState& st, const int* perm, const WeftFitItem* it, int n,
                                cudaStream_t s) {
    if (v == 1) launch_score<2, 1, 8>(st, perm, it, n, 8, 8, s);
    else if (v == 2) launch_score<1, 2, 8>(st, perm, it, n, 8, 8, s);
    else launch_score<2, 1, 7>(st, perm, it, n, 8, 8, s);
}

static void launch_score_class16(int v, const WeftFitState& st, const int* perm, const WeftFitItem* it, int n,
                                 cudaStream_t s) {
    if (v == 1) launch_score<4, 2, 6>(st, perm, it, n, 16, 16, s);
    else if (v == 2) launch_score<2, 4, 8>(st, perm, it, n, 16, 16, s);
    else launch_score<8, 1, 4>(st, perm, it, n, 16, 16, s);
}

static void launch_score_class32(int v, const WeftFitState& st, const int* perm, const WeftFitItem* it, int n,
                                 cudaStream_t s) {
    if (v == 1) launch_score<8, 4, 3>(st, perm, it, n, 32, 64, s);
    else if (v == 2) launch_score<8, 4, 5>(st, perm, it, n, 32, 64, s);
    else launch_score<8, 4, 4>(st, perm, it, n, 32, 64, s);
}

extern "C" int weftk_fit_variant(int size_class, int variant, int* pixels_per_lane, int* warps_per_candidate,
                                 int* ctas_per_sm) {
    const int c = size_class == 8 ? 0 : size_class == 16 ? 1 : size_class == 32 ? 2 : -1;
    WEFTK_REQUIRE(c >= 0 && variant >= 0 && variant < WEFTK_FIT_VARIANTS, "fit_variant: no such class or variant");
    if (pixels_per_lane) *pixels_per_lane = kShapes[c][variant].ppl;
    if (warps_per_candidate) *warps_per_candidate = kShapes[c][variant].wpc;
    if (ctas_per_sm) *ctas_per_sm = kShapes[c][variant].minb;
    return WEFTK_OK;
}

// Control block of the device-driven fit for the round being enqueued (host thread state:
// set only while weftk_fit_run enqueues its rounds).
static thread_local int* g_round_ctl = nullptr;

int launch_fit_reseed(const WeftFitState& st, const int* gate, cudaStream_t stream);

extern "C" int weftk_fit_run(const WeftFitState* st, int max_rounds, double lambda, double complex_threshold,
                             const int32_t* d_perm, const WeftFitItem* d_items8, int n_items8,
                             const WeftFitItem* d_items16, int n_items16, const WeftFitItem* d_items32,
                             int n_items32, int32_t* d_ctl, void* stream) {
    WEFTK_REQUIRE(st && d_ctl && max_rounds >= 0, "fit_run: bad arguments");
    WEFTK_REQUIRE(!g_timing.enabled, "fit_run: scoring timing is host-synchronised; disable it first");
    cudaStream_t s = (cudaStream_t)stream;
    WEFTK_CUDA(cudaMemsetAsync(d_ctl, 0, 4 * sizeof(int32_t), s));
    int rc = weftk_fit_round(st, WEFTK_FIT_INIT, lambda, complex_threshold, d_perm, d_items8, n_items8, d_items16,
                             n_items16, d_items32, n_items32, stream);
    for (int r = 0; !rc && r < max_rounds; ++r) {
        g_round_ctl = d_ctl;
        rc = weftk_fit_round(st, WEFTK_FIT_ROUND, lambda, complex_threshold, d_perm, d_items8, n_items8, d_items16,
                             n_items16, d_items32, n_items32, stream);
        g_round_ctl = nullptr;
        if (rc) break;
        fit_control_kernel<<<1, 32, 0, s>>>(st->status, d_ctl);
        rc = launch_fit_reseed(*st, d_ctl + 2, s);
    }
    if (!rc) WEFTK_CUDA(cudaGetLastError());
    return rc;
}

// Side streams of the current device for the calling host thread: the 16-px and 32/64-px classes'
// scoring launches run beside the 8-px class's (forked from and joined back into the caller's
// stream, which a CUDA graph capture follows).  Created on first use, kept for the process.
struct ClassStreams {
    cudaStream_t s[2] = {nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
};

static int class_streams(ClassStreams** out) {
    thread_local std::map<int, ClassStreams> per_device;
    int dev = 0;
    WEFTK_CUDA(cudaGetDevice(&dev));
    ClassStreams& cs = per_device[dev];
    if (cs.fork == nullptr) {
        for (int i = 0; i < 2; ++i) {
            WEFTK_CUDA(cudaStreamCreateWithFlags(&cs.s[i], cudaStreamNonBlocking));
            WEFTK_CUDA(cudaEventCreateWithFlags(&cs.join[i], cudaEventDisableTiming));
        }
        WEFTK_CUDA(cudaEventCreateWithFlags(&cs.fork, cudaEventDisableTiming));
    }
    *out = &cs;
    return WEFTK_OK;
}

extern "C" int weftk_fit_round(const WeftFitState* st, int mode, double lambda, double complex_threshold,
                               const int32_t* d_perm, const WeftFitItem* d_items8, int n_items8,
                               const WeftFitItem* d_items16, int n_items16, const WeftFitItem* d_items32,
                               int n_items32, void* stream) {
    WEFTK_REQUIRE(st && d_perm, "fit_round: null argument");
    WEFTK_REQUIRE(mode == WEFTK_FIT_INIT || mode == WEFTK_FIT_ROUND, "fit_round: bad mode");
    WEFTK_REQUIRE(mode == WEFTK_FIT_INIT || st->bg != nullptr, "fit_round: a greedy round needs the composite (bg)");
    WEFTK_REQUIRE(n_items8 >= 0 && n_items16 >= 0 && n_items32 >= 0, "fit_round: negative item count");
    for (int c = 0; c < 3; ++c)
        WEFTK_REQUIRE(st->variant[c] >= 0 && st->variant[c] < WEFTK_FIT_VARIANTS, "fit_round: bad scoring variant");
    if (st->n_tiles == 0) return WEFTK_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int nt = st->n_tiles;
    WEFTK_CUDA(cudaMemsetAsync(st->status, 0, 4 * sizeof(int32_t), s));
    fit_begin_kernel<<<ceil_div(nt, 256), 256, 0, s>>>(*st, mode, g_round_ctl);
    if (g_timing.enabled) {
        int rc = timing_collect();
        if (rc) return rc;
        WEFTK_CUDA(cudaEventRecord(g_timing.start, s));
    }
    g_mode_init = mode == WEFTK_FIT_INIT;
    const bool queued = st->queue != nullptr && st->queue_ctl != nullptr;
    if (queued) {
        int dev = 0;
        WEFTK_CUDA(cudaGetDevice(&dev));
        WEFTK_CUDA(cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev));
        WEFTK_CUDA(cudaMemsetAsync(st->queue_ctl, 0, 8 * sizeof(int32_t), s));
        const int total = n_items8 + n_items16 + n_items32;
        if (total > 0)
            fit_queue_kernel<<<ceil_div(total, 256), 256, 0, s>>>(*st, d_items8, n_items8, d_items16, n_items16,
                                                                  d_items32, n_items32);
    }
    // the size classes score disjoint tiles: the 16-px and 32/64-px classes run on side streams
    // beside the 8-px class (not while the scoring launches are being timed)
    ClassStreams* cs = nullptr;
    const bool side = !g_timing.enabled && (n_items16 > 0 || n_items32 > 0) && n_items8 + n_items16 + n_items32 > 0;
    if (side) {
        int rc = class_streams(&cs);
        if (rc) return rc;
        WEFTK_CUDA(cudaEventRecord(cs->fork, s));
        for (int i = 0; i < 2; ++i) WEFTK_CUDA(cudaStreamWaitEvent(cs->s[i], cs->fork, 0));
    }
    if (n_items32) {
        g_queue_class = queued ? 2 : -1;
        g_queue_base = n_items8 + n_items16;
        launch_score_class32(st->variant[2], *st, d_perm, d_items32, n_items32, side ? cs->s[1] : s);
    }
    if (n_items16) {
        g_queue_class = queued ? 1 : -1;
        g_queue_base = n_items8;
        launch_score_class16(st->variant[1], *st, d_perm, d_items16, n_items16, side ? cs->s[0] : s);
    }
    if (n_items8) {
        g_queue_class = queued ? 0 : -1;
        g_queue_base = 0;
        launch_score_class8(st->variant[0], *st, d_perm, d_items8, n_items8, s);
    }
    g_queue_class = -1;
    if (side) {
        WEFTK_CUDA(cudaGetLastError());
        for (int i = 0; i < 2; ++i) {
            WEFTK_CUDA(cudaEventRecord(cs->join[i], cs->s[i]));
            WEFTK_CUDA(cudaStreamWaitEvent(s, cs->join[i], 0));
        }
    }
    if (g_timing.enabled) {
        WEFTK_CUDA(cudaEventRecord(g_timing.stop, s));
        g_timing.pending = true;
    }
    fit_select_kernel<<<ceil_div(nt, 4), 128, 0, s>>>(*st, mode, (float)lambda, lambda);
    fit_end_kernel<<<ceil_div(nt, 256), 256, 0, s>>>(*st, mode, complex_threshold);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}
