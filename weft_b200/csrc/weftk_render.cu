// weftk_render.cu — generic per-eval scoring (batch_tile_objective replacement) and the
// decoder's primitive walk (decode_tile_pixels / render_scene_adaptive replacement).
//
// Generic scoring: one warp per eval; each lane owns 4 pixels of a 128-pixel chunk and
// composites the whole stack for them in registers; the per-lane squared error of a
// chunk is summed in float32 and accumulated in float64; one warp reduction per eval.
//
// Decode walk: work items of tile rows, one warp per item, a persistent one-wave grid.
// Lone constant tiles (almost every tile of a fit at q75) are written as whole 16-byte
// slots of their rows, other tiles per 4-pixel group with the stack composited in
// registers.  Output is float32 HWC.
#include <cuda_runtime.h>

#include <algorithm>

#include "weftk_common.cuh"
#include "weftk_prim.cuh"

namespace weftk {

__device__ int g_device_status = 0;  // first error code a kernel hit (0 = none)

__device__ __forceinline__ void report(int code) { atomicCAS(&g_device_status, 0, code); }

__device__ __forceinline__ WeftPrim load_prim(const WeftPrim* p) {
    WeftPrim r;
    const float* f = reinterpret_cast<const float*>(p);
    r.kind = __ldg(reinterpret_cast<const int*>(p));
#pragma unroll
    for (int i = 0; i < 7; ++i) r.geom[i] = __ldg(f + 1 + i);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        r.color0[i] = __ldg(f + 8 + i);
        r.color1[i] = __ldg(f + 11 + i);
    }
    r.alpha = __ldg(f + 14);
    return r;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

constexpr int SCORE_PPL = 4;

__global__ void __launch_bounds__(256) score_evals_kernel(const WeftEval* __restrict__ evals, int n_evals,
                                                          const WeftPrim* __restrict__ prims,
                                                          const float* __restrict__ tiles, float* __restrict__ out,
                                                          float off) {
    const int warp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= n_evals) return;
    const int4 e = __ldg(reinterpret_cast<const int4*>(evals) + warp);
    const int ts = e.w, npix = ts * ts;
    if (ts <= 0 || ts > 64 || e.y < 0) {
        if (lane == 0) {
            out[warp] = __int_as_float(0x7fc00000);
            report(WEFTK_E_ARG);
        }
        return;
    }
    const float* src = tiles + e.z;
    double acc = 0.0;
    for (int base = 0; base < npix; base += 32 * SCORE_PPL) {
        float fx[SCORE_PPL], fy[SCORE_PPL], cr[SCORE_PPL], cg[SCORE_PPL], cb[SCORE_PPL];
#pragma unroll
        for (int j = 0; j < SCORE_PPL; ++j) {
            int p = base + j * 32 + lane;
            fx[j] = (float)(p % ts) + off;
            fy[j] = (float)(p / ts) + off;
            cr[j] = cg[j] = cb[j] = 0.0f;
        }
        for (int k = 0; k < e.y; ++k) {
            WeftPrim P = load_prim(prims + e.x + k);
            Prep pr = prep_prim(P);
            if (pr.kind == K_BICUBIC) pr.kind = K_SKIP;  // the scorer never evaluates bicubic grids
            float a[SCORE_PPL], sr[SCORE_PPL], sg[SCORE_PPL], sb[SCORE_PPL];
            prim_eval<SCORE_PPL>(pr, fx, fy, a, sr, sg, sb, lane);
#pragma unroll
            for (int j = 0; j < SCORE_PPL; ++j) {
                cr[j] = blend(sr[j], a[j], cr[j]);
                cg[j] = blend(sg[j], a[j], cg[j]);
                cb[j] = blend(sb[j], a[j], cb[j]);
            }
        }
        float part = 0.0f;
#pragma unroll
        for (int j = 0; j < SCORE_PPL; ++j) {
            int p = base + j * 32 + lane;
            if (p < npix) {
                const float* s = src + 3 * p;
                float dr = clamp01(cr[j]) - __ldg(s), dg = clamp01(cg[j]) - __ldg(s + 1),
                      db = clamp01(cb[j]) - __ldg(s + 2);
                part = fmaf(dr, dr, fmaf(dg, dg, fmaf(db, db, part)));
            }
        }
        acc += (double)part;
    }
    acc = warp_sum(acc);
    if (lane == 0) out[warp] = (float)(acc / (double)(3 * npix));
}

constexpr int DEC_PPL = 4;
constexpr int DEC_THREADS = 128;
static_assert(DEC_PPL == 4, "a pixel group is 4 output pixels (48 bytes, three 16-byte slots)");
constexpr int MAX_TILE_PRIMS = 48;

// Sole-bicubic tile: float64 Bernstein evaluation of the 4x4x3 control grid at sample
// (lx, ly) of a side x side grid (src/weft/bicubic.py:106-115), clipped.  Kept out of
// line so the common path's register budget is not set by this rare one.
__device__ __noinline__ void bicubic_pixel(const float* ctrl, int lx, int ly, int side, float* rgb) {
    double by[4], bx[4];
    bernstein4(ly, side, by);
    bernstein4(lx, side, bx);
    double o[3] = {0.0, 0.0, 0.0};
    for (int r = 0; r < 4; ++r) {
        for (int ch = 0; ch < 3; ++ch) {
            double m = 0.0;
            for (int c = 0; c < 4; ++c) m = fma((double)ctrl[(r * 4 + c) * 3 + ch], bx[c], m);
            o[ch] = fma(by[r], m, o[ch]);
        }
    }
    rgb[0] = clamp01((float)o[0]);
    rgb[1] = clamp01((float)o[1]);
    rgb[2] = clamp01((float)o[2]);
}

// Work items: (tile, first row).  An item covers rows [first, first + R) of the tile's
// target rect, R = max(1, WEFTK_DECODE_ITEM_GROUPS / G), where G is the number of
// 4-pixel groups (aligned to output x multiples of 4) a rect row touches; rows outside
// the image are skipped.  Each item is rendered by ONE warp: the warp stages its tile's
// primitives in its own slice of shared memory and never waits on the rest of the CTA,
// so every resident warp works on a different item.  A persistent grid of one wave
// (every CTA resident) walks the list in rounds: in round r warp w takes item
// r * n_warps + w when r is even and r * n_warps + n_warps - 1 - w when r is odd, so
// with the items in descending cost order every warp gets a similar share of the work
// (the warps' finishing times, not their item counts, set the kernel's duration).  A
// warp fetches the records of its next DEC_BATCH items at once (item, descriptor and
// first primitive, one item per lane), so the dependent-load chain item -> descriptor
// -> primitive is paid once per batch instead of once per item.
//
// Three ways to write an item's rows:
//  * a lone constant layer without a RES1 grid is one colour: every lane stores whole
//    16-byte slots of the row's float run (slot s holds channels s, s+1, s+2, s mod 3 of
//    the colour), so a warp's stores are contiguous and fill every 32-byte sector they
//    touch; the at most three floats at each end of a row that share a slot with the
//    neighbouring tile are stored one by one;
//  * a lone constant layer with a RES1 grid: the same 16-byte slots, each the colour plus
//    the bilinear grid at its two pixels (no primitive evaluation);
//  * anything else: per 4-pixel group, the whole stack composited in registers.
// Which tile writes a pixel, and with what arithmetic, is the same on every path, so the
// image does not depend on the order or the path the items take.
constexpr int DEC_ITEM_GROUPS = WEFTK_DECODE_ITEM_GROUPS;
constexpr int DEC_WARPS = DEC_THREADS / 32;
constexpr int DEC_MINB = 4;  // resident CTAs per SM the register budget is set for
constexpr int DEC_BATCH = 8;

__device__ __forceinline__ int floor_div4(int v) { return v >= 0 ? (v >> 2) : -((-v + 3) >> 2); }

// c[p mod 3] of (c0, c1, c2) for p in 0..2
__device__ __forceinline__ float sel3(int p, float c0, float c1, float c2) { return p == 0 ? c0 : (p == 1 ? c1 : c2); }

// Rows [r0, r1) of a rect filled with one colour: the rect's columns [xa, xb) (inside the
// image) are the floats [3 xa, 3 xb) of each row.  Requires 3 W to be a multiple of 4 and
// 16-byte aligned rows, so that a row's 16-byte slot s holds the colour channels
// s, s+1, s+2, s (mod 3) whatever the row.
__device__ __forceinline__ void fill_rows(float* __restrict__ out, size_t row_floats, int gy0, int r0, int r1, int xa,
                                          int xb, float c0, float c1, float c2, int lane) {
    const int fa = 3 * xa, fb = 3 * xb;
    const int sa = (fa + 3) >> 2;             // first slot inside the run
    const int sb = max(sa, fb >> 2);          // one past the last slot inside the run
    const int n4 = sb - sa;
    if (n4 > 0) {
        if (n4 < 32) {
            // several rows per warp step: lane -> (row rr, slot cc), the same slot every row
            const int rs = 32 / n4;
            const int rr = lane / n4, cc = lane - rr * n4;
            if (rr < rs && r0 + rr < r1) {
                const int p = (sa + cc) % 3;
                const float v0 = sel3(p, c0, c1, c2);
                const float4 v = make_float4(v0, sel3(p, c1, c2, c0), sel3(p, c2, c0, c1), v0);
                float4* dst = reinterpret_cast<float4*>(out + (size_t)(gy0 + r0 + rr) * row_floats) + sa + cc;
                const size_t step = (size_t)rs * (row_floats >> 2);
                for (int r = r0 + rr; r < r1; r += rs, dst += step) *dst = v;
            }
        } else {
            const int p = (sa + lane) % 3;
            const float v0 = sel3(p, c0, c1, c2);
            const float4 v = make_float4(v0, sel3(p, c1, c2, c0), sel3(p, c2, c0, c1), v0);
            float4* dst = reinterpret_cast<float4*>(out + (size_t)(gy0 + r0) * row_floats) + sa;
            const size_t step = row_floats >> 2;
            for (int r = r0; r < r1; ++r, dst += step) {
                float4 u = v;
                for (int cc = lane; cc < n4; cc += 32) {
                    dst[cc] = u;
                    u = make_float4(u.z, u.x, u.y, u.z);  // 32 slots on: channels advance by 2 (mod 3)
                }
            }
        }
    }
    // the floats before the first and after the last whole slot: lane pairs per row
    const int head_end = min(4 * sa, fb), tail_begin = max(4 * sb, head_end);
    if (head_end > fa || fb > tail_begin) {
        const int f_lo = (lane & 1) ? tail_begin : fa, f_hi = (lane & 1) ? fb : head_end;
        for (int r = r0 + (lane >> 1); r < r1; r += 16) {
            float* rowp = out + (size_t)(gy0 + r) * row_floats;
            for (int f = f_lo; f < f_hi; ++f) rowp[f] = sel3(f % 3, c0, c1, c2);
        }
    }
}

// Bilinear 4x4 RES1 grid coordinate at a pixel centre of a side-h grid, edge-clamped
// (src/weft/render.py:474-515): cell index i0, i1 = min(i0 + 1, 3) and weight t.
__device__ __forceinline__ void res1_axis(int l, float gscale, int& i0, int& i1, float& t) {
    const float g = fminf(fmaxf(__fsub_rn(__fmul_rn((float)l + 0.5f, gscale), 0.5f), 0.0f), 3.0f);
    i0 = (int)floorf(g);
    i1 = min(i0 + 1, 3);
    t = __fsub_rn(g, (float)i0);
}

// x then y interpolation of one channel, in the reference's order
__device__ __forceinline__ float lerp_rn(float a, float b, float t) {
    return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, t)), __fmul_rn(b, t));
}

// Rows [r0, r1) of a lone constant layer with a RES1 grid: the base colour (c0, c1, c2)
// (RES0 added, clamped) plus the grid's bilinear value, clamped, with the slot layout of
// fill_rows (requires 3 W a multiple of 4 and 16-byte aligned rows).  A 16-byte slot
// holds parts of two pixels; a lane keeps the same slot over the rows it walks, so the
// slot's x interpolation weights are set once, and the x-interpolated grid rows once per
// grid row the walk enters; per row only the y blend remains.
__device__ __forceinline__ void fill_rows_res1(float* __restrict__ out, size_t row_floats, int gy0, int r0, int r1,
                                               int x0, int w, int xa, int xb, float gscale,
                                               const float* __restrict__ grid, float c0, float c1, float c2,
                                               int lane) {
    const int fa = 3 * xa, fb = 3 * xb;
    const int sa = (fa + 3) >> 2;
    const int sb = max(sa, fb >> 2);
    const int n4 = sb - sa;
    const float base[3] = {c0, c1, c2};
    if (n4 > 0) {
        const int per_row = n4 < 32 ? n4 : 32;
        const int rs = n4 < 32 ? 32 / n4 : 1;
        const int rr = lane / per_row, cl = lane - rr * per_row;
        if (rr < rs && r0 + rr < r1) {
            for (int col0 = 0; col0 < n4; col0 += per_row) {
                const int cc = col0 + cl;
                if (cc >= n4) break;
                const int S = sa + cc;        // the slot's floats 4S .. 4S + 3
                const int X = (4 * S) / 3;    // its first pixel; the second is X + 1
                const int p = S % 3;          // channel of the slot's first float
                int rx0[2], rx1[2];
                float wx[2];
#pragma unroll
                for (int j = 0; j < 2; ++j) res1_axis(min(max(X + j - x0, 0), w - 1), gscale, rx0[j], rx1[j], wx[j]);
                int ch[4], px[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    ch[k] = (p + k) % 3;
                    px[k] = (p + k) / 3;
                }
                float top[4], bot[4];
                int ry_cached = -1;
                float4* dst = reinterpret_cast<float4*>(out + (size_t)(gy0 + r0 + rr) * row_floats) + S;
                const size_t step = (size_t)rs * (row_floats >> 2);
                for (int r = r0 + rr; r < r1; r += rs, dst += step) {
                    int ry0, ry1;
                    float wy;
                    res1_axis(r, gscale, ry0, ry1, wy);
                    if (ry0 != ry_cached) {
                        ry_cached = ry0;
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const int a0 = rx0[px[k]], a1 = rx1[px[k]];
                            top[k] = lerp_rn(grid[(ry0 * 4 + a0) * 3 + ch[k]], grid[(ry0 * 4 + a1) * 3 + ch[k]],
                                             wx[px[k]]);
                            bot[k] = lerp_rn(grid[(ry1 * 4 + a0) * 3 + ch[k]], grid[(ry1 * 4 + a1) * 3 + ch[k]],
                                             wx[px[k]]);
                        }
                    }
                    float v[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k) v[k] = clamp01(base[ch[k]] + lerp_rn(top[k], bot[k], wy));
                    *dst = make_float4(v[0], v[1], v[2], v[3]);
                }
            }
        }
    }
    // the floats before the first and after the last whole slot: lane pairs per row
    const int head_end = min(4 * sa, fb), tail_begin = max(4 * sb, head_end);
    if (head_end > fa || fb > tail_begin) {
        const int f_lo = (lane & 1) ? tail_begin : fa, f_hi = (lane & 1) ? fb : head_end;
        for (int r = r0 + (lane >> 1); r < r1; r += 16) {
            int ry0, ry1;
            float wy;
            res1_axis(r, gscale, ry0, ry1, wy);
            float* rowp = out + (size_t)(gy0 + r) * row_floats;
            for (int f = f_lo; f < f_hi; ++f) {
                const int c = f % 3;
                int a0, a1;
                float wxf;
                res1_axis(min(max(f / 3 - x0, 0), w - 1), gscale, a0, a1, wxf);
                const float t = lerp_rn(grid[(ry0 * 4 + a0) * 3 + c], grid[(ry0 * 4 + a1) * 3 + c], wxf);
                const float b = lerp_rn(grid[(ry1 * 4 + a0) * 3 + c], grid[(ry1 * 4 + a1) * 3 + c], wxf);
                rowp[f] = clamp01(base[c] + lerp_rn(t, b, wy));
            }
        }
    }
}

__device__ __forceinline__ bool desc_ok(const WeftTileDecodeDesc& d) {
    return d.prim_count >= 0 && d.prim_count <= MAX_TILE_PRIMS && d.target_w > 0 && d.target_h > 0 &&
           d.target_w <= 8192 && d.target_h <= 8192 && d.source_size > 0;
}

// One work item (tile rows) rendered by one warp; p0 is the tile's first primitive (unset
// when the tile has none); sp / grid / ctrl are the warp's shared-memory slices.
__device__ __forceinline__ void render_item(const int2 item, const WeftTileDecodeDesc& d, const WeftPrim& p0,
                                            const WeftPrim* __restrict__ prims, const float* __restrict__ cp48,
                                            int n_cp48, const float* __restrict__ res1, int n_res1,
                                            float* __restrict__ out, int H, int W, bool w_aligned, size_t row_floats,
                                            Prep* sp, float* grid, float* ctrl, int lane) {
    const int n = d.prim_count, w = d.target_w, h = d.target_h;
    if (!desc_ok(d)) {
        if (lane == 0) report(WEFTK_E_ARG);
        return;
    }
    const int a0 = floor_div4(d.target_x0);
    const int G = floor_div4(d.target_x0 + w + 3) - a0;  // aligned groups per row
    // the item's rows, cropped to the image
    const int r0 = max(item.y, -d.target_y0);
    const int r1 = min(min(h, item.y + max(1, DEC_ITEM_GROUPS / G)), H - d.target_y0);
    const int xa = max(d.target_x0, 0), xb = min(d.target_x0 + w, W);
    if (r0 >= r1 || xa >= xb) return;  // nothing of this item is inside the image
    const bool has_res1 = res1 != nullptr && n_res1 > 0 && d.res1_index >= 0;
    if (has_res1 && d.res1_index >= n_res1) {
        if (lane == 0) report(WEFTK_E_ARG);
        return;
    }
    if (n == 1 && !has_res1 && w_aligned && p0.kind == K_CONST) {
        // a lone constant layer: the blend over black and the RES0 add, once per item
        const Prep c = prep_prim(p0);
        fill_rows(out, row_floats, d.target_y0, r0, r1, xa, xb,
                  clamp01(blend(c.cr, c.a, 0.0f) + d.res0_r), clamp01(blend(c.cg, c.a, 0.0f) + d.res0_g),
                  clamp01(blend(c.cb, c.a, 0.0f) + d.res0_b), lane);
        return;
    }
    for (int i = lane; i < n; i += 32)
        sp[i] = prep_prim(i == 0 ? p0 : load_prim(prims + d.prim_offset + i));
    if (has_res1)
        for (int i = lane; i < 48; i += 32) grid[i] = res1[(size_t)d.res1_index * 48 + i];
    __syncwarp();
    const bool bic = (n == 1 && sp[0].kind == K_BICUBIC);
    if (bic) {
        const int gi = (int)sp[0].q[0];
        if (cp48 == nullptr || gi < 0 || gi >= n_cp48) {
            if (lane == 0) report(WEFTK_E_ARG);
            return;
        }
        for (int i = lane; i < 48; i += 32) ctrl[i] = cp48[(size_t)gi * 48 + i];
        __syncwarp();
    }
    const int side = max(w, h);
    const float step = (side == d.source_size) ? 1.0f : (float)((double)d.source_size / (double)side);
    const float gscale = (float)(4.0 / (double)h);  // RES1 is upsampled at the cropped tile's height
    const int g_end = r1 * G;                           // < 2^24 for any rect the host accepts
    const float invG = 1.0f / (float)G;
    if (n == 1 && sp[0].kind == K_CONST && w_aligned && has_res1) {
        // a lone constant layer with a RES1 grid (the grid is staged in shared memory)
        fill_rows_res1(out, row_floats, d.target_y0, r0, r1, d.target_x0, w, xa, xb, gscale, grid,
                       clamp01(blend(sp[0].cr, sp[0].a, 0.0f) + d.res0_r),
                       clamp01(blend(sp[0].cg, sp[0].a, 0.0f) + d.res0_g),
                       clamp01(blend(sp[0].cb, sp[0].a, 0.0f) + d.res0_b), lane);
        return;
    }
    if (n == 1 && sp[0].kind == K_CONST && has_res1) {
        // A lone constant layer with a RES1 grid on rows that are not 16-byte aligned: one colour
        // plus the bilinear grid per pixel.  Each lane steps its group (row, column) by 32 groups
        // instead of dividing.  (Without a grid such a tile takes the general path below.)
        const float fr = clamp01(blend(sp[0].cr, sp[0].a, 0.0f) + d.res0_r);
        const float fg = clamp01(blend(sp[0].cg, sp[0].a, 0.0f) + d.res0_g);
        const float fb = clamp01(blend(sp[0].cb, sp[0].a, 0.0f) + d.res0_b);
        const int x0 = d.target_x0, x1 = d.target_x0 + w;
        const int drow = 32 / G, dcol = 32 - drow * G;
        int row = r0 + lane / G, col = lane - (lane / G) * G;
        for (int g = r0 * G + lane; g - lane < g_end; g += 32, row += drow, col += dcol) {
            if (col >= G) {
                col -= G;
                ++row;
            }
            if (g >= g_end) continue;
            const int gy = d.target_y0 + row;
            const int gxs = (a0 + col) * 4;
            float* dst = out + (size_t)gy * row_floats + (size_t)gxs * 3;
            const bool full = w_aligned && gxs >= x0 && gxs + DEC_PPL <= x1 && gxs >= 0 && gxs + DEC_PPL <= W;
            float o[DEC_PPL][3];
            // Bilinear 4x4 grid at pixel centres, edge-clamped (src/weft/render.py:474-515).
            const float gyf =
                fminf(fmaxf(__fsub_rn(__fmul_rn((float)row + 0.5f, gscale), 0.5f), 0.0f), 3.0f);
            const int ry0 = (int)floorf(gyf), ry1 = min(ry0 + 1, 3);
            const float wy = __fsub_rn(gyf, (float)ry0);
#pragma unroll
            for (int j = 0; j < DEC_PPL; ++j) {
                const int lxc = min(max(gxs + j - x0, 0), w - 1);
                const float gx =
                    fminf(fmaxf(__fsub_rn(__fmul_rn((float)lxc + 0.5f, gscale), 0.5f), 0.0f), 3.0f);
                const int rx0 = (int)floorf(gx), rx1 = min(rx0 + 1, 3);
                const float wx = __fsub_rn(gx, (float)rx0);
                const float base[3] = {fr, fg, fb};
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) {
                    const float c00 = grid[(ry0 * 4 + rx0) * 3 + ch], c01 = grid[(ry0 * 4 + rx1) * 3 + ch];
                    const float c10 = grid[(ry1 * 4 + rx0) * 3 + ch], c11 = grid[(ry1 * 4 + rx1) * 3 + ch];
                    const float top = __fadd_rn(__fmul_rn(c00, __fsub_rn(1.0f, wx)), __fmul_rn(c01, wx));
                    const float bot = __fadd_rn(__fmul_rn(c10, __fsub_rn(1.0f, wx)), __fmul_rn(c11, wx));
                    o[j][ch] = clamp01(base[ch] + __fadd_rn(__fmul_rn(top, __fsub_rn(1.0f, wy)),
                                                            __fmul_rn(bot, wy)));
                }
            }
            if (full) {
                float4* d4 = reinterpret_cast<float4*>(dst);
                d4[0] = make_float4(o[0][0], o[0][1], o[0][2], o[1][0]);
                d4[1] = make_float4(o[1][1], o[1][2], o[2][0], o[2][1]);
                d4[2] = make_float4(o[2][2], o[3][0], o[3][1], o[3][2]);
                continue;
            }
#pragma unroll
            for (int j = 0; j < DEC_PPL; ++j) {
                const int gxp = gxs + j;
                if (gxp >= x0 && gxp < x1 && gxp >= 0 && gxp < W) {
                    dst[3 * j] = o[j][0];
                    dst[3 * j + 1] = o[j][1];
                    dst[3 * j + 2] = o[j][2];
                }
            }
        }
        return;
    }
    for (int g0 = r0 * G; g0 < g_end; g0 += 32) {
        const int g = g0 + lane;
        const bool g_ok = g < g_end;
        // row = g / G via the float reciprocal, corrected by one step (exact for g < 2^24)
        int row = __float2int_rz(((float)g + 0.5f) * invG);
        row -= (row * G > g) ? 1 : 0;
        row += ((row + 1) * G <= g) ? 1 : 0;
        if (!g_ok) row = r0;
        const int gxs = (a0 + (g_ok ? g - row * G : 0)) * 4;
        float fx[DEC_PPL], fy[DEC_PPL], cr[DEC_PPL], cg[DEC_PPL], cb[DEC_PPL];
        int lx[DEC_PPL];
        bool valid[DEC_PPL];
#pragma unroll
        for (int j = 0; j < DEC_PPL; ++j) {
            lx[j] = gxs + j - d.target_x0;
            valid[j] = g_ok && lx[j] >= 0 && lx[j] < w;
            const int lxc = min(max(lx[j], 0), w - 1);
            fx[j] = __fmul_rn((float)lxc + 0.5f, step);
            fy[j] = __fmul_rn((float)row + 0.5f, step);
            cr[j] = cg[j] = cb[j] = 0.0f;
            lx[j] = lxc;
        }
        if (bic) {
            for (int j = 0; j < DEC_PPL; ++j) {
                float rgb[3];
                bicubic_pixel(ctrl, lx[j], min(row, side - 1), side, rgb);
                cr[j] = rgb[0];
                cg[j] = rgb[1];
                cb[j] = rgb[2];
            }
        } else {
            for (int k = 0; k < n; ++k) {
                Prep pr = sp[k];
                if (pr.kind == K_BICUBIC) pr.kind = K_SKIP;  // kind 5 inside a longer stack is skipped
                float a[DEC_PPL], sr[DEC_PPL], sg[DEC_PPL], sb[DEC_PPL];
                prim_eval<DEC_PPL>(pr, fx, fy, a, sr, sg, sb, lane);
#pragma unroll
                for (int j = 0; j < DEC_PPL; ++j) {
                    cr[j] = blend(sr[j], a[j], cr[j]);
                    cg[j] = blend(sg[j], a[j], cg[j]);
                    cb[j] = blend(sb[j], a[j], cb[j]);
                }
            }
        }
        float o[DEC_PPL][3];
#pragma unroll
        for (int j = 0; j < DEC_PPL; ++j) {
            float r = clamp01(cr[j] + d.res0_r), gg = clamp01(cg[j] + d.res0_g), b = clamp01(cb[j] + d.res0_b);
            if (has_res1) {
                // Bilinear 4x4 grid at pixel centres, edge-clamped (src/weft/render.py:474-515).
                float gx = fminf(fmaxf(__fsub_rn(__fmul_rn((float)lx[j] + 0.5f, gscale), 0.5f), 0.0f), 3.0f);
                float gy = fminf(fmaxf(__fsub_rn(__fmul_rn((float)row + 0.5f, gscale), 0.5f), 0.0f), 3.0f);
                int x0 = (int)floorf(gx), y0 = (int)floorf(gy);
                float wx = __fsub_rn(gx, (float)x0), wy = __fsub_rn(gy, (float)y0);
                int x1 = min(x0 + 1, 3), y1 = min(y0 + 1, 3);
                float v[3];
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) {
                    float c00 = grid[(y0 * 4 + x0) * 3 + ch], c01 = grid[(y0 * 4 + x1) * 3 + ch];
                    float c10 = grid[(y1 * 4 + x0) * 3 + ch], c11 = grid[(y1 * 4 + x1) * 3 + ch];
                    float top = __fadd_rn(__fmul_rn(c00, __fsub_rn(1.0f, wx)), __fmul_rn(c01, wx));
                    float bot = __fadd_rn(__fmul_rn(c10, __fsub_rn(1.0f, wx)), __fmul_rn(c11, wx));
                    v[ch] = __fadd_rn(__fmul_rn(top, __fsub_rn(1.0f, wy)), __fmul_rn(bot, wy));
                }
                r = clamp01(r + v[0]);
                gg = clamp01(gg + v[1]);
                b = clamp01(b + v[2]);
            }
            o[j][0] = r;
            o[j][1] = gg;
            o[j][2] = b;
        }
        if (!g_ok) continue;
        const int gy = d.target_y0 + row;
        float* dst = out + (size_t)gy * row_floats + (size_t)gxs * 3;
        if (w_aligned && valid[0] && valid[DEC_PPL - 1] && gxs >= 0 && gxs + DEC_PPL <= W) {
            float4* d4 = reinterpret_cast<float4*>(dst);
            d4[0] = make_float4(o[0][0], o[0][1], o[0][2], o[1][0]);
            d4[1] = make_float4(o[1][1], o[1][2], o[2][0], o[2][1]);
            d4[2] = make_float4(o[2][2], o[3][0], o[3][1], o[3][2]);
        } else {
#pragma unroll
            for (int j = 0; j < DEC_PPL; ++j) {
                const int gxp = gxs + j;
                if (valid[j] && gxp >= 0 && gxp < W) {
                    dst[3 * j] = o[j][0];
                    dst[3 * j + 1] = o[j][1];
                    dst[3 * j + 2] = o[j][2];
                }
            }
        }
    }
}

__global__ void __launch_bounds__(DEC_THREADS, DEC_MINB) render_tiles_kernel(
    const WeftTileDecodeDesc* __restrict__ descs, int n_tiles, const int2* __restrict__ items, int n_items,
    const WeftPrim* __restrict__ prims, const float* __restrict__ cp48, int n_cp48, const float* __restrict__ res1,
    int n_res1, float* __restrict__ out, int H, int W) {
    __shared__ Prep sp_all[DEC_WARPS][MAX_TILE_PRIMS];
    __shared__ float grid_all[DEC_WARPS][48];
    __shared__ float ctrl_all[DEC_WARPS][48];
    __shared__ int2 bitem_all[DEC_WARPS][DEC_BATCH];
    __shared__ WeftTileDecodeDesc bdesc_all[DEC_WARPS][DEC_BATCH];
    __shared__ WeftPrim bprim_all[DEC_WARPS][DEC_BATCH];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int2* bitem = bitem_all[wid];
    WeftTileDecodeDesc* bdesc = bdesc_all[wid];
    WeftPrim* bprim = bprim_all[wid];
    const bool w_aligned = (W & 3) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    const size_t row_floats = (size_t)3 * W;
    const int n_warps = gridDim.x * DEC_WARPS;
    const int gw = blockIdx.x * DEC_WARPS + wid;
    // round r of this warp: item r * n_warps + gw (r even) or r * n_warps + n_warps - 1 - gw (r odd)
    auto item_index = [&](int r) { return (long long)r * n_warps + ((r & 1) ? n_warps - 1 - gw : gw); };
    for (int round0 = 0; (long long)round0 * n_warps < n_items; round0 += DEC_BATCH) {
        __syncwarp();  // this warp's readers of the previous batch are done
        if (lane < DEC_BATCH) {
            const long long idx = item_index(round0 + lane);
            int2 itm = make_int2(-1, 0);
            if (idx < n_items) itm = items[idx];
            bitem[lane] = itm;
            if (itm.x >= 0 && itm.x < n_tiles) {
                const WeftTileDecodeDesc dd = descs[itm.x];
                bdesc[lane] = dd;
                if (desc_ok(dd) && dd.prim_count >= 1) bprim[lane] = load_prim(prims + dd.prim_offset);
            }
        }
        __syncwarp();
        for (int b = 0; b < DEC_BATCH; ++b) {
            if ((long long)(round0 + b) * n_warps >= n_items) break;
            if (item_index(round0 + b) >= n_items) continue;  // this warp has no item in the round
            const int2 item = bitem[b];
            __syncwarp();  // this warp's readers of sp/grid/ctrl from the previous item are done
            if (item.x < 0 || item.x >= n_tiles || item.y < 0) {
                if (lane == 0) report(WEFTK_E_ARG);
                continue;
            }
            render_item(item, bdesc[b], bprim[b], prims, cp48, n_cp48, res1, n_res1, out, H, W, w_aligned,
                        row_floats, sp_all[wid], grid_all[wid], ctrl_all[wid], lane);
        }
    }
}

int launch_score_evals(const WeftEval* d_evals, int n_evals, const WeftPrim* d_prims, const float* d_tiles,
                       float* d_mse, int flags, cudaStream_t stream) {
    if (n_evals == 0) return WEFTK_OK;
    WEFTK_REQUIRE(n_evals > 0 && d_evals && d_prims && d_tiles && d_mse, "score_evals: bad arguments");
    const float off = (flags & WEFTK_SAMPLE_CORNER) ? 0.0f : 0.5f;
    const int per_block = 256 / 32;
    score_evals_kernel<<<ceil_div(n_evals, per_block), 256, 0, stream>>>(d_evals, n_evals, d_prims, d_tiles, d_mse,
                                                                         off);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}

int launch_render_tiles(const WeftTileDecodeDesc* d_descs, int n_tiles, const int2* d_items, int n_items,
                        const WeftPrim* d_prims, const float* d_cp48, int n_cp48, const float* d_res1, int n_res1,
                        float* d_out, int out_h, int out_w, cudaStream_t stream) {
    if (n_tiles == 0) return WEFTK_OK;
    WEFTK_REQUIRE(n_tiles > 0 && d_descs && d_out && out_h > 0 && out_w > 0, "render_tiles: bad arguments");
    WEFTK_REQUIRE(n_cp48 >= 0 && n_res1 >= 0, "render_tiles: negative table size");
    WEFTK_REQUIRE(d_items != nullptr && n_items >= 0, "render_tiles: missing work items");
    if (n_items == 0) return WEFTK_OK;
    int dev = 0, sms = 148;
    WEFTK_CUDA(cudaGetDevice(&dev));
    WEFTK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = std::min((n_items + DEC_WARPS - 1) / DEC_WARPS, sms * DEC_MINB);
    render_tiles_kernel<<<blocks, DEC_THREADS, 0, stream>>>(d_descs, n_tiles, d_items, n_items, d_prims, d_cp48,
                                                            n_cp48, d_res1, n_res1, d_out, out_h, out_w);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}

int read_device_status(int* status, bool clear) {
    int v = 0;
    WEFTK_CUDA(cudaMemcpyFromSymbol(&v, g_device_status, sizeof(int)));
    if (clear && v != 0) {
        int z = 0;
        WEFTK_CUDA(cudaMemcpyToSymbol(g_device_status, &z, sizeof(int)));
    }
    *status = v;
    return WEFTK_OK;
}

}  // namespace weftk
