// weftk_render.cu — generic per-eval scoring (batch_tile_objective replacement) and the
// decoder's primitive walk (decode_tile_pixels / render_scene_adaptive replacement).
//
// Generic scoring: one warp per eval; each lane owns 4 pixels of a 128-pixel chunk and
// composites the whole stack for them in registers; the per-lane squared error of a
// chunk is summed in float32 and accumulated in float64; one warp reduction per eval.
//
// Decode walk: one 256-thread CTA per tile.  The tile's primitives are prepared once
// into shared memory; warps stride over 128-pixel chunks of the tile's target rect.
// Output is float32 HWC; consecutive lanes write consecutive pixels of a row.
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

constexpr int DEC_THREADS = 128;
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

// Output-major walk.  A work item is (tile, first row): rows [first, first + R) of the tile's
// target rect, R = max(1, WEFTK_DECODE_ITEM_PIXELS / w).  The rect's part of an output row is a
// run of 3w floats; the warp covers the item's runs with 16-byte float4 slots aligned in the
// image, slot q of the item at (row q / n4, float4 q % n4), one slot per lane per step, so the
// lanes of a store instruction write consecutive 16-byte slots (whole sectors) of at most a few
// rows.  A float4 holds parts of two pixels (pa = f / 3 and pa + 1 for its first float f), so a
// lane evaluates two pixels per slot; slots cut by the rect's left or right edge are written
// float by float (the neighbouring tile writes the rest).  The rest as before: a persistent
// grid of one wave, each warp walking items it, it + n_warps, ... and fetching the records of
// its next DEC_BATCH items at once (item, descriptor and first primitive, one item per lane).
constexpr int DEC_WARPS = DEC_THREADS / 32;
constexpr int DEC_MINB = 4;  // resident CTAs per SM the register budget is set for
constexpr int DEC_BATCH = 8;

__device__ __forceinline__ int floor_div(int v, int m) { return v >= 0 ? v / m : -((-v + m - 1) / m); }

__device__ __forceinline__ int rows_per_item(int w) { return max(1, WEFTK_DECODE_ITEM_PIXELS / w); }

// Colour of one channel c (0..2) of a pixel pair for float j of a slot whose first float is at
// phase ph = f % 3: floats j < 3 - ph belong to pixel a, the rest to pixel b.
__device__ __forceinline__ float slot_value(int j, int ph, const float (&A)[3], const float (&B)[3]) {
    const int c = (ph + j) % 3;
    return (j < 3 - ph) ? A[c] : B[c];
}

// Bilinear 4x4 RES1 grid at a pixel centre, edge-clamped (src/weft/render.py:474-515); the row
// terms (ry0, ry1, wy) are the caller's.
__device__ __forceinline__ void res1_at(const float* grid, int lx, float gscale, int ry0, int ry1, float wy,
                                        float (&v)[3]) {
    const float gx = fminf(fmaxf(__fsub_rn(__fmul_rn((float)lx + 0.5f, gscale), 0.5f), 0.0f), 3.0f);
    const int rx0 = (int)floorf(gx), rx1 = min(rx0 + 1, 3);
    const float wx = __fsub_rn(gx, (float)rx0);
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        const float c00 = grid[(ry0 * 4 + rx0) * 3 + ch], c01 = grid[(ry0 * 4 + rx1) * 3 + ch];
        const float c10 = grid[(ry1 * 4 + rx0) * 3 + ch], c11 = grid[(ry1 * 4 + rx1) * 3 + ch];
        const float top = __fadd_rn(__fmul_rn(c00, __fsub_rn(1.0f, wx)), __fmul_rn(c01, wx));
        const float bot = __fadd_rn(__fmul_rn(c10, __fsub_rn(1.0f, wx)), __fmul_rn(c11, wx));
        v[ch] = __fadd_rn(__fmul_rn(top, __fsub_rn(1.0f, wy)), __fmul_rn(bot, wy));
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
    Prep* sp = sp_all[wid];
    float* grid = grid_all[wid];
    float* ctrl = ctrl_all[wid];
    int2* bitem = bitem_all[wid];
    WeftTileDecodeDesc* bdesc = bdesc_all[wid];
    WeftPrim* bprim = bprim_all[wid];
    const bool w_aligned = (W & 3) == 0;  // rows start on 16-byte boundaries
    const long long row_floats = 3ll * W;
    const int n_warps = gridDim.x * DEC_WARPS;
    auto desc_ok = [](const WeftTileDecodeDesc& d) {
        return d.prim_count >= 0 && d.prim_count <= MAX_TILE_PRIMS && d.target_w > 0 && d.target_h > 0 &&
               d.target_w <= 8192 && d.target_h <= 8192 && d.source_size > 0;
    };
    for (int base = blockIdx.x * DEC_WARPS + wid; base < n_items; base += n_warps * DEC_BATCH) {
        __syncwarp();  // this warp's readers of the previous batch are done
        if (lane < DEC_BATCH) {
            const int idx = base + lane * n_warps;
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
            if (base + b * n_warps >= n_items) break;
            const int2 item = bitem[b];
            __syncwarp();  // this warp's readers of sp/grid/ctrl from the previous item are done
            if (item.x < 0 || item.x >= n_tiles) {
                if (lane == 0) report(WEFTK_E_ARG);
                continue;
            }
            const WeftTileDecodeDesc d = bdesc[b];
            const int n = d.prim_count, w = d.target_w, h = d.target_h;
            if (!desc_ok(d) || item.y < 0 || item.y >= h) {
                if (lane == 0) report(WEFTK_E_ARG);
                continue;
            }
            for (int i = lane; i < n; i += 32)
                sp[i] = prep_prim(i == 0 ? bprim[b] : load_prim(prims + d.prim_offset + i));
            const bool has_res1 = res1 != nullptr && n_res1 > 0 && d.res1_index >= 0;
            if (has_res1 && d.res1_index >= n_res1) {
                if (lane == 0) report(WEFTK_E_ARG);
                continue;
            }
            if (has_res1)
                for (int i = lane; i < 48; i += 32) grid[i] = res1[(size_t)d.res1_index * 48 + i];
            __syncwarp();
            const bool bic = (n == 1 && sp[0].kind == K_BICUBIC);
            if (bic) {
                const int gi = (int)sp[0].q[0];
                if (cp48 == nullptr || gi < 0 || gi >= n_cp48) {
                    if (lane == 0) report(WEFTK_E_ARG);
                    continue;
                }
                for (int i = lane; i < 48; i += 32) ctrl[i] = cp48[(size_t)gi * 48 + i];
                __syncwarp();
            }
            const bool lone_const = n == 1 && sp[0].kind == K_CONST;
            const int side = max(w, h);
            const float step = (side == d.source_size) ? 1.0f : (float)((double)d.source_size / (double)side);
            const float gscale = (float)(4.0 / (double)h);  // RES1 is upsampled at the cropped tile's height
            // A lone constant layer is one colour before RES1 (the blend over black and the RES0 add
            // are the general path's operations, done once per item).
            const float cfr = clamp01(blend(sp[0].cr, sp[0].a, 0.0f) + d.res0_r);
            const float cfg = clamp01(blend(sp[0].cg, sp[0].a, 0.0f) + d.res0_g);
            const float cfb = clamp01(blend(sp[0].cb, sp[0].a, 0.0f) + d.res0_b);
            const int x0 = d.target_x0, x1 = d.target_x0 + w;
            const int f_lo = 3 * x0, f_hi = 3 * x1;  // the rect's float run within a row
            const int k0 = floor_div(f_lo, 4), n4 = floor_div(f_hi + 3, 4) - k0;
            const int r0 = item.y, r1 = min(h, r0 + rows_per_item(w));
            const int total = (r1 - r0) * n4;
            // slot q = base + lane at (row, col); each step advances 32 slots
            const int drow = 32 / n4, dcol = 32 - drow * n4;
            int row = r0 + lane / n4, col = lane - (lane / n4) * n4;
            for (int sbase = 0; sbase < total; sbase += 32, row += drow, col += dcol) {
                if (col >= n4) {
                    col -= n4;
                    ++row;
                }
                const bool q_ok = sbase + lane < total;
                const int fa = 4 * (k0 + col);                 // first float of the slot in the row
                const int ph = ((fa % 3) + 3) % 3;
                const int pa = floor_div(fa, 3), pb = pa + 1;  // the slot's two pixels
                const int la = min(max(pa - x0, 0), w - 1), lb = min(max(pb - x0, 0), w - 1);
                const int rrow = q_ok ? row : r0;
                float A[3], B[3];
                if (lone_const) {
                    A[0] = B[0] = cfr;
                    A[1] = B[1] = cfg;
                    A[2] = B[2] = cfb;
                } else if (bic) {
                    bicubic_pixel(ctrl, la, min(rrow, side - 1), side, A);
                    bicubic_pixel(ctrl, lb, min(rrow, side - 1), side, B);
                } else {
                    float fx[2], fy[2], cr[2] = {0.0f, 0.0f}, cg[2] = {0.0f, 0.0f}, cb[2] = {0.0f, 0.0f};
                    fx[0] = __fmul_rn((float)la + 0.5f, step);
                    fx[1] = __fmul_rn((float)lb + 0.5f, step);
                    fy[0] = fy[1] = __fmul_rn((float)rrow + 0.5f, step);
                    for (int k = 0; k < n; ++k) {
                        Prep pr = sp[k];
                        if (pr.kind == K_BICUBIC) pr.kind = K_SKIP;  // kind 5 inside a longer stack is skipped
                        float a[2], sr[2], sg[2], sb[2];
                        prim_eval<2>(pr, fx, fy, a, sr, sg, sb, lane);
#pragma unroll
                        for (int j = 0; j < 2; ++j) {
                            cr[j] = blend(sr[j], a[j], cr[j]);
                            cg[j] = blend(sg[j], a[j], cg[j]);
                            cb[j] = blend(sb[j], a[j], cb[j]);
                        }
                    }
                    A[0] = clamp01(cr[0] + d.res0_r);
                    A[1] = clamp01(cg[0] + d.res0_g);
                    A[2] = clamp01(cb[0] + d.res0_b);
                    B[0] = clamp01(cr[1] + d.res0_r);
                    B[1] = clamp01(cg[1] + d.res0_g);
                    B[2] = clamp01(cb[1] + d.res0_b);
                }
                if (has_res1) {
                    const float gyf = fminf(fmaxf(__fsub_rn(__fmul_rn((float)rrow + 0.5f, gscale), 0.5f), 0.0f), 3.0f);
                    const int ry0 = (int)floorf(gyf), ry1 = min(ry0 + 1, 3);
                    const float wy = __fsub_rn(gyf, (float)ry0);
                    float va[3], vb[3];
                    res1_at(grid, la, gscale, ry0, ry1, wy, va);
                    res1_at(grid, lb, gscale, ry0, ry1, wy, vb);
#pragma unroll
                    for (int ch = 0; ch < 3; ++ch) {
                        A[ch] = clamp01(A[ch] + va[ch]);
                        B[ch] = clamp01(B[ch] + vb[ch]);
                    }
                }
                const int gy = d.target_y0 + row;
                if (!q_ok || gy < 0 || gy >= H) continue;
                float* dst = out + (size_t)gy * row_floats + fa;
                if (w_aligned && fa >= f_lo && fa + 4 <= f_hi && fa >= 0 && fa + 4 <= row_floats) {
                    *reinterpret_cast<float4*>(dst) = make_float4(slot_value(0, ph, A, B), slot_value(1, ph, A, B),
                                                                  slot_value(2, ph, A, B), slot_value(3, ph, A, B));
                } else {
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int f = fa + j;
                        if (f >= f_lo && f < f_hi && f >= 0 && f < row_floats) dst[j] = slot_value(j, ph, A, B);
                    }
                }
            }
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
