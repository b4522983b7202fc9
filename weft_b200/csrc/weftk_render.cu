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

constexpr int DEC_PPL = 4;
constexpr int DEC_THREADS = 128;
static_assert(WEFTK_DECODE_CHUNK_GROUPS == 32 && DEC_PPL == 4, "chunk layout is part of the C ABI");
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

// Work items: (tile, first chunk) pairs.  Each row of a tile's target rect is covered by
// 4-pixel groups aligned to output x multiples of 4, so a thread writes its 4 pixels
// (48 bytes) as three 16-byte stores.  A chunk is 32 groups (one per lane) and an item is
// up to DEC_ITEM_CHUNKS chunks, rendered by ONE warp: the warp stages its tile's
// primitives in its own slice of shared memory and never waits on the rest of the CTA,
// so every resident warp works on a different item.  A persistent grid of one wave
// (every CTA resident) walks the list.  A warp's items are it, it + n_warps, ...; it
// fetches the records of its next DEC_BATCH items at once (item, descriptor and first
// primitive, one item per lane), so the dependent-load chain item -> descriptor ->
// primitive is paid once per batch instead of once per item.
constexpr int DEC_ITEM_CHUNKS = WEFTK_DECODE_ITEM_CHUNKS;
constexpr int DEC_WARPS = DEC_THREADS / 32;
constexpr int DEC_MINB = 4;  // resident CTAs per SM the register budget is set for
constexpr int DEC_BATCH = 8;

__device__ __forceinline__ int floor_div4(int v) { return v >= 0 ? (v >> 2) : -((-v + 3) >> 2); }

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
    const bool w_aligned = (W & 3) == 0;
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
            if (!desc_ok(d)) {
                if (lane == 0) report(WEFTK_E_ARG);
                continue;
            }
            const int a0 = floor_div4(d.target_x0);
            const int G = floor_div4(d.target_x0 + w + 3) - a0;  // aligned groups per row
            const int n_groups = G * h;                          // < 2^24 for any rect the host accepts
            const int n_chunks = (n_groups + 31) / 32;
            const float invG = 1.0f / (float)G;
            const int c_end = min(n_chunks, item.y + DEC_ITEM_CHUNKS);
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
            const int side = max(w, h);
            const float step = (side == d.source_size) ? 1.0f : (float)((double)d.source_size / (double)side);
            const float gscale = (float)(4.0 / (double)h);  // RES1 is upsampled at the cropped tile's height
            if (n == 1 && sp[0].kind == K_CONST) {
                // A lone constant layer is one colour before RES1 (the blend over black and the RES0
                // add are the general path's operations, done once per item), so the walk only
                // writes it, or adds the bilinear RES1 grid per pixel.  Each lane steps its group
                // (row, column) by 32 groups per chunk instead of dividing.
                const float fr = clamp01(blend(sp[0].cr, sp[0].a, 0.0f) + d.res0_r);
                const float fg = clamp01(blend(sp[0].cg, sp[0].a, 0.0f) + d.res0_g);
                const float fb = clamp01(blend(sp[0].cb, sp[0].a, 0.0f) + d.res0_b);
                const int x0 = d.target_x0, x1 = d.target_x0 + w;
                const int g0 = item.y * 32 + lane, drow = 32 / G, dcol = 32 - drow * G;
                int row = g0 / G, col = g0 - row * G;
                for (int chunk = item.y; chunk < c_end; ++chunk, row += drow, col += dcol) {
                    if (col >= G) {
                        col -= G;
                        ++row;
                    }
                    const int gy = d.target_y0 + row;
                    if (row >= h || gy < 0 || gy >= H) continue;
                    const int gxs = (a0 + col) * 4;
                    float* dst = out + ((size_t)gy * W + gxs) * 3;
                    const bool full = w_aligned && gxs >= x0 && gxs + DEC_PPL <= x1 && gxs >= 0 && gxs + DEC_PPL <= W;
                    float o[DEC_PPL][3];
                    if (!has_res1) {
                        if (full) {
                            float4* d4 = reinterpret_cast<float4*>(dst);
                            d4[0] = make_float4(fr, fg, fb, fr);
                            d4[1] = make_float4(fg, fb, fr, fg);
                            d4[2] = make_float4(fb, fr, fg, fb);
                            continue;
                        }
#pragma unroll
                        for (int j = 0; j < DEC_PPL; ++j) {
                            o[j][0] = fr;
                            o[j][1] = fg;
                            o[j][2] = fb;
                        }
                    } else {
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
                continue;
            }
            for (int chunk = item.y; chunk < c_end; ++chunk) {
                const int g = chunk * 32 + lane;
                const bool g_ok = g < n_groups;
                // row = g / G via the float reciprocal, corrected by one step (exact for g < 2^24)
                int row = __float2int_rz(((float)g + 0.5f) * invG);
                row -= (row * G > g) ? 1 : 0;
                row += ((row + 1) * G <= g) ? 1 : 0;
                if (!g_ok) row = 0;
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
                const int gy = d.target_y0 + row;
                if (!g_ok || gy < 0 || gy >= H) continue;
                float* dst = out + ((size_t)gy * W + gxs) * 3;
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
