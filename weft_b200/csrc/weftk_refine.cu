// weftk_refine.cu — per-tile stack loss and its hand-written backward (see include/weftk_refine.h).
//
// One launch covers every tile.  Tiles are grouped by side so that each warp
// has at most 16 chunks of 32 pixels: a tile of side > 32 gets eight warps,
// 17..32 four, 9..16 two, <= 8 one; every CTA has eight warps and holds one or
// more such tile groups, and CTAs of the largest tiles come first so they start
// first.  Each warp of a tile owns a contiguous range of chunks and prefetches
// the next chunk's source pixels while it works on the current one.  The tile's
// parameter rows are prepared once into shared memory (and a curve's 31
// polyline segments into a segment table).  The backward re-renders a chunk
// front to back, keeping the composite *before* every layer in shared memory
// (layers x 32 lanes x 3 floats per warp, the only per-pixel state, never
// written to HBM), then sweeps the layers back to front:
//     c_k = s_k a_k + c_{k-1} (1 - a_k)
//     dL/ds_k = g a_k,  dL/da_k = g . (s_k - c_{k-1}),  g <- g (1 - a_k)
// and chains dL/ds, dL/da into the layer's parameters with the coverage
// recomputed at that pixel.  Every sum (gradients over pixels, block and
// quadrant sums of the residual loss) has a single owner and a fixed order, so
// results are deterministic.
//
// Residual-aware loss (WEFTK_LOSS_RESIDUAL): the file a fit becomes carries a
// per-tile 4x4 grid of block-mean errors that the decoder adds back with
// bilinear interpolation (src/weft/encoder.py:3248-3372, src/weft/render.py:474-515).
// With e = clamp(render) - src, M the 4x4 block-mean operator and B the decoder's
// bilinear upsampling, the decoded error is r = e - B M e (before the grid's
// 8-bit quantisation and clamping), and the loss is mean(r^2) with gradient
// 2 (I - M^T B^T) r / (3n).  Pixels are visited block-major, quadrant-major
// inside a block, so block sums and the per-quadrant sums of B^T r are
// segmented warp reductions over aligned lane groups.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>

#include "../../include/weftk_fit.h"
#include "../../include/weftk_refine.h"
#include "weftk_common.cuh"
#include "weftk_prim.cuh"

namespace weftk {

extern __device__ int g_device_status;

constexpr int MAXL = WEFTK_REFINE_MAX_PRIMS;
constexpr float TRI_SOFT_W = 0.5f;  // surrogate edge width in pixels

// The layers of one tile, staged in shared memory.
struct Layers {
    const Prep* prep;
    const float (*raw)[16];
    const float4 (*seg)[31][2];
};

__device__ __forceinline__ WeftPrim row_to_prim(const float* r, int kind) {
    WeftPrim p;
    p.kind = kind;
#pragma unroll
    for (int i = 0; i < 7; ++i) p.geom[i] = r[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        p.color0[i] = r[7 + i];
        p.color1[i] = r[10 + i];
    }
    p.alpha = r[13];
    return p;
}

__device__ __forceinline__ float sigmoid(float x) { return 1.0f / (1.0f + __expf(-x)); }

// Soft triangle coverage and, if grad != nullptr, its gradient w.r.t. the 6 vertex
// coordinates.  s_i = signed distance to edge i (positive inside), cov = prod sigmoid(s_i / w).
__device__ float tri_soft(const float* g, float px, float py, float* grad) {
    const float vx[3] = {g[0], g[2], g[4]}, vy[3] = {g[1], g[3], g[5]};
    const float a2 = (vx[1] - vx[0]) * (vy[2] - vy[0]) - (vy[1] - vy[0]) * (vx[2] - vx[0]);
    const float o = a2 >= 0.0f ? 1.0f : -1.0f;
    float sd[3], sig[3], dsa[3][2], dsb[3][2];
    float cov = 1.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int ia = (i + 1) % 3, ib = (i + 2) % 3;  // edge opposite vertex i
        const float ex = vx[ib] - vx[ia], ey = vy[ib] - vy[ia];
        const float rx = px - vx[ia], ry = py - vy[ia];
        const float C = ex * ry - ey * rx;
        const float L = sqrtf(ex * ex + ey * ey) + 1e-12f;
        sd[i] = o * C / L;
        sig[i] = sigmoid(sd[i] / TRI_SOFT_W);
        cov *= sig[i];
        const float iL = 1.0f / L, iL2 = iL * iL;
        // dC/da = (-ry + ey, rx - ex), dC/db = (ry, -rx); dL/da = -e/L, dL/db = e/L
        dsa[i][0] = o * ((-ry + ey) * L + C * ex * iL) * iL2;
        dsa[i][1] = o * ((rx - ex) * L + C * ey * iL) * iL2;
        dsb[i][0] = o * (ry * L - C * ex * iL) * iL2;
        dsb[i][1] = o * (-rx * L - C * ey * iL) * iL2;
    }
    if (grad) {
#pragma unroll
        for (int k = 0; k < 6; ++k) grad[k] = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int ia = (i + 1) % 3, ib = (i + 2) % 3;
            const float dc = cov * (1.0f - sig[i]) / TRI_SOFT_W;
            grad[2 * ia] += dc * dsa[i][0];
            grad[2 * ia + 1] += dc * dsa[i][1];
            grad[2 * ib] += dc * dsb[i][0];
            grad[2 * ib + 1] += dc * dsb[i][1];
        }
    }
    return cov;
}

// Source colour and alpha of layer k at one pixel (the renderer's formulas).
__device__ __forceinline__ void layer_eval(const Layers& s, int k, float px, float py, bool soft, float (&src)[3],
                                           float& a) {
    const Prep& P = s.prep[k];
    float fx[1] = {px}, fy[1] = {py}, av[1], sr[1], sg[1], sb[1];
    if (P.kind == K_CURVE) {
        sr[0] = P.cr;
        sg[0] = P.cg;
        sb[0] = P.cb;
        curve_alpha_smem<1>(P, s.seg[k], fx, fy, av);
    } else if (P.kind == K_TRI && soft) {
        sr[0] = P.cr;
        sg[0] = P.cg;
        sb[0] = P.cb;
        av[0] = tri_soft(s.raw[k], px, py, nullptr) * P.a;
    } else {
        prim_eval<1>(P, fx, fy, av, sr, sg, sb, 0);
    }
    src[0] = sr[0];
    src[1] = sg[0];
    src[2] = sb[0];
    a = av[0];
}

// Gradient contribution of layer k at one pixel.  g = dL/dc_k, cp = c_{k-1}.
__device__ void layer_grad(const Layers& s, int k, float px, float py, bool soft, const float (&g)[3],
                           const float (&cp)[3], float& a_out, float (&d)[14]) {
    const Prep& P = s.prep[k];
    const float* r = s.raw[k];
#pragma unroll
    for (int i = 0; i < 14; ++i) d[i] = 0.0f;
    float src[3], a;
    layer_eval(s, k, px, py, soft, src, a);
    a_out = a;
    if (P.kind == K_SKIP) return;
    const float A = P.a;
    const float dA = (r[13] >= 0.0f && r[13] <= 1.0f) ? 1.0f : 0.0f;
    float dLds[3], dLda = 0.0f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        dLds[c] = g[c] * a;
        dLda = fmaf(g[c], src[c] - cp[c], dLda);
    }
    const float cov = A > 0.0f ? a / A : 0.0f;
    const float dLdcov = dLda * A;
    switch (P.kind) {
        case K_CONST:
            d[7] = dLds[0];
            d[8] = dLds[1];
            d[9] = dLds[2];
            d[13] = dLda * dA;
            break;
        case K_LINEAR: {
            const float x0 = r[0], y0 = r[1], vx = r[2] - r[0], vy = r[3] - r[1];
            const float D = vx * vx + vy * vy + 1e-8f;
            const float qx = px - x0, qy = py - y0, N = qx * vx + qy * vy;
            const float traw = fmaf(qx, P.q[2], qy * P.q[3]);
            const float t = clamp01(traw);
            d[7] = dLds[0] * (1.0f - t);
            d[8] = dLds[1] * (1.0f - t);
            d[9] = dLds[2] * (1.0f - t);
            d[10] = dLds[0] * t;
            d[11] = dLds[1] * t;
            d[12] = dLds[2] * t;
            d[13] = dLda * dA;
            if (traw > 0.0f && traw < 1.0f) {
                const float dLdt = dLds[0] * (r[10] - r[7]) + dLds[1] * (r[11] - r[8]) + dLds[2] * (r[12] - r[9]);
                const float iD2 = 1.0f / (D * D);
                // dN/dp0 = -v - q, dN/dp1 = q; dD/dp0 = -2v, dD/dp1 = 2v
                d[0] = dLdt * ((-vx - qx) * D + N * 2.0f * vx) * iD2;
                d[1] = dLdt * ((-vy - qy) * D + N * 2.0f * vy) * iD2;
                d[2] = dLdt * (qx * D - N * 2.0f * vx) * iD2;
                d[3] = dLdt * (qy * D - N * 2.0f * vy) * iD2;
            }
            break;
        }
        case K_LINE:
        case K_CURVE: {
            d[7] = dLds[0];
            d[8] = dLds[1];
            d[9] = dLds[2];
            d[13] = dLda * cov * dA;
            const float thick = P.kind == K_LINE ? r[4] : r[6];
            const float sigma = fmaxf(0.5f, thick);
            const float K = P.kind == K_LINE ? P.q[6] : P.q[0];
            // closest point: segment start (ax, ay), direction v, projection u
            float ax, ay, vx, vy, ux, uy;
            int kseg = 0;
            if (P.kind == K_LINE) {
                ax = P.q[0]; ay = P.q[1]; vx = P.q[2]; vy = P.q[3]; ux = P.q[4]; uy = P.q[5];
            } else {
                float best = 1e30f;
                for (int j = 0; j < 31; ++j) {
                    const float4 s0 = s.seg[k][j][0], s1 = s.seg[k][j][1];
                    const float dd = seg_d2(px, py, s0.x, s0.y, s0.z, s0.w, s1.x, s1.y);
                    if (dd < best) {
                        best = dd;
                        kseg = j;
                    }
                }
                const float4 s0 = s.seg[k][kseg][0], s1 = s.seg[k][kseg][1];
                ax = s0.x; ay = s0.y; vx = s0.z; vy = s0.w; ux = s1.x; uy = s1.y;
            }
            const float dx = px - ax, dy = py - ay;
            const float t = clamp01(fmaf(dx, ux, dy * uy));
            const float ex = fmaf(-t, vx, dx), ey = fmaf(-t, vy, dy);
            const float d2 = fmaf(ex, ex, ey * ey);
            const float dLdd2 = dLdcov * K * cov;
            // dd2/d(start) = -2e(1-t), dd2/d(end) = -2e t
            const float gsx = -2.0f * ex * (1.0f - t) * dLdd2, gsy = -2.0f * ey * (1.0f - t) * dLdd2;
            const float gex = -2.0f * ex * t * dLdd2, gey = -2.0f * ey * t * dLdd2;
            if (P.kind == K_LINE) {
                d[0] = gsx; d[1] = gsy; d[2] = gex; d[3] = gey;
                if (thick > 0.5f) d[4] = dLdcov * cov * d2 / (sigma * sigma * sigma);
            } else {
                // polyline points are Bezier samples q_j = u^2 P0 + 2ut C + t^2 P1
#pragma unroll
                for (int e2 = 0; e2 < 2; ++e2) {
                    const int j = kseg + e2;
                    const float tj = (j >= 31) ? 1.0f : (float)((double)j * (1.0 / 31.0));
                    const float uj = 1.0f - tj;
                    const float w0 = uj * uj, w1 = 2.0f * uj * tj, w2 = tj * tj;
                    const float gx = e2 ? gex : gsx, gy = e2 ? gey : gsy;
                    d[0] += w0 * gx; d[1] += w0 * gy;
                    d[2] += w1 * gx; d[3] += w1 * gy;
                    d[4] += w2 * gx; d[5] += w2 * gy;
                }
                if (thick > 0.5f) d[6] = dLdcov * cov * d2 / (sigma * sigma * sigma);
            }
            break;
        }
        case K_TRI: {
            d[7] = dLds[0];
            d[8] = dLds[1];
            d[9] = dLds[2];
            d[13] = dLda * cov * dA;
            float gg[6];
            tri_soft(r, px, py, gg);
#pragma unroll
            for (int i = 0; i < 6; ++i) d[i] = dLdcov * gg[i];
            break;
        }
        default:
            break;
    }
}

// Shared-memory carve-up of one tile group (the WPT warps working on one tile).
// Byte offsets for L staged layers; every region starts on a 16-byte boundary
// except the trailing doubles (8-byte aligned).
struct GroupLayout {
    int prep, seg, raw, madam, vadam, msum, quad, hnode, hist, gacc, lacc, lred, mom, bytes;
};

// Stacks of at most this many layers accumulate gradients per lane (one slot per
// lane, column and layer) and reduce once per tile; longer stacks reduce every chunk.
constexpr int RF_LANE_ACC_MAX = 2;

// msum/quad/hnode exist only for the residual loss, lacc only for short stacks.
__host__ __device__ __forceinline__ GroupLayout group_layout(int L, int wpt, bool resid) {
    GroupLayout g;
    g.prep = 0;
    g.seg = g.prep + L * 64;
    g.raw = g.seg + L * 992;
    g.madam = g.raw + L * 64;   // Adam moments of the rows (RF_STEP)
    g.vadam = g.madam + L * 64;
    g.msum = g.vadam + L * 64;
    g.quad = g.msum + (resid ? 48 * 4 : 0);
    g.hnode = g.quad + (resid ? 768 * 4 : 0);
    g.hist = g.hnode + (resid ? 48 * 4 : 0);
    g.gacc = g.hist + wpt * L * 384;
    g.lacc = (g.gacc + wpt * L * 56 + 15) & ~15;
    g.lred = g.lacc + (L <= RF_LANE_ACC_MAX ? wpt * L * 14 * 32 * 4 : 0);
    g.mom = g.lred + wpt * 8;  // pixel moments of a lone constant layer's tile: per warp, then total
    g.bytes = (g.mom + (wpt + 1) * 6 * 8 + 15) & ~15;
    return g;
}

// Adam (PyTorch's update rule, FP32) for one value at step t (1-based), then the
// projection onto what the wire format carries: colours and alpha in [0, 1],
// coordinates in [0, 15], thickness in [0, 4] (src/weft/primitives.py:102-177).
// Projection of column col of a row onto its valid range (colours and alpha [0, 1], thickness
// [0, 4], other geometry [0, 15]).
__device__ __forceinline__ float adam_project(float x, int kind, int col) {
    if (col >= 7) return fminf(fmaxf(x, 0.0f), 1.0f);
    const bool thick = (kind == K_LINE && col == 4) || (kind == K_CURVE && col == 6);
    return fminf(fmaxf(x, 0.0f), thick ? 4.0f : 15.0f);
}

__device__ __forceinline__ float adam_update_bc(float p, float g, float& m, float& v, float bc1, float bc2, float lr,
                                                float b1, float b2, float eps, int kind, int col) {
    m = fmaf(b1, m, (1.0f - b1) * g);
    v = fmaf(b2, v, (1.0f - b2) * g * g);
    return adam_project(p - lr * (m / bc1) / (sqrtf(v / bc2) + eps), kind, col);
}

// Bias corrections 1 - beta^t of step t (1-based).
__device__ __forceinline__ void adam_bias(float b1, float b2, float t, float& bc1, float& bc2) {
    bc1 = 1.0f - powf(b1, t);
    bc2 = 1.0f - powf(b2, t);
}

__device__ __forceinline__ float adam_update(float p, float g, float& m, float& v, float t, float lr, float b1,
                                             float b2, float eps, int kind, int col) {
    float bc1, bc2;
    adam_bias(b1, b2, t, bc1, bc2);
    return adam_update_bc(p, g, m, v, bc1, bc2, lr, b1, b2, eps, kind, col);
}

// Optimiser state of the fused refine step; the per-row step count lives in m[row * 16 + 15].
struct AdamArgs {
    float* m;
    float* v;
    float lr, b1, b2, eps;
};

// CTA classes of one launch, in launch order: tiles of side > 32 (8 warps per
// tile), 17..32 (4 warps), 9..16 (2 warps), <= 8 (1 warp).  Every CTA has 8
// warps; a CTA of class c holds groups[c] tiles.
constexpr int RF_THREADS = 256;
constexpr int RF_CLASSES = 4;
constexpr int RF_SMEM_MAX = 227 * 1024;

struct RefinePlan {
    int cta_end[RF_CLASSES];  // exclusive prefix sums of the classes' CTA counts
    int list_off[RF_CLASSES];
    int n_list[RF_CLASSES];
    int groups[RF_CLASSES];
};

__host__ __device__ __forceinline__ int class_wpt(int c) { return 8 >> c; }

// a[c] without dynamic indexing (keeps the plan in registers, off the stack)
__device__ __forceinline__ int pick(const int (&a)[RF_CLASSES], int c) {
    return c == 0 ? a[0] : c == 1 ? a[1] : c == 2 ? a[2] : a[3];
}

// Gradient columns a layer of this kind can produce (bit i = column i).
__device__ __forceinline__ unsigned grad_columns(int kind) {
    switch (kind) {
        case K_CONST: return 0x2380u;   // 7 8 9 13
        case K_LINEAR: return 0x3f8fu;  // 0-3 7-13
        case K_LINE: return 0x239fu;    // 0-4 7 8 9 13
        case K_CURVE: return 0x23ffu;   // 0-6 7 8 9 13
        case K_TRI: return 0x23bfu;     // 0-5 7 8 9 13
        default: return 0u;
    }
}

// Bilinear node pair (lo, hi) and weight of the decoder's 4x4 residual grid for a
// pixel index along one axis of a tile with gscale = 4 / side (src/weft/render.py:474-515:
// centre sampling, edge clamp).
__device__ __forceinline__ void grid_coord(int p, float gscale, int& lo, int& hi, float& w) {
    const float g = fminf(fmaxf(__fsub_rn(__fmul_rn((float)p + 0.5f, gscale), 0.5f), 0.0f), 3.0f);
    lo = (int)floorf(g);
    hi = min(lo + 1, 3);
    w = g - (float)lo;
}

// Quadrant columns (0..7: block q / 2, half q % 2) whose pixels interpolate from grid
// node n along one axis, with the slot (0: lower node, 1: upper node) they use.  Lower
// node n: the right half of block n, the left half of block n + 1, and for n = 0 the left
// half of block 0 (clamped).  Upper node n: the right half of block n - 1, the left half
// of block n (n >= 1), and for n = 3 the right half of block 3 (clamped, weight 0).  The
// left half of block 0 also names node 1 as its upper node, with weight 0; it is skipped.
// Returns the count (<= 4); entries are (column << 1) | slot.
__device__ __forceinline__ int node_sources(int n, int (&out)[4]) {
    int c = 0;
    if (n == 0) out[c++] = (0 << 1) | 0;
    if (2 * n + 1 <= 7) out[c++] = ((2 * n + 1) << 1) | 0;
    if (2 * n + 2 <= 7) out[c++] = ((2 * n + 2) << 1) | 0;
    if (n >= 1) out[c++] = ((2 * n - 1) << 1) | 1;
    if (n >= 1) out[c++] = ((2 * n) << 1) | 1;
    if (n == 3) out[c++] = (7 << 1) | 1;
    return c;
}

// Barrier over the warps of one tile group (named barrier 1 + group; one warp: __syncwarp).
__device__ __forceinline__ void group_sync(int wpt, int grp) {
    if (wpt == 1)
        __syncwarp();
    else
        asm volatile("bar.sync %0, %1;" ::"r"(grp + 1), "r"(wpt * 32) : "memory");
}

// Single-layer stacks of a constant or linear primitive (the refined fit's stacks): the layer's
// source colour, alpha and the linear ramp parameter at one pixel, with the renderer's formulas
// (prim_eval), so the forward is the same float sequence; any other kind is a no-op here.
struct ClEval {
    float s[3], a, t, traw;
};

__device__ __forceinline__ ClEval eval_cl(const Prep& P, float px, float py) {
    ClEval r;
    r.s[0] = P.cr;
    r.s[1] = P.cg;
    r.s[2] = P.cb;
    r.a = (P.kind == K_CONST || P.kind == K_LINEAR) ? P.a : 0.0f;
    r.t = r.traw = 0.0f;
    if (P.kind == K_LINEAR) {
        r.traw = fmaf(px - P.q[0], P.q[2], (py - P.q[1]) * P.q[3]);
        r.t = clamp01(r.traw);
        const float u = 1.0f - r.t;
        r.s[0] = fmaf(P.q[4], r.t, P.cr * u);
        r.s[1] = fmaf(P.q[5], r.t, P.cg * u);
        r.s[2] = fmaf(P.q[6], r.t, P.cb * u);
    }
    return r;
}

// Gradient of that layer over black (c_{-1} = 0), accumulated into acc[14]; the same chain
// rule as layer_grad's constant and linear cases.
__device__ __forceinline__ void grad_cl(const Prep& P, const float* r, const ClEval& v, float px, float py,
                                        const float (&g)[3], float (&acc)[14]) {
    if (P.kind != K_CONST && P.kind != K_LINEAR) return;
    const float dA = (r[13] >= 0.0f && r[13] <= 1.0f) ? 1.0f : 0.0f;
    float dLds[3], dLda = 0.0f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        dLds[c] = g[c] * v.a;
        dLda = fmaf(g[c], v.s[c], dLda);
    }
    acc[13] = fmaf(dLda, dA, acc[13]);
    if (P.kind == K_CONST) {
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[7 + c] += dLds[c];
        return;
    }
    const float t = v.t;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        acc[7 + c] = fmaf(dLds[c], 1.0f - t, acc[7 + c]);
        acc[10 + c] = fmaf(dLds[c], t, acc[10 + c]);
    }
    if (v.traw > 0.0f && v.traw < 1.0f) {
        const float x0 = r[0], y0 = r[1], vx = r[2] - r[0], vy = r[3] - r[1];
        const float D = vx * vx + vy * vy + 1e-8f;
        const float qx = px - x0, qy = py - y0, N = qx * vx + qy * vy;
        const float dLdt = dLds[0] * (r[10] - r[7]) + dLds[1] * (r[11] - r[8]) + dLds[2] * (r[12] - r[9]);
        const float iD2 = 1.0f / (D * D);
        acc[0] += dLdt * ((-vx - qx) * D + N * 2.0f * vx) * iD2;
        acc[1] += dLdt * ((-vy - qy) * D + N * 2.0f * vy) * iD2;
        acc[2] += dLdt * (qx * D - N * 2.0f * vx) * iD2;
        acc[3] += dLdt * (qy * D - N * 2.0f * vy) * iD2;
    }
}

// One kernel for the loss (MODE 0), loss + gradient (MODE 1), and loss + gradient +
// Adam step on the tile's own rows (MODE 2: params are updated in place; a group reads
// its rows once at staging and writes them once at the end, and rows belong to one tile).
// Loss sum and colour / alpha gradient of a lone constant layer over black from the tile's pixel
// sums S = (S1 r, g, b, S2 r, g, b) over n pixels: the layer renders q = colour * alpha per
// channel, so sum (q - s)^2 = n q^2 - 2 q S1 + S2 and sum (q - s) = n q - S1.  g4 (may be null):
// d/dcolour0 (3) and d/dalpha, scaled by gscale.  Every float64 operation is rounded on its own,
// so both kernels that use it agree bit for bit.
__device__ __forceinline__ double const_layer_closed(const Prep& P, float alpha_raw, const double* S, int n,
                                                     float gscale, float* g4) {
    const float sv[3] = {P.cr, P.cg, P.cb};
    const double nd = (double)n;
    double tot = 0.0, galpha = 0.0;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        const float c = __fmul_rn(sv[ch], P.a);  // blend over black: colour * alpha
        const double cc = (double)clamp01(c);
        const double e = __dadd_rn(__dsub_rn(__dmul_rn(__dmul_rn(nd, cc), cc), __dmul_rn(__dmul_rn(2.0, cc), S[ch])),
                                   S[3 + ch]);
        tot = __dadd_rn(tot, e);
        const float G = (c >= 0.0f && c <= 1.0f)
                            ? (float)__dmul_rn((double)gscale, __dsub_rn(__dmul_rn(nd, (double)c), S[ch]))
                            : 0.0f;
        if (g4) g4[ch] = __fmul_rn(G, P.a);
        galpha = __dadd_rn(galpha, (double)__fmul_rn(G, sv[ch]));
    }
    if (g4) g4[3] = (alpha_raw >= 0.0f && alpha_raw <= 1.0f) ? (float)galpha : 0.0f;
    return tot;
}

constexpr int RF_LOSS = 0, RF_GRAD = 1, RF_STEP = 2;

// CL1: every stack has at most one layer, of kind constant or linear (checked per tile): the
// forward and backward then run out of registers (no composite history, no kind dispatch).
template <int MODE, bool CL1>
__global__ void __launch_bounds__(RF_THREADS, 3)
    refine_tiles_kernel(WeftStackSet set, float* __restrict__ params, const float* __restrict__ grad_loss,
                        float* __restrict__ grad, float* __restrict__ loss, int flags, RefinePlan plan, int L,
                        AdamArgs adam, int n_steps) {
    constexpr bool BWD = MODE != RF_LOSS;
    extern __shared__ __align__(16) unsigned char rf_smem[];
    const int bx = blockIdx.x;
    const int cls = (bx >= plan.cta_end[0]) + (bx >= plan.cta_end[1]) + (bx >= plan.cta_end[2]);
    const int cta0 = cls ? pick(plan.cta_end, cls - 1) : 0;
    const int wpt = class_wpt(cls), G = pick(plan.groups, cls);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = warp / wpt, wig = warp - grp * wpt;  // group, warp inside the group
    if (grp >= G) return;
    const int li = ((int)blockIdx.x - cta0) * G + grp;
    if (li >= pick(plan.n_list, cls)) return;  // uniform over the group
    const int lo = pick(plan.list_off, cls);
    const int t = set.order ? set.order[lo + li] : lo + li;
    const bool resid = flags & WEFTK_LOSS_RESIDUAL;
    const bool soft = flags & WEFTK_SOFT_TRIANGLES;
    const bool lane_acc = L <= RF_LANE_ACC_MAX;
    const GroupLayout lay = group_layout(L, wpt, resid);
    unsigned char* base = rf_smem + (size_t)grp * lay.bytes;
    Prep* prep = reinterpret_cast<Prep*>(base + lay.prep);
    float4(*seg)[31][2] = reinterpret_cast<float4(*)[31][2]>(base + lay.seg);
    float(*raw)[16] = reinterpret_cast<float(*)[16]>(base + lay.raw);
    float* madam = reinterpret_cast<float*>(base + lay.madam);
    float* vadam = reinterpret_cast<float*>(base + lay.vadam);
    float* msum = reinterpret_cast<float*>(base + lay.msum);
    float* quad = reinterpret_cast<float*>(base + lay.quad);
    float* hnode = reinterpret_cast<float*>(base + lay.hnode);
    float* hist = reinterpret_cast<float*>(base + lay.hist) + (size_t)wig * L * 96;
    float* gacc_all = reinterpret_cast<float*>(base + lay.gacc);
    float* gacc = gacc_all + (size_t)wig * L * 14;
    float* lacc = reinterpret_cast<float*>(base + lay.lacc) + (size_t)wig * L * 14 * 32;
    double* lred = reinterpret_cast<double*>(base + lay.lred);
    double* mom = reinterpret_cast<double*>(base + lay.mom);

    const int ts = set.size[t];
    const int p0 = set.prim_off[t];
    const int K = set.prim_off[t + 1] - p0;
    bool ok = ts >= 1 && ts <= 64 && K >= 0 && K <= L && (!CL1 || K <= 1);
    if (resid) ok = ok && (ts == 8 || ts == 16 || ts == 32 || ts == 64);
    if (!ok) {
        if (wig == 0 && lane == 0) {
            atomicCAS(&g_device_status, 0, WEFTK_E_ARG);
            if (loss) loss[t] = __int_as_float(0x7fc00000);
        }
        return;
    }
    // a lone constant layer runs in refine_const_kernel when the tiles' pixel sums are given
    if (CL1 && !resid && set.moments != nullptr && K == 1 && set.kind[p0] == K_CONST) return;
    const int gt = wig * 32 + lane, GT = wpt * 32;

    // ---- stage the layers (rows, and for STEP the Adam moments, stay in shared memory
    //      across the launch's steps; everything else is re-derived every step)
    for (int i = gt; i < K * 16; i += GT) {
        raw[i >> 4][i & 15] = params[(size_t)p0 * 16 + i];
        if (MODE == RF_STEP) {
            madam[i] = adam.m[(size_t)p0 * 16 + i];
            vadam[i] = adam.v[(size_t)p0 * 16 + i];
        }
    }
    const Layers S{prep, raw, seg};
    const float4* src = reinterpret_cast<const float4*>(set.src) + set.px_off[t];
    const int n = ts * ts;
    const int chunks = (n + 31) >> 5;
    const int c_begin = (chunks * wig) / wpt, c_end = (chunks * (wig + 1)) / wpt;
    // Residual-mode geometry (side a power of two >= 8): block side b, block pixels bb,
    // quadrant side h = b / 2, quadrant pixels Q = bb / 4.
    const int lb = resid ? (__ffs(ts) - 1) - 2 : 0;  // log2(b)
    const int b = 1 << lb, lbb = 2 * lb, bb = 1 << lbb;
    const int lq = resid ? lbb - 2 : 0, Q = 1 << lq, lh = resid ? lb - 1 : 0, h = 1 << lh;
    const float gscale = resid ? 4.0f / (float)ts : 0.0f;
    const float inv_bb = resid ? 1.0f / (float)bb : 0.0f;
    const int lts = (ts & (ts - 1)) == 0 ? __ffs(ts) - 1 : -1;  // log2(side) for power-of-two sides

    // pixel (x, y) of visit index q: row-major, or block-major / quadrant-major in residual mode
    auto pixel_of = [&](int q, int& x, int& y) {
        if (resid) {
            const int j = q >> lbb, o = q & (bb - 1), qd = o >> lq, u = o & (Q - 1);
            x = (j & 3) * b + (qd & 1) * h + (u & (h - 1));
            y = (j >> 2) * b + (qd >> 1) * h + (u >> lh);
        } else if (lts >= 0) {
            y = q >> lts;
            x = q & (ts - 1);
        } else {
            y = q / ts;
            x = q - y * ts;
        }
    };
    auto load_src = [&](int q) -> float4 {
        if (q >= n) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        int x, y;
        pixel_of(q, x, y);
        return src[y * ts + x];
    };
    auto composite = [&](float px, float py, float (&c)[3], float* hrow) {
        c[0] = c[1] = c[2] = 0.0f;
        if (CL1) {
            if (K == 1) {
                const ClEval v = eval_cl(prep[0], px, py);
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) c[ch] = blend(v.s[ch], v.a, 0.0f);
            }
            return;
        }
        for (int k = 0; k < K; ++k) {
            if (hrow) {
                float* hh = hrow + ((size_t)k * 32 + lane) * 3;
                hh[0] = c[0];
                hh[1] = c[1];
                hh[2] = c[2];
            }
            float sv[3], a;
            layer_eval(S, k, px, py, soft, sv, a);
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) c[ch] = blend(sv[ch], a, c[ch]);
        }
    };
    // decoded-error correction B M e at a pixel (block means in msum, already divided)
    auto correction = [&](int x, int y, float (&v)[3]) {
        int x0, x1, y0, y1;
        float wx, wy;
        grid_coord(x, gscale, x0, x1, wx);
        grid_coord(y, gscale, y0, y1, wy);
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            const float c00 = msum[(y0 * 4 + x0) * 3 + ch], c01 = msum[(y0 * 4 + x1) * 3 + ch];
            const float c10 = msum[(y1 * 4 + x0) * 3 + ch], c11 = msum[(y1 * 4 + x1) * 3 + ch];
            const float top = fmaf(c01 - c00, wx, c00), bot = fmaf(c11 - c10, wx, c10);
            v[ch] = fmaf(bot - top, wy, top);
        }
    };

    // A lone constant layer over black renders one colour q per channel (q = colour * alpha), so
    // its loss and gradient follow from the tile's pixel sums S1 = sum src, S2 = sum src^2:
    // sum over pixels of (q - src) = n q - S1, sum of (q - src)^2 = n q^2 - 2 q S1 + S2.  They are
    // taken once per launch (float64, a fixed order: per lane, then per warp, then per group).
    const bool cf = CL1 && !resid && K == 1 && set.kind[p0] == K_CONST;
    if (cf) {
        double m6[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int q = gt; q < n; q += GT) {
            const float4 v = src[q];
            m6[0] += v.x;
            m6[1] += v.y;
            m6[2] += v.z;
            m6[3] += (double)v.x * v.x;
            m6[4] += (double)v.y * v.y;
            m6[5] += (double)v.z * v.z;
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m6[i] += __shfl_xor_sync(FULL, m6[i], o);
        }
        if (lane == 0)
#pragma unroll
            for (int i = 0; i < 6; ++i) mom[wig * 6 + i] = m6[i];
        group_sync(wpt, grp);
        if (gt < 6) {
            double tot = 0.0;
            for (int w = 0; w < wpt; ++w) tot += mom[w * 6 + gt];
            mom[wpt * 6 + gt] = tot;
        }
    }
    const double* S12 = mom + wpt * 6;
    // loss (and, with g4, the colour / alpha gradient) of the lone constant layer
    auto const_closed = [&](float gscale, float* g4) -> double {
        return const_layer_closed(prep[0], raw[0][13], S12, n, gscale, g4);
    };

    double sse = 0.0;
    for (int step = 0; step < n_steps; ++step) {
    sse = 0.0;
    group_sync(wpt, grp);
    for (int k = gt; k < K; k += GT) {
        Prep P = prep_prim(row_to_prim(raw[k], set.kind[p0 + k]));
        if (P.kind == K_BICUBIC) P.kind = K_SKIP;
        prep[k] = P;
    }
    group_sync(wpt, grp);
    for (int i = gt; !CL1 && i < K * 31; i += GT) {
        const int k = i / 31, j = i - k * 31;
        if (prep[k].kind == K_CURVE) {
            const Seg g = lane_segment(prep[k], j);
            seg[k][j][0] = make_float4(g.ax, g.ay, g.vx, g.vy);
            seg[k][j][1] = make_float4(g.ux, g.uy, 0.0f, 0.0f);
        }
    }
    if (BWD) {
        for (int i = lane; i < K * 14; i += 32) gacc[i] = 0.0f;
        if (!CL1 && lane_acc)
            for (int i = lane; i < K * 14 * 32; i += 32) lacc[i] = 0.0f;
    }
    if (resid)
        for (int i = gt; i < 48 + 768; i += GT) {
            if (i < 48)
                msum[i] = 0.0f;
            else
                quad[i - 48] = 0.0f;
        }
    group_sync(wpt, grp);
    if (CL1 && K == 1 && gt == 0 && prep[0].kind != K_CONST && prep[0].kind != K_LINEAR && prep[0].kind != K_SKIP)
        atomicCAS(&g_device_status, 0, WEFTK_E_ARG);  // not a constant/linear layer: treated as absent

    if (resid) {
        // ---- pass 1: block sums of e (segments of bb visits; one owner per block)
        float4 vn = c_begin < c_end ? load_src(c_begin * 32 + lane) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (int cidx = c_begin; cidx < c_end; ++cidx) {
            const int q = cidx * 32 + lane;
            const float4 v = vn;
            if (cidx + 1 < c_end) vn = load_src(q + 32);
            int x, y;
            pixel_of(q, x, y);
            float c[3];
            composite((float)x + 0.5f, (float)y + 0.5f, c, nullptr);
            float e[3] = {clamp01(c[0]) - v.x, clamp01(c[1]) - v.y, clamp01(c[2]) - v.z};
            const int span = bb < 32 ? bb : 32;
            for (int o = 1; o < span; o <<= 1)
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) e[ch] += __shfl_xor_sync(FULL, e[ch], o);
            if ((lane & (span - 1)) == 0) {
                const int j = q >> lbb;
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) msum[j * 3 + ch] += e[ch];
            }
        }
        group_sync(wpt, grp);
        for (int i = gt; i < 48; i += GT) msum[i] *= inv_bb;
        group_sync(wpt, grp);
        // ---- pass 2: r = e - B M e; loss; per-quadrant sums of (bilinear weight x r)
        vn = c_begin < c_end ? load_src(c_begin * 32 + lane) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (int cidx = c_begin; cidx < c_end; ++cidx) {
            const int q = cidx * 32 + lane;
            const float4 v = vn;
            if (cidx + 1 < c_end) vn = load_src(q + 32);
            int x, y;
            pixel_of(q, x, y);
            float c[3], corr[3];
            composite((float)x + 0.5f, (float)y + 0.5f, c, nullptr);
            correction(x, y, corr);
            const float r[3] = {clamp01(c[0]) - v.x - corr[0], clamp01(c[1]) - v.y - corr[1],
                                clamp01(c[2]) - v.z - corr[2]};
            sse += (double)fmaf(r[0], r[0], fmaf(r[1], r[1], r[2] * r[2]));
            if (BWD) {
                int x0, x1, y0, y1;
                float wx, wy;
                grid_coord(x, gscale, x0, x1, wx);
                grid_coord(y, gscale, y0, y1, wy);
                const float w4[4] = {(1.0f - wx) * (1.0f - wy), wx * (1.0f - wy), (1.0f - wx) * wy, wx * wy};
                float acc[12];
#pragma unroll
                for (int s4 = 0; s4 < 4; ++s4)
#pragma unroll
                    for (int ch = 0; ch < 3; ++ch) acc[s4 * 3 + ch] = w4[s4] * r[ch];
                const int span = Q < 32 ? Q : 32;
                for (int o = 1; o < span; o <<= 1)
#pragma unroll
                    for (int i = 0; i < 12; ++i) acc[i] += __shfl_xor_sync(FULL, acc[i], o);
                if ((lane & (span - 1)) == 0) {
                    const int qi = q >> lq;  // quadrant index, block-major
#pragma unroll
                    for (int i = 0; i < 12; ++i) quad[qi * 12 + i] += acc[i];
                }
            }
        }
        if (BWD) {
            group_sync(wpt, grp);
            // B^T r per node: sum of the (column, slot) x (row, slot) quadrant entries that
            // interpolate from this node.
            for (int i = gt; i < 48; i += GT) {
                const int node = i / 3, ch = i - node * 3;
                int sx[4], sy[4];
                const int nsx = node_sources(node & 3, sx), nsy = node_sources(node >> 2, sy);
                float acc = 0.0f;
                for (int a = 0; a < nsy; ++a) {
                    const int qy = sy[a] >> 1, sly = sy[a] & 1;
                    for (int c = 0; c < nsx; ++c) {
                        const int qx = sx[c] >> 1, slx = sx[c] & 1;
                        const int qi = (((qy >> 1) * 4 + (qx >> 1)) << 2) + ((qy & 1) << 1) + (qx & 1);
                        acc += quad[qi * 12 + (sly * 2 + slx) * 3 + ch];
                    }
                }
                hnode[i] = acc * inv_bb;
            }
            group_sync(wpt, grp);
        }
    }

    if (BWD) {
        // ---- backward pass
        const float scale = grad_loss[t] * 2.0f / (3.0f * (float)n);
        float4 vn = c_begin < c_end ? load_src(c_begin * 32 + lane) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        float acc[14];
#pragma unroll
        for (int i = 0; i < 14; ++i) acc[i] = 0.0f;
        if (cf && gt == 0) {
            float g4[4];
            sse = const_closed(scale, g4);
            gacc[7] = g4[0];
            gacc[8] = g4[1];
            gacc[9] = g4[2];
            gacc[13] = g4[3];
        }
        for (int cidx = c_begin; CL1 && !cf && cidx < c_end; ++cidx) {
            // single constant/linear layer over black: everything in registers
            const int q = cidx * 32 + lane;
            const float4 v4 = vn;
            if (cidx + 1 < c_end) vn = load_src(q + 32);
            if (q >= n || K == 0) {
                continue;
            }
            int x, y;
            pixel_of(q, x, y);
            const float px = (float)x + 0.5f, py = (float)y + 0.5f;
            const ClEval v = eval_cl(prep[0], px, py);
            float c[3], e[3], g[3];
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) c[ch] = blend(v.s[ch], v.a, 0.0f);
            e[0] = clamp01(c[0]) - v4.x;
            e[1] = clamp01(c[1]) - v4.y;
            e[2] = clamp01(c[2]) - v4.z;
            if (resid) {
                float corr[3];
                correction(x, y, corr);
                const int j = q >> lbb;
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) e[ch] = e[ch] - corr[ch] - hnode[j * 3 + ch];
            } else {
                sse += (double)fmaf(e[0], e[0], fmaf(e[1], e[1], e[2] * e[2]));
            }
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) g[ch] = (c[ch] >= 0.0f && c[ch] <= 1.0f) ? scale * e[ch] : 0.0f;
            grad_cl(prep[0], raw[0], v, px, py, g, acc);
        }
        if (CL1 && K == 1 && !cf) {
            const unsigned cols = grad_columns(prep[0].kind);
#pragma unroll
            for (int i = 0; i < 14; ++i) {
                if (!((cols >> i) & 1u)) continue;
                float s2 = acc[i];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(FULL, s2, o);
                if (lane == 0) gacc[i] = s2;
            }
        }
        for (int cidx = c_begin; !CL1 && cidx < c_end; ++cidx) {
            const int q = cidx * 32 + lane;
            const bool valid = q < n;
            const float4 v = vn;
            if (cidx + 1 < c_end) vn = load_src(q + 32);
            int x, y;
            pixel_of(q, x, y);
            const float px = (float)x + 0.5f, py = (float)y + 0.5f;
            float c[3];
            composite(px, py, c, hist);
            float g[3] = {0.0f, 0.0f, 0.0f};
            if (valid) {
                float e[3] = {clamp01(c[0]) - v.x, clamp01(c[1]) - v.y, clamp01(c[2]) - v.z};
                if (resid) {
                    float corr[3];
                    correction(x, y, corr);
                    const int j = q >> lbb;
#pragma unroll
                    for (int ch = 0; ch < 3; ++ch) e[ch] = e[ch] - corr[ch] - hnode[j * 3 + ch];
                } else {
                    sse += (double)fmaf(e[0], e[0], fmaf(e[1], e[1], e[2] * e[2]));
                }
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) g[ch] = (c[ch] >= 0.0f && c[ch] <= 1.0f) ? scale * e[ch] : 0.0f;
            }
            for (int k = K - 1; k >= 0; --k) {
                const float* hh = hist + ((size_t)k * 32 + lane) * 3;
                const float cp[3] = {hh[0], hh[1], hh[2]};
                float d[14], a;
                layer_grad(S, k, px, py, soft, g, cp, a, d);
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) g[ch] *= (1.0f - a);
                const unsigned cols = grad_columns(prep[k].kind);
                if (lane_acc) {
                    float* la = lacc + (size_t)k * 14 * 32 + lane;
#pragma unroll
                    for (int i = 0; i < 14; ++i)
                        if ((cols >> i) & 1u) la[i * 32] += d[i];
                } else {
#pragma unroll
                    for (int i = 0; i < 14; ++i) {
                        if (!((cols >> i) & 1u)) continue;
                        float s = d[i];
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
                        if (lane == 0) gacc[k * 14 + i] += s;
                    }
                }
            }
        }
        if (!CL1 && lane_acc) {
            // lane j sums slot j's 32 lane partials, starting at lane j (no bank conflicts)
            __syncwarp();
            for (int j = lane; j < K * 14; j += 32) {
                const float* la = lacc + (size_t)j * 32;
                float s = 0.0f;
                for (int l = 0; l < 32; ++l) s += la[(l + j) & 31];
                gacc[j] = s;
            }
        }
        if (MODE == RF_STEP)  // each row's bias corrections for this step, once (column 14 is free)
            for (int k = gt; k < K; k += GT) adam_bias(adam.b1, adam.b2, madam[k * 16 + 15] + 1.0f,
                                                       madam[k * 16 + 14], vadam[k * 16 + 14]);
        group_sync(wpt, grp);
        for (int i = gt; i < K * 16; i += GT) {
            const int k = i >> 4, j = i & 15;
            float s = 0.0f;
            if (j < 14)
                for (int w = 0; w < wpt; ++w) s += gacc_all[((size_t)w * L + k) * 14 + j];
            const size_t at = (size_t)(p0 + k) * 16 + j;
            if (grad && step == n_steps - 1) grad[at] = s;
            if (MODE == RF_STEP && j < 14) {
                float m = madam[k * 16 + j], v = vadam[k * 16 + j];
                raw[k][j] = adam_update_bc(raw[k][j], s, m, v, madam[k * 16 + 14], vadam[k * 16 + 14], adam.lr,
                                           adam.b1, adam.b2, adam.eps, set.kind[p0 + k], j);
                madam[k * 16 + j] = m;
                vadam[k * 16 + j] = v;
            }
        }
        if (MODE == RF_STEP) {
            group_sync(wpt, grp);  // every column of a row has read its step count
            for (int k = gt; k < K; k += GT) madam[k * 16 + 15] += 1.0f;
        }
    } else if (!resid) {
        if (cf && gt == 0) sse = const_closed(0.0f, nullptr);
        float4 vn = c_begin < c_end && !cf ? load_src(c_begin * 32 + lane) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (int cidx = c_begin; !cf && cidx < c_end; ++cidx) {
            const int q = cidx * 32 + lane;
            const float4 v = vn;
            if (cidx + 1 < c_end) vn = load_src(q + 32);
            if (q >= n) continue;
            int x, y;
            pixel_of(q, x, y);
            float c[3];
            composite((float)x + 0.5f, (float)y + 0.5f, c, nullptr);
            const float dr = clamp01(c[0]) - v.x, dg = clamp01(c[1]) - v.y, db = clamp01(c[2]) - v.z;
            sse += (double)fmaf(dr, dr, fmaf(dg, dg, db * db));
        }
    }
    }  // steps
    if (MODE == RF_STEP) {
        group_sync(wpt, grp);
        for (int i = gt; i < K * 16; i += GT) {
            const bool scratch = (i & 15) == 14;  // bias-correction scratch, not state
            params[(size_t)p0 * 16 + i] = raw[i >> 4][i & 15];
            adam.m[(size_t)p0 * 16 + i] = scratch ? 0.0f : madam[i];
            adam.v[(size_t)p0 * 16 + i] = scratch ? 0.0f : vadam[i];
        }
    }
    if (loss != nullptr) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sse += __shfl_xor_sync(FULL, sse, o);
        if (lane == 0) lred[wig] = sse;
        group_sync(wpt, grp);
        if (gt == 0) {
            double tot = 0.0;
            for (int w = 0; w < wpt; ++w) tot += lred[w];
            loss[t] = (float)(tot / (3.0 * n));
        }
    }
}

// One thread per tile whose stack is one constant layer (register path, primitives-only loss,
// the tiles' pixel sums given): the same arithmetic as refine_tiles_kernel's closed form for such a
// tile — loss n q^2 - 2 q S1 + S2 and gradient from n q - S1 per channel, Adam with projection on
// the row's colour and alpha (its other columns have zero gradient and stay where they are), the
// row's step count and bias corrections as the group path keeps them.
template <int MODE>
__global__ void __launch_bounds__(128) refine_const_kernel(WeftStackSet set, float* __restrict__ params,
                                                           const float* __restrict__ grad_loss,
                                                           float* __restrict__ grad, float* __restrict__ loss,
                                                           AdamArgs adam, int n_steps) {
    constexpr bool BWD = MODE != RF_LOSS;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= set.n_tiles) return;
    const int p0 = set.prim_off[t];
    if (set.prim_off[t + 1] - p0 != 1 || set.kind[p0] != K_CONST) return;
    const int ts = set.size[t];
    if (ts < 1 || ts > 64) return;  // reported by refine_tiles_kernel
    const int n = ts * ts;
    double S[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) S[i] = set.moments[(size_t)t * 6 + i];
    float* row = params + (size_t)p0 * 16;
    float r[16], m[16], v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        r[i] = row[i];
        m[i] = MODE == RF_STEP ? adam.m[(size_t)p0 * 16 + i] : 0.0f;
        v[i] = MODE == RF_STEP ? adam.v[(size_t)p0 * 16 + i] : 0.0f;
    }
    const float scale = BWD ? grad_loss[t] * 2.0f / (3.0f * (float)n) : 0.0f;
    // Columns other than the colour (7..9) and alpha (13) have zero gradient.  Where their moments
    // start at zero an Adam update leaves them at zero and moves the value by exactly 0, so such a
    // column only takes the projection, at the first step.
    unsigned idle = 0;
#pragma unroll
    for (int j = 0; j < 14; ++j)
        if (!(j >= 7 && j <= 9) && j != 13 && m[j] == 0.0f && v[j] == 0.0f) idle |= 1u << j;
    double sse = 0.0;
    float g4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int step = 0; step < n_steps; ++step) {
        const Prep P = prep_prim(row_to_prim(r, K_CONST));
        const double tot = const_layer_closed(P, r[13], S, n, scale, g4);
        sse = tot;
        if (MODE == RF_STEP) {
            adam_bias(adam.b1, adam.b2, m[15] + 1.0f, m[14], v[14]);
#pragma unroll
            for (int j = 0; j < 14; ++j) {
                if ((idle >> j) & 1u) {
                    if (step == 0) r[j] = adam_project(r[j], K_CONST, j);
                    continue;
                }
                const float gj = j >= 7 && j <= 9 ? g4[j - 7] : j == 13 ? g4[3] : 0.0f;
                r[j] = adam_update_bc(r[j], gj, m[j], v[j], m[14], v[14], adam.lr, adam.b1, adam.b2, adam.eps,
                                     K_CONST, j);
            }
            m[15] += 1.0f;
        }
    }
    if (BWD && grad) {
#pragma unroll
        for (int j = 0; j < 16; ++j)
            grad[(size_t)p0 * 16 + j] = j >= 7 && j <= 9 ? g4[j - 7] : j == 13 ? g4[3] : 0.0f;
    }
    if (MODE == RF_STEP) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            row[i] = r[i];
            adam.m[(size_t)p0 * 16 + i] = i == 14 ? 0.0f : m[i];
            adam.v[(size_t)p0 * 16 + i] = i == 14 ? 0.0f : v[i];
        }
    }
    if (loss != nullptr) loss[t] = (float)(sse / (3.0 * n));
}

// A side stream of the current device for the calling host thread, with the two events that fork
// work onto it and join it back.  Created on first use and kept for the life of the process (one
// per host thread and device, so concurrent callers never share the events).
struct SideStream {
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};

static int side_stream(SideStream** out) {
    thread_local std::map<int, SideStream> per_device;
    int dev = 0;
    WEFTK_CUDA(cudaGetDevice(&dev));
    SideStream& s = per_device[dev];
    if (s.stream == nullptr) {
        WEFTK_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
        WEFTK_CUDA(cudaEventCreateWithFlags(&s.fork, cudaEventDisableTiming));
        WEFTK_CUDA(cudaEventCreateWithFlags(&s.join, cudaEventDisableTiming));
    }
    *out = &s;
    return WEFTK_OK;
}

template <int MODE>
static int launch_refine(const WeftStackSet& set, float* params, const float* grad_loss, float* grad, float* loss,
                         int flags, AdamArgs adam, cudaStream_t stream, const char* what, int n_steps = 1) {
    if (n_steps < 1 || (MODE != RF_STEP && n_steps != 1)) return fail(WEFTK_E_ARG, std::string(what) + ": bad step count");
    if (set.n_tiles == 0) return WEFTK_OK;
    if (set.max_prims < 0 || set.max_prims > MAXL) return fail(WEFTK_E_RANGE, std::string(what) + ": stack too long");
    if (!params || !set.src || !set.px_off || !set.size || !set.prim_off || (set.max_prims > 0 && !set.kind))
        return fail(WEFTK_E_ARG, std::string(what) + ": null pointer in the stack set");
    const int L = set.max_prims > 0 ? set.max_prims : 1;
    RefinePlan plan{};
    int counts[RF_CLASSES] = {0, 0, 0, 0};
    if (set.order == nullptr) {
        counts[1] = set.n_tiles;  // no split: four warps per tile
    } else {
        if (set.n_big < 0 || set.n_mid < 0 || set.n_s16 < 0 ||
            (long long)set.n_big + set.n_mid + set.n_s16 > set.n_tiles)
            return fail(WEFTK_E_ARG, std::string(what) + ": bad size-class counts");
        counts[0] = set.n_big;
        counts[1] = set.n_mid;
        counts[2] = set.n_s16;
        counts[3] = set.n_tiles - set.n_big - set.n_mid - set.n_s16;
    }
    int smem = 0, ctas = 0, off = 0;
    for (int c = 0; c < RF_CLASSES; ++c) {
        const int wpt = class_wpt(c);
        const int bytes = group_layout(L, wpt, (flags & WEFTK_LOSS_RESIDUAL) != 0).bytes;
        const int g = std::min(8 / wpt, RF_SMEM_MAX / bytes);
        plan.groups[c] = g;
        plan.list_off[c] = off;
        plan.n_list[c] = counts[c];
        off += counts[c];
        ctas += (counts[c] + g - 1) / g;
        plan.cta_end[c] = ctas;
        if (counts[c]) smem = std::max(smem, g * bytes);
    }
    // single constant/linear layers only (declared by the caller, checked per tile): register path
    const bool cl1 = set.max_prims <= 1 && set.kinds_mask != 0 && (set.kinds_mask & ~0x3) == 0;
    // the dynamic shared-memory opt-in is per device and per kernel instance: remember the
    // largest size set on each device (under a lock, so concurrent first calls agree)
    {
        int dev = 0;
        WEFTK_CUDA(cudaGetDevice(&dev));
        static std::mutex mu;
        static std::map<int, int> granted[2];
        std::lock_guard<std::mutex> lock(mu);
        int& have = granted[cl1].try_emplace(dev, 48 * 1024).first->second;
        if (smem > have) {
            if (cl1)
                WEFTK_CUDA(cudaFuncSetAttribute(refine_tiles_kernel<MODE, true>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            else
                WEFTK_CUDA(cudaFuncSetAttribute(refine_tiles_kernel<MODE, false>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            have = smem;
        }
    }
    // lone constant layers (closed form, a thread per tile) run beside the other tiles' launch, on
    // this thread's side stream of the device (forked from and joined back into `stream`, which a
    // CUDA graph capture follows)
    const bool const_side = cl1 && set.moments != nullptr && !(flags & WEFTK_LOSS_RESIDUAL);
    SideStream* side = nullptr;
    if (const_side) {
        int rc = side_stream(&side);
        if (rc) return rc;
        WEFTK_CUDA(cudaEventRecord(side->fork, stream));
        WEFTK_CUDA(cudaStreamWaitEvent(side->stream, side->fork, 0));
        refine_const_kernel<MODE><<<(set.n_tiles + 127) / 128, 128, 0, side->stream>>>(set, params, grad_loss, grad,
                                                                                        loss, adam, n_steps);
        WEFTK_CUDA(cudaGetLastError());
        WEFTK_CUDA(cudaEventRecord(side->join, side->stream));
    }
    if (cl1)
        refine_tiles_kernel<MODE, true><<<ctas, RF_THREADS, smem, stream>>>(set, params, grad_loss, grad, loss, flags,
                                                                            plan, L, adam, n_steps);
    else
        refine_tiles_kernel<MODE, false><<<ctas, RF_THREADS, smem, stream>>>(set, params, grad_loss, grad, loss,
                                                                             flags, plan, L, adam, n_steps);
    WEFTK_CUDA(cudaGetLastError());
    if (side) WEFTK_CUDA(cudaStreamWaitEvent(stream, side->join, 0));
    return WEFTK_OK;
}

// Row r of a refinement started from a fit: thread per (row, column).
__global__ void refine_start_kernel(WeftFitState fit, const int* __restrict__ tiles, int n_rows,
                                    float* __restrict__ params, float* __restrict__ m, float* __restrict__ v,
                                    int* __restrict__ kind_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_rows * 16) return;
    const int row = i >> 4, col = i & 15;
    const int t = tiles[row];
    m[i] = 0.0f;
    v[i] = 0.0f;
    float x = 0.0f;
    int kind = -1;
    if (t >= 0 && t < fit.n_tiles && fit.n_sel[t] >= 1) {
        const int sel = fit.sel[(size_t)t * fit.cap_max];
        const WeftPrim& P = fit.cand[fit.pool_off[t] + sel];
        kind = P.kind;
        if (col < 7) {
            const bool thick = (kind == K_LINE && col == 4) || (kind == K_CURVE && col == 6);
            x = fminf(fmaxf(P.geom[col], 0.0f), thick ? 4.0f : 15.0f);
        } else if (col < 14) {
            const float c = col < 10 ? P.color0[col - 7] : col < 13 ? P.color1[col - 10] : P.alpha;
            x = fminf(fmaxf(c, 0.0f), 1.0f);
        }
    } else if (t < 0 || t >= fit.n_tiles) {
        if (col == 0) atomicCAS(&g_device_status, 0, WEFTK_E_ARG);
    }
    params[i] = x;
    if (col == 0) kind_out[row] = kind;
}

// Adam (PyTorch's rule) + projection onto the wire-representable box, one thread per value.
__global__ void adam_project_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                    float* __restrict__ v, const int* __restrict__ kind, int n_rows, float lr,
                                    float b1, float b2, float eps, const int* __restrict__ step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_rows * 16) return;
    const int col = i & 15, row = i >> 4;
    if (col >= 14) return;
    float mi = m[i], vi = v[i];
    p[i] = adam_update(p[i], g[i], mi, vi, (float)(*step + 1), lr, b1, b2, eps, kind[row], col);
    m[i] = mi;
    v[i] = vi;
}

__global__ void step_increment_kernel(int* step) { *step += 1; }

}  // namespace weftk

using namespace weftk;

extern "C" int weftk_stack_loss(const WeftStackSet* set, const float* d_params, float* d_loss, int flags,
                                void* stream) {
    WEFTK_REQUIRE(set && d_loss, "stack_loss: null argument");
    return launch_refine<RF_LOSS>(*set, const_cast<float*>(d_params), nullptr, nullptr, d_loss, flags, AdamArgs{},
                                  (cudaStream_t)stream, "stack_loss");
}

extern "C" int weftk_refine_start(const WeftFitState* fit, const int32_t* d_tiles, int n_rows, float* d_params,
                                  float* d_m, float* d_v, int32_t* d_kind, void* stream) {
    WEFTK_REQUIRE(fit && n_rows >= 0, "refine_start: bad arguments");
    if (n_rows == 0) return WEFTK_OK;
    WEFTK_REQUIRE(d_tiles && d_params && d_m && d_v && d_kind, "refine_start: null pointer");
    const int n = n_rows * 16;
    refine_start_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(*fit, d_tiles, n_rows, d_params, d_m, d_v,
                                                                            d_kind);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}

extern "C" int weftk_adam_step(float* d_params, const float* d_grads, float* d_m, float* d_v, const int32_t* d_kind,
                               int n_rows, float lr, float beta1, float beta2, float eps, int32_t* d_step,
                               void* stream) {
    WEFTK_REQUIRE(n_rows >= 0 && (n_rows == 0 || (d_params && d_grads && d_m && d_v && d_kind && d_step)),
                  "adam_step: bad arguments");
    if (n_rows == 0) return WEFTK_OK;
    const int n = n_rows * 16;
    adam_project_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_params, d_grads, d_m, d_v, d_kind, n_rows,
                                                                            lr, beta1, beta2, eps, d_step);
    step_increment_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(d_step);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}

extern "C" int weftk_stack_loss_backward(const WeftStackSet* set, const float* d_params, const float* d_grad_loss,
                                         float* d_grad_params, float* d_loss, int flags, void* stream) {
    WEFTK_REQUIRE(set && d_grad_loss && d_grad_params, "stack_loss_backward: null argument");
    return launch_refine<RF_GRAD>(*set, const_cast<float*>(d_params), d_grad_loss, d_grad_params, d_loss, flags,
                                  AdamArgs{}, (cudaStream_t)stream, "stack_loss_backward");
}

extern "C" int weftk_refine_step(const WeftStackSet* set, float* d_params, float* d_m, float* d_v,
                                 const float* d_grad_loss, float* d_loss, float* d_grad_params, float lr, float beta1,
                                 float beta2, float eps, int flags, void* stream) {
    WEFTK_REQUIRE(set && d_params && d_m && d_v && d_grad_loss, "refine_step: null argument");
    return launch_refine<RF_STEP>(*set, d_params, d_grad_loss, d_grad_params, d_loss, flags,
                                  AdamArgs{d_m, d_v, lr, beta1, beta2, eps}, (cudaStream_t)stream, "refine_step");
}

extern "C" int weftk_refine_steps(const WeftStackSet* set, int steps, float* d_params, float* d_m, float* d_v,
                                  const float* d_grad_loss, float* d_loss, float* d_grad_params, float lr, float beta1,
                                  float beta2, float eps, int flags, void* stream) {
    WEFTK_REQUIRE(set && d_params && d_m && d_v && d_grad_loss && steps >= 1, "refine_steps: bad argument");
    return launch_refine<RF_STEP>(*set, d_params, d_grad_loss, d_grad_params, d_loss, flags,
                                  AdamArgs{d_m, d_v, lr, beta1, beta2, eps}, (cudaStream_t)stream, "refine_steps",
                                  steps);
}
