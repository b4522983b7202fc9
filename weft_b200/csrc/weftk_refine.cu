// weftk_refine.cu — per-tile stack loss and its hand-written backward (see include/weftk_refine.h).
//
// One CTA per tile; the tile's parameter rows are prepared once into shared
// memory (and a curve's 31 polyline segments into a segment table).  Each
// thread owns one pixel of a chunk.  The backward re-renders the chunk's pixels
// front to back, keeping the composite *before* every layer in shared memory
// (layers x threads x 3 floats, the only per-pixel state, never written to HBM),
// then sweeps the layers back to front:
//     c_k = s_k a_k + c_{k-1} (1 - a_k)
//     dL/ds_k = g a_k,  dL/da_k = g . (s_k - c_{k-1}),  g <- g (1 - a_k)
// and chains dL/ds, dL/da into the layer's parameters with the coverage
// recomputed at that pixel.  Per-layer gradients are reduced over the CTA in a
// fixed order, so results are deterministic.
#include <cuda_runtime.h>

#include "../../include/weftk_refine.h"
#include "weftk_common.cuh"
#include "weftk_prim.cuh"

namespace weftk {

extern __device__ int g_device_status;

constexpr int RF_THREADS = 128;
constexpr int RF_WARPS = RF_THREADS / 32;
constexpr int MAXL = WEFTK_REFINE_MAX_PRIMS;
constexpr float TRI_SOFT_W = 0.5f;  // surrogate edge width in pixels

struct RfShared {
    Prep prep[MAXL];
    float raw[MAXL][16];
    float4 seg[MAXL][31][2];
    float red[RF_WARPS][14];
    float gacc[MAXL][14];
    double lred[RF_WARPS];
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

// Stage the tile's rows: raw parameters, prepared terms, curve segment tables.
__device__ bool stage_tile(const WeftStackSet& set, const float* params, int t, RfShared& s, int& K) {
    const int p0 = set.prim_off[t];
    K = set.prim_off[t + 1] - p0;
    if (K < 0 || K > MAXL) return false;
    for (int i = threadIdx.x; i < K * 16; i += blockDim.x) s.raw[i / 16][i % 16] = params[(size_t)p0 * 16 + i];
    __syncthreads();
    if ((int)threadIdx.x < K) {
        const int k = threadIdx.x;
        Prep P = prep_prim(row_to_prim(s.raw[k], set.kind[p0 + k]));
        if (P.kind == K_BICUBIC) P.kind = K_SKIP;
        s.prep[k] = P;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < K * 31; i += blockDim.x) {
        const int k = i / 31, j = i % 31;
        if (s.prep[k].kind == K_CURVE) {
            const Seg g = lane_segment(s.prep[k], j);
            s.seg[k][j][0] = make_float4(g.ax, g.ay, g.vx, g.vy);
            s.seg[k][j][1] = make_float4(g.ux, g.uy, 0.0f, 0.0f);
        }
    }
    for (int i = threadIdx.x; i < K * 14; i += blockDim.x) s.gacc[i / 14][i % 14] = 0.0f;
    __syncthreads();
    return true;
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
__device__ __forceinline__ void layer_eval(const RfShared& s, int k, float px, float py, bool soft, float (&src)[3],
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
__device__ void layer_grad(const RfShared& s, int k, float px, float py, bool soft, const float (&g)[3],
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

__global__ void __launch_bounds__(RF_THREADS) stack_loss_kernel(WeftStackSet set, const float* __restrict__ params,
                                                                float* __restrict__ loss, int flags) {
    __shared__ RfShared s;
    const int t = blockIdx.x;
    int K = 0;
    const int ts = set.size[t];
    if (ts <= 0 || ts > 64 || !stage_tile(set, params, t, s, K)) {
        if (threadIdx.x == 0) {
            atomicCAS(&g_device_status, 0, WEFTK_E_ARG);
            loss[t] = __int_as_float(0x7fc00000);
        }
        return;
    }
    const bool soft = flags & WEFTK_SOFT_TRIANGLES;
    const float4* src = reinterpret_cast<const float4*>(set.src) + set.px_off[t];
    const int n = ts * ts;
    double acc = 0.0;
    for (int p = threadIdx.x; p < n; p += RF_THREADS) {
        const float px = (float)(p % ts) + 0.5f, py = (float)(p / ts) + 0.5f;
        float c[3] = {0.0f, 0.0f, 0.0f};
        for (int k = 0; k < K; ++k) {
            float sv[3], a;
            layer_eval(s, k, px, py, soft, sv, a);
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) c[ch] = blend(sv[ch], a, c[ch]);
        }
        const float4 v = src[p];
        const float dr = clamp01(c[0]) - v.x, dg = clamp01(c[1]) - v.y, db = clamp01(c[2]) - v.z;
        acc += (double)fmaf(dr, dr, fmaf(dg, dg, db * db));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
    if ((threadIdx.x & 31) == 0) s.lred[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < RF_WARPS; ++w) tot += s.lred[w];
        loss[t] = (float)(tot / (3.0 * n));
    }
}

__global__ void __launch_bounds__(RF_THREADS) stack_backward_kernel(WeftStackSet set, const float* __restrict__ params,
                                                                    const float* __restrict__ grad_loss,
                                                                    float* __restrict__ grad, float* __restrict__ loss,
                                                                    int flags) {
    extern __shared__ float hist[];  // [K][RF_THREADS][3]: composite before each layer
    __shared__ RfShared s;
    const int t = blockIdx.x;
    int K = 0;
    const int ts = set.size[t];
    if (ts <= 0 || ts > 64 || !stage_tile(set, params, t, s, K)) {
        if (threadIdx.x == 0) atomicCAS(&g_device_status, 0, WEFTK_E_ARG);
        return;
    }
    const bool soft = flags & WEFTK_SOFT_TRIANGLES;
    const float4* src = reinterpret_cast<const float4*>(set.src) + set.px_off[t];
    const int n = ts * ts, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float scale = grad_loss[t] * 2.0f / (3.0f * (float)n);
    double sse = 0.0;
    for (int base = 0; base < n; base += RF_THREADS) {
        const int p = base + tid;
        const bool valid = p < n;
        const float px = (float)(p % ts) + 0.5f, py = (float)(p / ts) + 0.5f;
        float c[3] = {0.0f, 0.0f, 0.0f};
        for (int k = 0; k < K; ++k) {
            float* h = hist + ((size_t)k * RF_THREADS + tid) * 3;
            h[0] = c[0];
            h[1] = c[1];
            h[2] = c[2];
            float sv[3], a;
            layer_eval(s, k, px, py, soft, sv, a);
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) c[ch] = blend(sv[ch], a, c[ch]);
        }
        float g[3] = {0.0f, 0.0f, 0.0f};
        if (valid) {
            const float4 v = src[p];
            const float sv[3] = {v.x, v.y, v.z};
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) {
                const float e = clamp01(c[ch]) - sv[ch];
                sse += (double)(e * e);
                g[ch] = (c[ch] >= 0.0f && c[ch] <= 1.0f) ? scale * e : 0.0f;
            }
        }
        for (int k = K - 1; k >= 0; --k) {
            const float* h = hist + ((size_t)k * RF_THREADS + tid) * 3;
            const float cp[3] = {h[0], h[1], h[2]};
            float d[14], a;
            layer_grad(s, k, px, py, soft, g, cp, a, d);
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) g[ch] *= (1.0f - a);
#pragma unroll
            for (int i = 0; i < 14; ++i) {
                float v = d[i];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
                if (lane == 0) s.red[warp][i] = v;
            }
            __syncthreads();
            if (tid < 14) {
                float v = s.red[0][tid];
                for (int w = 1; w < RF_WARPS; ++w) v += s.red[w][tid];
                s.gacc[k][tid] += v;
            }
            __syncthreads();
        }
    }
    const int p0 = set.prim_off[t];
    for (int i = tid; i < K * 16; i += RF_THREADS) {
        const int k = i / 16, j = i % 16;
        grad[(size_t)(p0 + k) * 16 + j] = j < 14 ? s.gacc[k][j] : 0.0f;
    }
    if (loss != nullptr) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sse += __shfl_xor_sync(FULL, sse, o);
        if (lane == 0) s.lred[warp] = sse;
        __syncthreads();
        if (tid == 0) {
            double tot = 0.0;
            for (int w = 0; w < RF_WARPS; ++w) tot += s.lred[w];
            loss[t] = (float)(tot / (3.0 * n));
        }
    }
}

// Adam (PyTorch's rule) + projection onto the wire-representable box, one thread per value.
__global__ void adam_project_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                    float* __restrict__ v, const int* __restrict__ kind, int n_rows, float lr,
                                    float b1, float b2, float eps, const int* __restrict__ step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_rows * 16) return;
    const int col = i & 15, row = i >> 4;
    if (col >= 14) return;
    const float t = (float)(*step + 1);
    const float gi = g[i];
    const float mi = fmaf(b1, m[i], (1.0f - b1) * gi);
    const float vi = fmaf(b2, v[i], (1.0f - b2) * gi * gi);
    m[i] = mi;
    v[i] = vi;
    const float bc1 = 1.0f - powf(b1, t), bc2 = 1.0f - powf(b2, t);
    float x = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    const int k = kind[row];
    if (col >= 7) {
        x = fminf(fmaxf(x, 0.0f), 1.0f);
    } else {
        const bool thick = (k == K_LINE && col == 4) || (k == K_CURVE && col == 6);
        x = fminf(fmaxf(x, 0.0f), thick ? 4.0f : 15.0f);
    }
    p[i] = x;
}

__global__ void step_increment_kernel(int* step) { *step += 1; }

}  // namespace weftk

using namespace weftk;

extern "C" int weftk_stack_loss(const WeftStackSet* set, const float* d_params, float* d_loss, int flags,
                                void* stream) {
    WEFTK_REQUIRE(set && d_loss, "stack_loss: null argument");
    if (set->n_tiles == 0) return WEFTK_OK;
    WEFTK_REQUIRE(set->max_prims >= 0 && set->max_prims <= WEFTK_REFINE_MAX_PRIMS, "stack_loss: stack too long");
    stack_loss_kernel<<<set->n_tiles, RF_THREADS, 0, (cudaStream_t)stream>>>(*set, d_params, d_loss, flags);
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
    if (set->n_tiles == 0) return WEFTK_OK;
    WEFTK_REQUIRE(set->max_prims >= 0 && set->max_prims <= WEFTK_REFINE_MAX_PRIMS,
                  "stack_loss_backward: stack too long");
    const int smem = (set->max_prims > 0 ? set->max_prims : 1) * RF_THREADS * 3 * (int)sizeof(float);
    static int attr = 0;
    if (smem > attr) {
        WEFTK_CUDA(cudaFuncSetAttribute(stack_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        MAXL * RF_THREADS * 3 * (int)sizeof(float)));
        attr = MAXL * RF_THREADS * 3 * (int)sizeof(float);
    }
    stack_backward_kernel<<<set->n_tiles, RF_THREADS, smem, (cudaStream_t)stream>>>(*set, d_params, d_grad_loss,
                                                                                     d_grad_params, d_loss, flags);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}
