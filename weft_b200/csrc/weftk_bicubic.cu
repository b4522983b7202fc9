// weftk_bicubic.cu — the per-tile bicubic R-D swap of the adaptive fit
// (src/weft/encoder.py:2841-2873): least-squares 4x4x3 Bezier grid per tile, rounded to u8
// steps, evaluated and scored against the tile's selected stack.
//
// One 128-thread CTA per tile.  The fit is pinv(B) @ T @ pinv(B^T) per channel in float64,
// associated left to right as the reference's numpy expression is: threads own columns x of
// L = pinv(B) @ T (4 x n x 3, in shared memory), then 48 threads form the control grid.  The
// evaluation is (B @ Q) @ B^T, again left to right; its squared error and the stack's (the
// stack rendered at pixel centres with the scorer's per-pixel code, clipped) are summed in
// float64 and reduced over the CTA.
#include <cuda_runtime.h>

#include "../../include/weftk_bicubic.h"
#include "../../include/weftk_fit.h"
#include "weftk_common.cuh"
#include "weftk_prim.cuh"

namespace weftk {

extern __device__ int g_device_status;

namespace {

constexpr int BC_THREADS = 128;
constexpr int BC_WARPS = BC_THREADS / 32;
constexpr int BC_MAX_PRIMS = 48;
constexpr int BC_PPL = 4;
__constant__ int c_bic_prim_bytes[8] = WEFTK_PRIM_BYTES;

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

__global__ void __launch_bounds__(BC_THREADS) bicubic_swap_kernel(
    const float4* __restrict__ px, const int32_t* __restrict__ px_off, const int32_t* __restrict__ size, int n_tiles,
    const WeftPrim* __restrict__ prims, int n_prims, const int32_t* __restrict__ prim_off,
    const double* __restrict__ basis, double lam, float* __restrict__ grid_out, int32_t* __restrict__ swap_out,
    double* __restrict__ score_out) {
    __shared__ double L[4][64][3];   // pinv(B) @ T
    __shared__ double BQ[64][4][3];  // B @ Q
    __shared__ float Q[48];
    __shared__ Prep sp[BC_MAX_PRIMS];
    __shared__ double red[2][BC_WARPS];
    const int t = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int n = size[t];
    const int s0 = prim_off[t], np = prim_off[t + 1] - s0;
    if (!(n == 8 || n == 16 || n == 32 || n == 64) || np < 0 || np > BC_MAX_PRIMS || s0 < 0 || s0 + np > n_prims) {
        if (tid == 0) atomicCAS(&g_device_status, 0, WEFTK_E_ARG);
        return;
    }
    const double* A = basis + 12 * (n - 8);  // pinv(B), 4 x n
    const double* C = A + 4 * n;             // pinv(B^T), n x 4
    const double* B = C + 4 * n;             // B, n x 4
    const float4* T = px + px_off[t];
    const int npx = n * n;

    // L[r][x][ch] = sum_y A[r][y] T[y][x][ch]
    for (int x = tid; x < n; x += BC_THREADS) {
        double acc[4][3];
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[r][0] = acc[r][1] = acc[r][2] = 0.0;
        for (int y = 0; y < n; ++y) {
            const float4 v = T[y * n + x];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const double a = A[r * n + y];
                acc[r][0] = fma(a, (double)v.x, acc[r][0]);
                acc[r][1] = fma(a, (double)v.y, acc[r][1]);
                acc[r][2] = fma(a, (double)v.z, acc[r][2]);
            }
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            L[r][x][0] = acc[r][0];
            L[r][x][1] = acc[r][1];
            L[r][x][2] = acc[r][2];
        }
    }
    for (int i = tid; i < np; i += BC_THREADS) sp[i] = prep_prim(prims[s0 + i]);
    __syncthreads();
    // control grid: P[r][c][ch] = sum_x L[r][x][ch] C[x][c], float32, clipped, rounded to u8 steps
    if (tid < 48) {
        const int r = tid / 12, c = (tid / 3) % 4, ch = tid % 3;
        double acc = 0.0;
        for (int x = 0; x < n; ++x) acc = fma(L[r][x][ch], C[x * 4 + c], acc);
        const float cp = __saturatef((float)acc);
        const float q = __fdiv_rn(rintf(__fmul_rn(cp, 255.0f)), 255.0f);
        Q[tid] = q;
        grid_out[(size_t)t * 48 + tid] = q;
    }
    __syncthreads();
    // BQ[y][c][ch] = sum_r B[y][r] Q[r][c][ch]
    for (int i = tid; i < n * 12; i += BC_THREADS) {
        const int y = i / 12, c = (i / 3) % 4, ch = i % 3;
        double acc = 0.0;
#pragma unroll
        for (int r = 0; r < 4; ++r) acc = fma(B[y * 4 + r], (double)Q[(r * 4 + c) * 3 + ch], acc);
        BQ[y][c][ch] = acc;
    }
    __syncthreads();
    // squared error of the bicubic evaluation (B @ Q) @ B^T, float32, clipped
    double e_bic = 0.0;
    for (int i = tid; i < npx; i += BC_THREADS) {
        const int y = i / n, x = i - y * n;
        const float4 v = T[i];
        const float s[3] = {v.x, v.y, v.z};
        float part = 0.0f;
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            double o = 0.0;
#pragma unroll
            for (int c = 0; c < 4; ++c) o = fma(BQ[y][c][ch], B[x * 4 + c], o);
            const float d = __fsub_rn(s[ch], __saturatef((float)o));
            part = __fadd_rn(part, __fmul_rn(d, d));
        }
        e_bic += (double)part;
    }
    // squared error of the stack rendered at pixel centres (over black, clipped)
    double e_stack = 0.0;
    for (int base = wid * 32 * BC_PPL; base < npx; base += BC_WARPS * 32 * BC_PPL) {
        float fx[BC_PPL], fy[BC_PPL], cr[BC_PPL], cg[BC_PPL], cb[BC_PPL];
#pragma unroll
        for (int j = 0; j < BC_PPL; ++j) {
            const int p = min(base + j * 32 + lane, npx - 1);
            fx[j] = (float)(p % n) + 0.5f;
            fy[j] = (float)(p / n) + 0.5f;
            cr[j] = cg[j] = cb[j] = 0.0f;
        }
        for (int k = 0; k < np; ++k) {
            Prep pr = sp[k];
            if (pr.kind == K_BICUBIC) pr.kind = K_SKIP;
            float a[BC_PPL], sr[BC_PPL], sg[BC_PPL], sb[BC_PPL];
            prim_eval<BC_PPL>(pr, fx, fy, a, sr, sg, sb, lane);
#pragma unroll
            for (int j = 0; j < BC_PPL; ++j) {
                cr[j] = blend(sr[j], a[j], cr[j]);
                cg[j] = blend(sg[j], a[j], cg[j]);
                cb[j] = blend(sb[j], a[j], cb[j]);
            }
        }
        float part = 0.0f;
#pragma unroll
        for (int j = 0; j < BC_PPL; ++j) {
            const int p = base + j * 32 + lane;
            if (p < npx) {
                const float4 v = T[p];
                const float dr = __fsub_rn(v.x, clamp01(cr[j])), dg = __fsub_rn(v.y, clamp01(cg[j])),
                            db = __fsub_rn(v.z, clamp01(cb[j]));
                part = __fadd_rn(part, __fadd_rn(__fadd_rn(__fmul_rn(dr, dr), __fmul_rn(dg, dg)), __fmul_rn(db, db)));
            }
        }
        e_stack += (double)part;
    }
    e_bic = warp_sum_d(e_bic);
    e_stack = warp_sum_d(e_stack);
    if (lane == 0) {
        red[0][wid] = e_bic;
        red[1][wid] = e_stack;
    }
    __syncthreads();
    if (tid == 0) {
        double sb = 0.0, ss = 0.0;
        for (int w = 0; w < BC_WARPS; ++w) {
            sb += red[0][w];
            ss += red[1][w];
        }
        int bits = 8;
        for (int k = 0; k < np; ++k) {
            const int kind = prims[s0 + k].kind;
            bits += 8 * ((kind >= 0 && kind < 8) ? c_bic_prim_bytes[kind] : 20);
        }
        const double denom = 3.0 * (double)npx;
        const double bic_score = sb / denom + lam * (double)WEFTK_BICUBIC_BITS;
        const double stack_score = ss / denom + lam * (double)bits;
        swap_out[t] = bic_score < stack_score ? 1 : 0;
        score_out[2 * (size_t)t] = bic_score;
        score_out[2 * (size_t)t + 1] = stack_score;
    }
}

}  // namespace

}  // namespace weftk

extern "C" int weftk_bicubic_swap(const float* d_pixels, const int32_t* d_px_off, const int32_t* d_size, int n_tiles,
                                  const WeftPrim* d_prims, int n_prims, const int32_t* d_prim_off,
                                  const double* d_basis, double lam, float* d_grid, int32_t* d_swap, double* d_score,
                                  void* stream) {
    using namespace weftk;
    if (n_tiles == 0) return WEFTK_OK;
    WEFTK_REQUIRE(n_tiles > 0 && n_prims >= 0 && (n_prims == 0 || d_prims) && d_pixels && d_px_off && d_size &&
                      d_prim_off && d_basis && d_grid && d_swap && d_score,
                  "bicubic_swap: bad arguments");
    WEFTK_REQUIRE((reinterpret_cast<uintptr_t>(d_pixels) & 15) == 0, "bicubic_swap: pixels must be 16-byte aligned");
    bicubic_swap_kernel<<<n_tiles, BC_THREADS, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const float4*>(d_pixels), d_px_off, d_size, n_tiles, d_prims, n_prims, d_prim_off, d_basis, lam,
        d_grid, d_swap, d_score);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}
