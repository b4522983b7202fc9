// weftk_wire.cu — selected primitives snapped to the bitstream's quantisation grid on the
// device (include/weftk_wire.h): the reference's _quantize_primitive
// (src/weft/encoder.py:211-237) for every row at once, so the fit's output can be produced
// inside the same CUDA graph as the fit.
#include <cuda_runtime.h>

#include "../../include/weftk_fit.h"
#include "../../include/weftk_wire.h"
#include "weftk_common.cuh"

namespace weftk {

extern __device__ int g_device_status;

namespace {

// round(clamp(v / range, 0, 1) * steps) / steps * range in float64, rint = round half to even
// (Python's round); every operation rounded on its own (no fused multiply-add), as the
// reference's float64 expression.
__device__ __forceinline__ float snap(float v, double steps, double range) {
    double u = __ddiv_rn((double)v, range);
    u = fmin(1.0, fmax(0.0, u));
    const double q = rint(__dmul_rn(u, steps));
    return (float)__dmul_rn(__ddiv_rn(q, steps), range);
}

// Number of leading geometry values that are coordinates, and the column of the thickness
// (-1: none), per kind: linear 4 / -, line 4 / 4, curve 6 / 6, triangle 6 / -.  Constant
// patches, bicubic rows and kind < 0 keep their geometry.
__device__ __forceinline__ void wire_geom(int kind, int& n_coord, int& thick) {
    n_coord = 0;
    thick = -1;
    if (kind == 1) n_coord = 4;
    else if (kind == 2) { n_coord = 4; thick = 4; }
    else if (kind == 3) { n_coord = 6; thick = 6; }
    else if (kind == 4) n_coord = 6;
}

__device__ __forceinline__ void quantize_row(const float* in, int kind, float* out) {
    float r[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) r[c] = in[c];
    int n_coord, thick;
    wire_geom(kind, n_coord, thick);
#pragma unroll
    for (int c = 0; c < 7; ++c) {
        if (c < n_coord) r[c] = snap(r[c], 65535.0, 15.0);
        else if (c == thick) r[c] = snap(r[c], 65535.0, 4.0);
    }
#pragma unroll
    for (int c = 7; c < 13; ++c) r[c] = snap(r[c], 255.0, 1.0);
    r[13] = snap(r[13], 65535.0, 1.0);
#pragma unroll
    for (int c = 0; c < 16; ++c) out[c] = r[c];
}

__global__ void quantize_rows_kernel(const float* __restrict__ params, const int32_t* __restrict__ kinds, int n_rows,
                                     float* __restrict__ out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    quantize_row(params + (size_t)r * 16, kinds[r], out + (size_t)r * 16);
}

__global__ void fit_selected_rows_kernel(WeftFitState st, float* __restrict__ rows, int32_t* __restrict__ kinds) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)st.n_tiles * st.cap_max) return;
    const int t = (int)(i / st.cap_max);
    const int j = (int)(i % st.cap_max);
    float* out = rows + i * 16;
    int kind = -1;
    if (j < st.n_sel[t]) {
        const int s = st.sel[i];
        const long long slot = (long long)st.pool_off[t] + s;
        if (s >= 0 && s < st.pool_cap[t] && slot < st.n_slots) {
            const WeftPrim p = st.cand[slot];
            float in[16];
#pragma unroll
            for (int c = 0; c < 7; ++c) in[c] = p.geom[c];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                in[7 + c] = p.color0[c];
                in[10 + c] = p.color1[c];
            }
            in[13] = p.alpha;
            in[14] = in[15] = 0.0f;
            kind = p.kind;
            quantize_row(in, kind, out);
        } else {
            atomicCAS(&g_device_status, 0, WEFTK_E_ARG);
        }
    }
    if (kind < 0) {
#pragma unroll
        for (int c = 0; c < 16; ++c) out[c] = 0.0f;
    }
    kinds[i] = kind;
}

}  // namespace
}  // namespace weftk

using namespace weftk;

extern "C" int weftk_quantize_rows(const float* d_params, const int32_t* d_kind, int n_rows, float* d_out,
                                   void* stream) {
    WEFTK_REQUIRE(n_rows >= 0, "quantize_rows: negative row count");
    if (n_rows == 0) return WEFTK_OK;
    WEFTK_REQUIRE(d_params && d_kind && d_out, "quantize_rows: null pointer");
    quantize_rows_kernel<<<ceil_div(n_rows, 128), 128, 0, (cudaStream_t)stream>>>(d_params, d_kind, n_rows, d_out);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}

extern "C" int weftk_fit_selected_rows(const WeftFitState* st, float* d_rows, int32_t* d_kind, void* stream) {
    WEFTK_REQUIRE(st && st->n_tiles >= 0 && st->cap_max >= 1, "fit_selected_rows: bad fit state");
    const long long n = (long long)st->n_tiles * st->cap_max;
    if (n == 0) return WEFTK_OK;
    WEFTK_REQUIRE(d_rows && d_kind, "fit_selected_rows: null pointer");
    WEFTK_REQUIRE(n < (1ll << 31), "fit_selected_rows: too many rows");
    fit_selected_rows_kernel<<<ceil_div(n, 128), 128, 0, (cudaStream_t)stream>>>(*st, d_rows, d_kind);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}
