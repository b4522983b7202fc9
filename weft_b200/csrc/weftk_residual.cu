// weftk_residual.cu — RES0 / RES1 build per tile (see include/weftk_residual.h).
#include <cuda_runtime.h>

#include "../../include/weftk_residual.h"
#include "weftk_common.cuh"
#include "weftk_prim.cuh"

namespace weftk {

extern __device__ int g_device_status;

__device__ __forceinline__ float recon_at(const float4* r, int i, int ch, bool clamp) {
    const float4 v = r[i];
    const float x = ch == 0 ? v.x : ch == 1 ? v.y : v.z;
    return clamp ? fminf(fmaxf(x, 0.0f), 1.0f) : x;
}

__device__ __forceinline__ float src_at(const float4* s, int i, int ch) {
    const float4 v = s[i];
    return ch == 0 ? v.x : ch == 1 ? v.y : v.z;
}

// One CTA of 64 threads per tile.  Threads 0-2: RES0 per channel; then threads 0-47: one RES1 cell
// and channel each.  Every sum runs sequentially in row-major pixel order, as numpy's reduction
// over the leading axes of an (h, w, 3) float32 array does.
__global__ void __launch_bounds__(64) build_residuals_kernel(const float4* __restrict__ src,
                                                             const float4* __restrict__ recon, bool clamp,
                                                             const int* __restrict__ px_off,
                                                             const int* __restrict__ size, int n_tiles,
                                                             int8_t* __restrict__ res0, int8_t* __restrict__ res1) {
    __shared__ float d_add[3];
    const int t = blockIdx.x;
    if (t >= n_tiles) return;
    const int ts = size[t];
    if (ts < 4 || ts > 64 || (ts & 3) != 0) {
        if (threadIdx.x == 0) atomicCAS(&g_device_status, 0, WEFTK_E_ARG);
        return;
    }
    const float4* s = src + px_off[t];
    const float4* r = recon + px_off[t];
    const int n = ts * ts;
    if (threadIdx.x < 3) {
        const int ch = threadIdx.x;
        float acc = 0.0f;
        for (int i = 0; i < n; ++i) acc = __fadd_rn(acc, __fsub_rn(src_at(s, i, ch), recon_at(r, i, ch, clamp)));
        const float mean = __fdiv_rn(acc, (float)n);
        double v = rint((double)mean * 255.0);  // Python float product, numpy round (half to even)
        v = fmin(fmax(v, -127.0), 127.0);
        res0[(size_t)t * 3 + ch] = (int8_t)(int)v;
        d_add[ch] = __fdiv_rn((float)(int)v, 255.0f);  // float32 array / 255.0 stays float32
    }
    __syncthreads();
    if (threadIdx.x < 48) {
        const int cell = threadIdx.x / 3, ch = threadIdx.x - cell * 3;
        const int ga = cell >> 2, gc = cell & 3, b = ts >> 2;
        const float dc = d_add[ch];
        float acc = 0.0f;
        for (int bb = 0; bb < b; ++bb) {
            const int row = ga * b + bb;
            for (int dd = 0; dd < b; ++dd) {
                const int i = row * ts + gc * b + dd;
                const float pred = fminf(fmaxf(__fadd_rn(recon_at(r, i, ch, clamp), dc), 0.0f), 1.0f);
                acc = __fadd_rn(acc, __fsub_rn(src_at(s, i, ch), pred));
            }
        }
        const float mean = __fdiv_rn(acc, (float)(b * b));
        float v = rintf(__fmul_rn(mean, 255.0f));
        v = fminf(fmaxf(v, -127.0f), 127.0f);
        res1[(size_t)t * 48 + cell * 3 + ch] = (int8_t)(int)v;
    }
}

}  // namespace weftk

using namespace weftk;

extern "C" int weftk_build_residuals(const float* d_src, const float* d_recon, int clamp_recon, const int32_t* d_px_off,
                                     const int32_t* d_size, int n_tiles, int8_t* d_res0, int8_t* d_res1,
                                     void* stream) {
    WEFTK_REQUIRE(n_tiles >= 0, "build_residuals: negative tile count");
    if (n_tiles == 0) return WEFTK_OK;
    WEFTK_REQUIRE(d_src && d_recon && d_px_off && d_size && d_res0 && d_res1, "build_residuals: null pointer");
    build_residuals_kernel<<<n_tiles, 64, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const float4*>(d_src), reinterpret_cast<const float4*>(d_recon), clamp_recon != 0, d_px_off,
        d_size, n_tiles, d_res0, d_res1);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}
