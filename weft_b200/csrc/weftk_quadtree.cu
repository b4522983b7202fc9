// weftk_quadtree.cu — quadtree tiling (variance rule) and tile extraction on the device
// (include/weftk_quadtree.h).
//
// Tiling: one CTA per macro tile.  The macro tile's luminance (float64, the host's expression
// 0.2126 R + 0.7152 G + 0.0722 B on u8 values, left to right) goes to shared memory; one warp per
// candidate square takes its variance (mean, then mean of squared deviations, float64); one
// thread walks the split tree in the reference's order and stages the tiles.  A one-CTA scan of
// the per-macro-tile counts places them in the output.  Extraction: one CTA per tile, pixels
// through the host's 256-entry sRGB-decode table, float4 per pixel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/weftk_quadtree.h"
#include "weftk_common.cuh"

namespace weftk {

extern __device__ int g_device_status;

namespace {

constexpr int QT_MAX = 64;                       // largest macro tile side
constexpr int QT_MAX_TILES = (QT_MAX / 8) * (QT_MAX / 8);  // tiles per macro tile, bound
constexpr int QT_SCAN_THREADS = 1024;
static_assert(QT_SCAN_THREADS == 32 * 32, "the placement scan is two levels of 32");

__device__ __forceinline__ double lum_u8(const uint8_t* p) {
    return __dadd_rn(__dadd_rn(__dmul_rn(0.2126, (double)p[0]), __dmul_rn(0.7152, (double)p[1])),
                     __dmul_rn(0.0722, (double)p[2]));
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// squares of side s > min_tile at every level, level l of side MT >> l, row-major inside a level
__global__ void __launch_bounds__(256) qt_split_kernel(const uint8_t* __restrict__ img, int h, int w, int MT, int mt,
                                                       double thr, int n_mx, int32_t* __restrict__ stage,
                                                       int32_t* __restrict__ counts) {
    __shared__ double lum[QT_MAX * QT_MAX];
    __shared__ unsigned char split[1 + 4 + 16 + 64];
    const int mb = blockIdx.x, my = mb / n_mx, mx = mb - my * n_mx;
    const int x0 = mx * MT, y0 = my * MT;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < MT * MT; i += blockDim.x) {
        const int yy = min(y0 + i / MT, h - 1), xx = min(x0 + i % MT, w - 1);  // edge padding
        lum[i] = lum_u8(img + ((size_t)yy * w + xx) * 3);
    }
    __syncthreads();
    int n_sq = 0, levels = 0;
    for (int s = MT; s > mt; s >>= 1, ++levels) n_sq += (MT / s) * (MT / s);
    for (int q = warp; q < n_sq; q += blockDim.x / 32) {
        int l = 0, base = 0, per = 1;
        while (q >= base + per) {
            base += per;
            ++l;
            per *= 4;
        }
        const int s = MT >> l, side = MT / s, k = q - base;
        const int sx = (k % side) * s, sy = (k / side) * s;
        const int n = s * s;
        double sum = 0.0;
        for (int i = lane; i < n; i += 32) sum += lum[(sy + i / s) * MT + sx + i % s];
        const double mean = warp_sum_d(sum) / (double)n;
        double sq = 0.0;
        for (int i = lane; i < n; i += 32) {
            const double d = lum[(sy + i / s) * MT + sx + i % s] - mean;
            sq += d * d;
        }
        const double var = warp_sum_d(sq) / (double)n;
        if (lane == 0) split[q] = var > thr;
    }
    __syncthreads();
    if (tid == 0) {
        // depth-first walk: top-left, top-right, bottom-left, bottom-right
        int sx[24], sy[24], ss[24], top = 0, cnt = 0;
        sx[0] = 0;
        sy[0] = 0;
        ss[0] = MT;
        top = 1;
        while (top > 0) {
            --top;
            const int x = sx[top], y = sy[top], s = ss[top];
            bool sp = false;
            if (s > mt) {
                int l = 0, base = 0, per = 1;
                while ((MT >> l) != s) {
                    base += per;
                    per *= 4;
                    ++l;
                }
                const int side = MT / s;
                sp = split[base + (y / s) * side + x / s];
            }
            if (sp) {
                const int hs = s / 2;  // pushed in reverse so top-left is visited first
                const int cx[4] = {x + hs, x, x + hs, x}, cy[4] = {y + hs, y + hs, y, y};
                for (int c = 0; c < 4; ++c) {
                    sx[top] = cx[c];
                    sy[top] = cy[c];
                    ss[top] = hs;
                    ++top;
                }
            } else {
                int32_t* o = stage + ((size_t)mb * QT_MAX_TILES + cnt) * 3;
                o[0] = x0 + x;
                o[1] = y0 + y;
                o[2] = s;
                ++cnt;
            }
        }
        counts[mb] = cnt;
    }
}

// exclusive scan of the per-macro-tile counts (one CTA), then every macro tile's staged tiles
// copied to their place
__global__ void __launch_bounds__(QT_SCAN_THREADS) qt_place_kernel(const int32_t* __restrict__ stage,
                                                                   const int32_t* __restrict__ counts, int n_macro,
                                                                   int32_t* __restrict__ tiles, int max_tiles,
                                                                   int32_t* __restrict__ n_out) {
    __shared__ int wtot[QT_SCAN_THREADS / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int per = (n_macro + QT_SCAN_THREADS - 1) / QT_SCAN_THREADS;
    const int lo = min(n_macro, tid * per), hi = min(n_macro, lo + per);
    int s = 0;
    for (int i = lo; i < hi; ++i) s += counts[i];
    // exclusive prefix sum of the threads' counts: inclusive scans in each warp, then of the
    // warps' totals
    int v = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) wtot[warp] = v;
    __syncthreads();
    if (warp == 0) {
        int w = wtot[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += u;
        }
        wtot[lane] = w;
    }
    __syncthreads();
    if (tid == 0) {
        const int run = wtot[QT_SCAN_THREADS / 32 - 1];
        *n_out = min(run, max_tiles);
        if (run > max_tiles) atomicCAS(&g_device_status, 0, WEFTK_E_RANGE);
    }
    int off = v - s + (warp ? wtot[warp - 1] : 0);
    for (int i = lo; i < hi; ++i) {
        const int c = counts[i];
        for (int j = 0; j < c; ++j, ++off) {
            if (off >= max_tiles) break;
            const int32_t* src = stage + ((size_t)i * QT_MAX_TILES + j) * 3;
            tiles[(size_t)off * 3] = src[0];
            tiles[(size_t)off * 3 + 1] = src[1];
            tiles[(size_t)off * 3 + 2] = src[2];
        }
    }
}

// one CTA of EX_THREADS per tile (most tiles are 8 px: 64 pixels); the 1 KB sRGB table is read
// through the read-only cache
constexpr int EX_THREADS = 64;

__global__ void __launch_bounds__(EX_THREADS) extract_tiles_kernel(const uint8_t* __restrict__ img, int h, int w,
                                                                   const float* __restrict__ tab,
                                                                   const int32_t* __restrict__ tiles, int n_tiles,
                                                                   const int32_t* __restrict__ px_off,
                                                                   float4* __restrict__ out) {
    const int t = blockIdx.x;
    const int tx = tiles[t * 3], ty = tiles[t * 3 + 1], s = tiles[t * 3 + 2];
    if (s < 1 || s > 64) {
        if (threadIdx.x == 0) atomicCAS(&g_device_status, 0, WEFTK_E_ARG);
        return;
    }
    float4* dst = out + px_off[t];
    for (int i = threadIdx.x; i < s * s; i += blockDim.x) {
        const int yy = min(ty + i / s, h - 1), xx = min(tx + i % s, w - 1);
        const uint8_t* p = img + ((size_t)yy * w + xx) * 3;
        dst[i] = make_float4(__ldg(tab + p[0]), __ldg(tab + p[1]), __ldg(tab + p[2]), 0.0f);
    }
}

bool pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

}  // namespace
}  // namespace weftk

using namespace weftk;

extern "C" int weftk_quadtree_work_bytes(int h, int w, int max_tile, int min_tile, int64_t* bytes) {
    WEFTK_REQUIRE(bytes && h > 0 && w > 0 && pow2(max_tile) && pow2(min_tile) && min_tile >= 8 &&
                      min_tile <= max_tile && max_tile <= QT_MAX,
                  "quadtree_work_bytes: bad size");
    const int64_t n_macro = (int64_t)((h + max_tile - 1) / max_tile) * ((w + max_tile - 1) / max_tile);
    *bytes = n_macro * (QT_MAX_TILES * 3 + 1) * (int64_t)sizeof(int32_t);
    return WEFTK_OK;
}

extern "C" int weftk_quadtree_variance(const uint8_t* d_img, int h, int w, double threshold, int max_tile,
                                       int min_tile, int32_t* d_tiles, int max_tiles, int32_t* d_n_tiles,
                                       void* d_work, void* stream) {
    int64_t need = 0;
    int rc = weftk_quadtree_work_bytes(h, w, max_tile, min_tile, &need);
    if (rc) return rc;
    WEFTK_REQUIRE(d_img && d_tiles && d_n_tiles && d_work && max_tiles >= 0, "quadtree_variance: null pointer");
    const int n_mx = (w + max_tile - 1) / max_tile, n_my = (h + max_tile - 1) / max_tile;
    const long long n_macro = (long long)n_mx * n_my;
    WEFTK_REQUIRE(n_macro < (1ll << 30), "quadtree_variance: image too large");
    int32_t* stage = static_cast<int32_t*>(d_work);
    int32_t* counts = stage + n_macro * QT_MAX_TILES * 3;
    cudaStream_t s = (cudaStream_t)stream;
    qt_split_kernel<<<(unsigned)n_macro, 256, 0, s>>>(d_img, h, w, max_tile, min_tile, threshold, n_mx, stage, counts);
    WEFTK_CUDA(cudaGetLastError());
    qt_place_kernel<<<1, QT_SCAN_THREADS, 0, s>>>(stage, counts, (int)n_macro, d_tiles, max_tiles, d_n_tiles);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}

extern "C" int weftk_extract_tiles(const uint8_t* d_img, int h, int w, const float* d_lut, const int32_t* d_tiles,
                                   int n_tiles, const int32_t* d_px_off, float* d_src4, void* stream) {
    WEFTK_REQUIRE(h > 0 && w > 0 && n_tiles >= 0, "extract_tiles: bad size");
    if (n_tiles == 0) return WEFTK_OK;
    WEFTK_REQUIRE(d_img && d_lut && d_tiles && d_px_off && d_src4, "extract_tiles: null pointer");
    extract_tiles_kernel<<<n_tiles, EX_THREADS, 0, (cudaStream_t)stream>>>(d_img, h, w, d_lut, d_tiles, n_tiles, d_px_off,
                                                                     reinterpret_cast<float4*>(d_src4));
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}
