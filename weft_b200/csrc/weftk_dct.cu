// weftk_dct.cu — the decoder's raster branch: per-tile DCT residual layer and the u8 BILINEAR
// resize (see include/weftk_dct.h).
//
// DCT layer: one CTA per tile.  Each channel's quantized block is gathered straight from the
// coefficient stream (tile-major or band-major zigzag: the band-to-tile permutation is only an
// address computation), dequantized and inverse-transformed in float64 as two separable passes
// through shared memory, rounded to float32; the three channels are then colour-transformed,
// added to the image and clipped.  The transform is the orthonormal DCT-III written as a
// matrix product with the DCT-II basis A[k][x] = c_k cos(pi (2x + 1) k / (2n)).
//
// Resize: Pillow's ImagingResample for 8-bit images.  A sample's taps (bounds, float64 triangle
// weights normalised by their sum, rounded to 22-bit fixed point) are derived exactly as Pillow's
// precompute_coeffs / normalize_coeffs_8bpc do, once per CTA column (pass 1) or output row
// (pass 2), then accumulated in int32 and rounded with the same clip.  Pass 1 (a thread per output
// column over 8 source rows) writes the 8-bit intermediate; pass 2 (a thread per output column
// over 8 output rows) reads it.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "../../include/weftk_dct.h"
#include "weftk_common.cuh"

namespace weftk {

extern __device__ int g_device_status;

// Basis and zigzag tables for block sides n = 2, 4, ..., 64, back to back: side n = 2^L starts
// at (4^L - 4) / 3.
constexpr int kDctTab = 5460;
__device__ double g_dct_basis[kDctTab];  // [k * n + x] = A[k][x]
__device__ short g_dct_zigzag[kDctTab];  // [u * n + v] = zigzag scan position of (u, v)

__host__ __device__ constexpr int dct_tab_off(int log2n) { return ((1 << (2 * log2n)) - 4) / 3; }

__device__ __forceinline__ int ilog2(int n) { return 31 - __clz(n); }

__global__ void dct_tables_kernel() {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kDctTab) return;
    int L = 1;
    while (L < 6 && i >= dct_tab_off(L + 1)) ++L;
    const int n = 1 << L, r = i - dct_tab_off(L);
    const int k = r >> L, x = r & (n - 1);
    // basis: sqrt(1/n) for k = 0, else cos(((pi * (2x + 1)) * k) / (2n)) * sqrt(2/n)
    if (k == 0) {
        g_dct_basis[i] = sqrt(1.0 / (double)n);
    } else {
        const double arg = __ddiv_rn(__dmul_rn(__dmul_rn(3.141592653589793, (double)(2 * x + 1)), (double)k),
                                     (double)(2 * n));
        g_dct_basis[i] = __dmul_rn(cos(arg), sqrt(2.0 / (double)n));
    }
    // zigzag position of row-major (u, v) = (k, x): anti-diagonal s = u + v holds rows
    // lo..hi, scanned bottom-left to top-right (rows descending) when s is even, else ascending.
    const int u = k, v = x, s = u + v;
    const int before = s < n ? s * (s + 1) / 2 : n * n - (2 * n - 1 - s) * (2 * n - s) / 2;
    const int lo = s - n + 1 > 0 ? s - n + 1 : 0, hi = s < n - 1 ? s : n - 1;
    g_dct_zigzag[i] = (short)(before + ((s & 1) == 0 ? hi - u : u - lo));
}

__global__ void __launch_bounds__(256) dct_apply_kernel(const WeftDctTile* __restrict__ tiles, int n_tiles,
                                                        const int16_t* __restrict__ coeffs, long long n_coeffs,
                                                        int chroma, int band, double step_luma, double step_chroma,
                                                        double alpha, int max_size, float* __restrict__ image,
                                                        int width, int height) {
    extern __shared__ double dct_smem[];
    const int t = blockIdx.x;
    if (t >= n_tiles) return;
    const WeftDctTile* tp = tiles + t;
    const int S = tp->size;
    const int tx0 = tp->x, ty0 = tp->y;
    const double step_scale = tp->step_scale;
    if (S < 4 || S > max_size || S > WEFTK_DCT_MAX_TILE || (S & (S - 1)) != 0) {
        if (threadIdx.x == 0) atomicCAS(&g_device_status, 0, WEFTK_E_ARG);
        return;
    }
    const int M2 = max_size * max_size;
    double* X = dct_smem;                          // dequantized block [u * n + v]
    double* T = dct_smem + M2;                     // after the pass along v: [u * n + x]
    float* R = reinterpret_cast<float*>(dct_smem + 2 * M2);  // 3 planes of float32 results
    const int LS = ilog2(S);

    for (int c = 0; c < 3; ++c) {
        const int L = (chroma == 2 && c > 0) ? LS - 1 : LS;
        const int n = 1 << L, nn = n * n;
        const double step = (chroma != 0 && c > 0) ? step_chroma : step_luma;
        const double* A = g_dct_basis + dct_tab_off(L);
        const short* Z = g_dct_zigzag + dct_tab_off(L);
        const long long base = tp->coef_base[c], stride = tp->coef_stride[c];
        const double ramp_den = 2.0 * (double)(n - 1);
        for (int idx = threadIdx.x; idx < nn; idx += blockDim.x) {
            const long long pos = band ? (long long)Z[idx] : (long long)idx;
            const long long a = base + pos * stride;
            int q = 0;
            if (a >= 0 && a < n_coeffs) {
                q = coeffs[a];
            } else {
                atomicCAS(&g_device_status, 0, WEFTK_E_ARG);
            }
            double g = step;
            if (alpha > 0.0) {
                const double ramp = __ddiv_rn((double)((idx >> L) + (idx & (n - 1))), ramp_den);
                g = __dmul_rn(step, __dadd_rn(1.0, __dmul_rn(alpha, ramp)));
            }
            g = __dmul_rn(g, step_scale);
            X[idx] = __dmul_rn((double)q, g);
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < nn; idx += blockDim.x) {
            const int u = idx >> L, x = idx & (n - 1);
            double acc = 0.0;
            for (int v = 0; v < n; ++v) acc = fma(A[v * n + x], X[u * n + v], acc);
            T[idx] = acc;
        }
        __syncthreads();
        float* Rc = R + c * M2;
        for (int idx = threadIdx.x; idx < nn; idx += blockDim.x) {
            const int y = idx >> L, x = idx & (n - 1);
            double acc = 0.0;
            for (int u = 0; u < n; ++u) acc = fma(A[u * n + y], T[u * n + x], acc);
            Rc[idx] = __double2float_rn(acc);
        }
        __syncthreads();
    }

    const float* R0 = R;
    const float* R1 = R + M2;
    const float* R2 = R + 2 * M2;
    for (int p = threadIdx.x; p < S * S; p += blockDim.x) {
        const int y = p >> LS, x = p & (S - 1);
        const long long gx = (long long)tx0 + x, gy = (long long)ty0 + y;
        if (gx < 0 || gy < 0 || gx >= width || gy >= height) continue;
        float res[3];
        if (chroma == 0) {
            res[0] = R0[p];
            res[1] = R1[p];
            res[2] = R2[p];
        } else {
            const int ci = chroma == 2 ? (y >> 1) * (S >> 1) + (x >> 1) : p;
            const double Y = R0[p], Cb = R1[ci], Cr = R2[ci];
            // rows of the BT.601 YCbCr -> RGB residual matrix, each a left-to-right dot product
            res[0] = __double2float_rn(__dadd_rn(__dadd_rn(__dmul_rn(Y, 1.0), __dmul_rn(Cb, 0.0)), __dmul_rn(Cr, 1.402)));
            res[1] = __double2float_rn(
                __dadd_rn(__dadd_rn(__dmul_rn(Y, 1.0), __dmul_rn(Cb, -0.344136)), __dmul_rn(Cr, -0.714136)));
            res[2] = __double2float_rn(__dadd_rn(__dadd_rn(__dmul_rn(Y, 1.0), __dmul_rn(Cb, 1.772)), __dmul_rn(Cr, 0.0)));
        }
        float* px = image + (gy * width + gx) * 3;
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) px[ch] = fminf(fmaxf(__fadd_rn(px[ch], res[ch]), 0.0f), 1.0f);
    }
}

__global__ void clip01_kernel(float* __restrict__ image, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        image[i] = fminf(fmaxf(image[i], 0.0f), 1.0f);
}

// ---------------------------------------------------------------------------------- resize
constexpr int kResampleBits = 22;

__device__ __forceinline__ double triangle(double d) {
    if (d < 0.0) d = -d;
    return d < 1.0 ? __dsub_rn(1.0, d) : 0.0;
}

// Taps of output sample o of an in_size -> out_size BILINEAR resample (Pillow precompute_coeffs).
struct Taps {
    int first, count;
    double center, inv_fs, ww;
};

__device__ __forceinline__ Taps resample_taps(int in_size, int out_size, int o) {
    Taps t;
    const double scale = __ddiv_rn((double)in_size, (double)out_size);
    const double fs = scale < 1.0 ? 1.0 : scale;
    const double support = fs;  // triangle support 1.0 x filter scale
    t.center = __dmul_rn(__dadd_rn((double)o, 0.5), scale);
    t.inv_fs = __ddiv_rn(1.0, fs);
    int lo = (int)__dadd_rn(__dsub_rn(t.center, support), 0.5);
    if (lo < 0) lo = 0;
    int hi = (int)__dadd_rn(__dadd_rn(t.center, support), 0.5);
    if (hi > in_size) hi = in_size;
    t.first = lo;
    t.count = hi - lo;
    double ww = 0.0;
    for (int x = 0; x < t.count; ++x)
        ww = __dadd_rn(ww, triangle(__dmul_rn(__dadd_rn(__dsub_rn((double)(x + lo), t.center), 0.5), t.inv_fs)));
    t.ww = ww;
    return t;
}

__device__ __forceinline__ int tap_weight(const Taps& t, int x) {
    double w = triangle(__dmul_rn(__dadd_rn(__dsub_rn((double)(x + t.first), t.center), 0.5), t.inv_fs));
    if (t.ww != 0.0) w = __ddiv_rn(w, t.ww);
    const double s = __dmul_rn(w, (double)(1 << kResampleBits));
    return w < 0.0 ? (int)__dadd_rn(-0.5, s) : (int)__dadd_rn(0.5, s);
}

__device__ __forceinline__ int clip8(int acc) {
    const int v = acc >> kResampleBits;
    return v < 0 ? 0 : (v > 255 ? 255 : v);
}

__device__ __forceinline__ int to_u8(float v) {
    const float p = fminf(fmaxf(__fmul_rn(v, 255.0f), 0.0f), 255.0f);
    return (int)p;  // truncation, as numpy's astype(uint8)
}

// Both passes: a CTA covers RS_COLS output columns x RS_ROWS rows.  A sample's taps (Pillow's
// bounds and 22-bit integer weights) depend on its output column (row pass) or output row (column
// pass) only, so they are derived once per CTA column or row and reused, not once per pixel; a
// sample with more than RS_MAXT taps (a downscale by more than about 3.5) derives each weight where
// it is used.  The weights are the same integers either way.
constexpr int RS_COLS = 128, RS_ROWS = 8, RS_MAXT = 8;

__global__ void __launch_bounds__(RS_COLS) resize_rows_kernel(const float* __restrict__ src, int src_w, int src_h,
                                                              uint8_t* __restrict__ tmp, int dst_w) {
    const int xx = blockIdx.x * RS_COLS + threadIdx.x;
    const int y0 = blockIdx.y * RS_ROWS;
    if (xx >= dst_w) return;
    const Taps t = resample_taps(src_w, dst_w, xx);
    const bool cached = t.count <= RS_MAXT;
    int k[RS_MAXT], sx[RS_MAXT];
#pragma unroll
    for (int j = 0; j < RS_MAXT; ++j) {
        k[j] = cached && j < t.count ? tap_weight(t, j) : 0;
        sx[j] = min(t.first + j, src_w - 1);
    }
    for (int r = 0; r < RS_ROWS; ++r) {
        const int y = y0 + r;
        if (y >= src_h) break;
        int a0 = 1 << (kResampleBits - 1), a1 = a0, a2 = a0;
        const float* row = src + (long long)y * src_w * 3;
        if (cached) {
#pragma unroll
            for (int j = 0; j < RS_MAXT; ++j) {
                if (j < t.count) {
                    const float* q = row + sx[j] * 3;
                    a0 += to_u8(q[0]) * k[j];
                    a1 += to_u8(q[1]) * k[j];
                    a2 += to_u8(q[2]) * k[j];
                }
            }
        } else {
            for (int x = 0; x < t.count; ++x) {
                const int s = min(t.first + x, src_w - 1);
                const int w = tap_weight(t, x);
                a0 += to_u8(row[s * 3 + 0]) * w;
                a1 += to_u8(row[s * 3 + 1]) * w;
                a2 += to_u8(row[s * 3 + 2]) * w;
            }
        }
        uint8_t* o = tmp + ((long long)y * dst_w + xx) * 3;
        o[0] = (uint8_t)clip8(a0);
        o[1] = (uint8_t)clip8(a1);
        o[2] = (uint8_t)clip8(a2);
    }
}

__global__ void __launch_bounds__(RS_COLS) resize_cols_kernel(const uint8_t* __restrict__ tmp, int src_h, int dst_w,
                                                              float* __restrict__ dst, int dst_h) {
    __shared__ int s_first[RS_ROWS], s_count[RS_ROWS], s_k[RS_ROWS][RS_MAXT];
    __shared__ Taps s_taps[RS_ROWS];
    const int xx = blockIdx.x * RS_COLS + threadIdx.x;
    const int y0 = blockIdx.y * RS_ROWS;
    // the CTA's output rows' taps, once
    if (threadIdx.x < RS_ROWS && y0 + (int)threadIdx.x < dst_h) {
        const int r = threadIdx.x;
        const Taps t = resample_taps(src_h, dst_h, y0 + r);
        s_taps[r] = t;
        s_first[r] = t.first;
        s_count[r] = t.count;
        for (int j = 0; j < RS_MAXT; ++j) s_k[r][j] = t.count <= RS_MAXT && j < t.count ? tap_weight(t, j) : 0;
    }
    __syncthreads();
    if (xx >= dst_w) return;
    for (int r = 0; r < RS_ROWS; ++r) {
        const int yy = y0 + r;
        if (yy >= dst_h) break;
        const int first = s_first[r], count = s_count[r];
        int a0 = 1 << (kResampleBits - 1), a1 = a0, a2 = a0;
        for (int y = 0; y < count; ++y) {
            const int sy = min(first + y, src_h - 1);
            const int k = count <= RS_MAXT ? s_k[r][y] : tap_weight(s_taps[r], y);
            const uint8_t* p = tmp + ((long long)sy * dst_w + xx) * 3;
            a0 += (int)p[0] * k;
            a1 += (int)p[1] * k;
            a2 += (int)p[2] * k;
        }
        float* o = dst + ((long long)yy * dst_w + xx) * 3;
        o[0] = __fdiv_rn((float)clip8(a0), 255.0f);
        o[1] = __fdiv_rn((float)clip8(a1), 255.0f);
        o[2] = __fdiv_rn((float)clip8(a2), 255.0f);
    }
}

namespace {
std::mutex g_tab_mu;
bool g_tab_ready[64] = {};

int ensure_tables(cudaStream_t stream) {
    int dev = 0;
    WEFTK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(WEFTK_E_RANGE, "dct: device index beyond 63");
    std::lock_guard<std::mutex> lock(g_tab_mu);
    if (!g_tab_ready[dev]) {
        dct_tables_kernel<<<ceil_div(kDctTab, 256), 256, 0, stream>>>();
        WEFTK_CUDA(cudaGetLastError());
        WEFTK_CUDA(cudaStreamSynchronize(stream));  // later calls may come on other streams
        g_tab_ready[dev] = true;
    }
    return WEFTK_OK;
}

int grid_for(long long total) {
    const long long blocks = (total + 255) / 256;
    return (int)(blocks < 148LL * 64 ? (blocks > 0 ? blocks : 1) : 148LL * 64);
}
}  // namespace

}  // namespace weftk

using namespace weftk;

extern "C" int weftk_dct_apply(const WeftDctTile* d_tiles, int n_tiles, const int16_t* d_coeffs, int64_t n_coeffs,
                               int chroma_mode, int band_layout, float quant_step, float freq_alpha, int max_size,
                               float* d_image, int width, int height, int clip_all, void* stream) {
    static_assert(sizeof(WeftDctTile) == 64, "WeftDctTile must be 64 bytes");
    WEFTK_REQUIRE(n_tiles >= 0 && n_coeffs >= 0, "dct_apply: negative count");
    WEFTK_REQUIRE(chroma_mode >= 0 && chroma_mode <= 2, "dct_apply: chroma_mode must be 0, 1 or 2");
    WEFTK_REQUIRE(band_layout == 0 || band_layout == 1, "dct_apply: layout must be 0 or 1");
    WEFTK_REQUIRE(width > 0 && height > 0 && d_image, "dct_apply: bad image");
    WEFTK_REQUIRE(max_size >= 4 && max_size <= WEFTK_DCT_MAX_TILE && (max_size & (max_size - 1)) == 0,
                  "dct_apply: max_size must be a power of two in 4..64");
    WEFTK_REQUIRE(!(freq_alpha < 0.0f), "dct_apply: freq_alpha must be >= 0");
    cudaStream_t s = (cudaStream_t)stream;
    if (n_tiles > 0) {
        WEFTK_REQUIRE(d_tiles && (d_coeffs || n_coeffs == 0), "dct_apply: null pointer");
        int rc = ensure_tables(s);
        if (rc != WEFTK_OK) return rc;
        const size_t smem = (size_t)max_size * max_size * (2 * sizeof(double) + 3 * sizeof(float));
        WEFTK_CUDA(cudaFuncSetAttribute(dct_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const double step = (double)quant_step;
        // a CTA of one thread per pixel of the launch's largest tile, at most 256: small tiles leave
        // no threads idle and more of their CTAs stay resident (every loop strides by blockDim.x)
        const int threads = std::min(256, std::max(32, max_size * max_size));
        dct_apply_kernel<<<n_tiles, threads, smem, s>>>(d_tiles, n_tiles, d_coeffs, (long long)n_coeffs, chroma_mode,
                                                    band_layout, step, step * 1.5, (double)freq_alpha, max_size,
                                                    d_image, width, height);
        WEFTK_CUDA(cudaGetLastError());
    }
    if (clip_all) {
        const long long n = (long long)width * height * 3;
        clip01_kernel<<<grid_for(n), 256, 0, s>>>(d_image, n);
        WEFTK_CUDA(cudaGetLastError());
    }
    return WEFTK_OK;
}

extern "C" int weftk_raster_resize(const float* d_src, int src_w, int src_h, float* d_dst, int dst_w, int dst_h,
                                   uint8_t* d_tmp, void* stream) {
    WEFTK_REQUIRE(d_src && d_dst && d_tmp, "raster_resize: null pointer");
    WEFTK_REQUIRE(src_w > 0 && src_h > 0 && dst_w > 0 && dst_h > 0 && src_w <= 65535 && src_h <= 65535 &&
                      dst_w <= 65535 && dst_h <= 65535,
                  "raster_resize: sizes must be in 1..65535");
    cudaStream_t s = (cudaStream_t)stream;
    const dim3 grid_r(ceil_div(dst_w, RS_COLS), ceil_div(src_h, RS_ROWS));
    const dim3 grid_c(ceil_div(dst_w, RS_COLS), ceil_div(dst_h, RS_ROWS));
    WEFTK_REQUIRE(grid_r.y <= 65535 && grid_c.y <= 65535, "raster_resize: image too tall");
    resize_rows_kernel<<<grid_r, RS_COLS, 0, s>>>(d_src, src_w, src_h, d_tmp, dst_w);
    WEFTK_CUDA(cudaGetLastError());
    resize_cols_kernel<<<grid_c, RS_COLS, 0, s>>>(d_tmp, src_h, dst_w, d_dst, dst_h);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}
