// weftk_pool.cu — initial constant / linear candidate pools generated on the device
// (include/weftk_pool.h).
//
// One CTA per tile, launched per tile side so that shared memory is sized for it.  The
// stages follow the reference's per-tile worker (src/weft/encoder.py:2490-2517):
//   1. pixels into shared memory as three channel planes; float32 luminance;
//   2. the reference's Sobel (src/weft/edge_analysis.py:17-41: every tap of its offset slices
//      reads lum[y-1][x-1], summed tap by tap in float32), magnitude, angle in [0, pi);
//   3. orientation histogram: pixels counting-sorted by bin (stable, raster order inside a
//      bin), then numpy's pairwise float32 sum per bin; the dominant orientations;
//   4. luminance sorted by (value, pixel index) for the palette runs and the 25th / 75th
//      percentiles; the np.gradient magnitude and its 75th percentile;
//   5. every mean the two generators take, as numpy computes it: a sequential float32 sum per
//      channel in the reference's pixel order (raster, or luminance order for palette runs),
//      divided by the count in float32 — one thread per (region, channel);
//   6. the candidate list in the reference's order (one thread), the coarse de-duplication
//      key of every candidate, first occurrences kept (one thread per candidate), and the
//      surviving records written to the tile's slots.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <set>

#include "../../include/weftk_pool.h"
#include "weftk_common.cuh"

namespace weftk {

extern __device__ int g_device_status;

namespace {

constexpr int NB = 12;                           // orientation histogram bins
constexpr int MAXC = WEFTK_POOL_MAX_CONST_LINEAR;
constexpr int MAXR = 33 + 2 * NB + 2 * WEFTK_POOL_MAX_SPECS;  // regions whose means are taken
constexpr int MAXPAL = 16;
constexpr int KEYS = 12;

enum : int { RG_ALL, RG_RECT, RG_RUN, RG_LUM_GT, RG_LUM_LT, RG_MAGT_GE, RG_SIDE_A, RG_SIDE_B };

struct Region {
    int type;
    int a, b, c, d;  // rect rows [a, b) x cols [c, d); run [a, b) of the luminance order
    float4 coef;     // threshold in x; side test coefficients x0, y0, y1 - y0, x1 - x0
};

// per-tile scratch besides the pixel planes (static part of the shared memory)
struct Scratch {
    Region reg[MAXR];
    float rsum[MAXR][3];
    int rcnt[MAXR];
    int n_reg;
    float hist[NB];
    int bin_start[NB + 1];
    int peaks[NB];
    int n_peaks;
    float p25, p75, pm75;
    // palettes (the template palette extends the edge palette) and the candidate list's segments
    float pal[MAXPAL][3];
    int npal_e, npal_t;
    int seg[8];
    int n_cand;
    unsigned long long hash[MAXC];
    int keep[MAXC];
    int n_out;
    int wcnt[16][NB];
};

__device__ __forceinline__ float clamp01(float v) { return fmaxf(0.0f, fminf(1.0f, v)); }

// numpy's pairwise float32 summation of x[0..n) (the contiguous add-reduce loop: fewer than 8
// sequentially, up to 128 with 8 accumulators combined pairwise, larger halves split at a
// multiple of 8), each addition rounded on its own.
__device__ float pairwise_sum(const float* x, int n) {
    if (n < 8) {
        float r = -0.0f;
        for (int i = 0; i < n; ++i) r = __fadd_rn(r, x[i]);
        return r;
    }
    if (n <= 128) {
        float r[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) r[j] = x[j];
        int i = 8;
        for (; i < n - (n % 8); i += 8) {
#pragma unroll
            for (int j = 0; j < 8; ++j) r[j] = __fadd_rn(r[j], x[i + j]);
        }
        float res = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[1]), __fadd_rn(r[2], r[3])),
                              __fadd_rn(__fadd_rn(r[4], r[5]), __fadd_rn(r[6], r[7])));
        for (; i < n; ++i) res = __fadd_rn(res, x[i]);
        return res;
    }
    int n2 = n / 2;
    n2 -= n2 % 8;
    return __fadd_rn(pairwise_sum(x, n2), pairwise_sum(x + n2, n - n2));
}

// numpy's linear percentile of sorted float32 values (the whole computation in float32:
// q / 100, the virtual index (n - 1) q, gamma, and the two-sided lerp).
__device__ float percentile_sorted(const float* s, int n, int q) {
    const float qf = __fdiv_rn((float)q, 100.0f);
    const float vi = __fmul_rn((float)(n - 1), qf);
    const int lo = (int)floorf(vi);
    const int hi = min(lo + 1, n - 1);
    const float g = __fsub_rn(vi, (float)lo);
    const float a = s[lo], b = s[hi];
    const float d = __fsub_rn(b, a);
    if (g >= 0.5f) return __fsub_rn(b, __fmul_rn(d, __fsub_rn(1.0f, g)));
    return __fadd_rn(a, __fmul_rn(d, g));
}

// side test of the reference's split: (x - x0) * (y1 - y0) - (y - y0) * (x1 - x0) >= 0 in float32
__device__ __forceinline__ bool side_a(float4 c, int x, int y) {
    const float t = __fsub_rn(__fmul_rn(__fsub_rn((float)x, c.x), c.z), __fmul_rn(__fsub_rn((float)y, c.y), c.w));
    return t >= 0.0f;
}

// sum over (a - b)^2 < 0.002 in float64, as the reference's palette test (Python floats)
__device__ bool near_any(const float* c, const float (*pal)[3], int n) {
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) {
            const double d = __dsub_rn((double)c[k], (double)pal[i][k]);
            s = __dadd_rn(s, __dmul_rn(d, d));
        }
        if (s < 0.002) return true;
    }
    return false;
}

__device__ __forceinline__ int qkey(double v, double s) { return (int)(long long)__dadd_rn(__dmul_rn(v, s), 0.5); }

// Dynamic shared memory of one tile of N pixels: seven float planes (r, g, b, luminance, the
// np.gradient magnitude, the Sobel magnitude, a sort key), the sorted pixel indices, the bins.
constexpr size_t POOL_FLOAT_PLANES = 7;
__host__ __device__ constexpr size_t pool_smem_bytes(int n) {
    return (size_t)n * (POOL_FLOAT_PLANES * sizeof(float) + sizeof(int) + sizeof(uint8_t));
}

template <int TS, int NT>
__global__ void __launch_bounds__(NT) gen_pool_kernel(WeftPoolTables tb, WeftPoolJob job, int si, int quality) {
    constexpr int N = TS * TS;
    constexpr int NW = NT / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* col = reinterpret_cast<float*>(smem_raw);  // [3][N]
    float* lum = col + 3 * N;                         // [N]
    float* magt = lum + N;                            // [N] np.gradient magnitude
    float* mags = magt + N;                           // [N] Sobel magnitude, then sorted magt
    float* skey = mags + N;                           // [N] bin-sorted magnitudes, then sorted lum
    int* sidx = reinterpret_cast<int*>(skey + N);     // [N] pixel of each sorted luminance
    uint8_t* bin = reinterpret_cast<uint8_t*>(sidx + N);  // [N]
    static_assert(POOL_FLOAT_PLANES == 7, "the planes above are col[3], lum, magt, mags, skey");
    static_assert(NW <= 16, "the histogram's per-warp counters hold 16 warps");
    __shared__ Scratch S;
    (void)quality;

    const int t = job.tiles[si][blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool want0 = job.kinds_mask & 1, want1 = job.kinds_mask & 2;

    // 1. pixels and luminance 0.2126 r + 0.7152 g + 0.0722 b (float32, left to right)
    const float4* src = reinterpret_cast<const float4*>(job.src) + job.px_off[t];
    for (int p = tid; p < N; p += NT) {
        const float4 v = src[p];
        col[p] = v.x;
        col[N + p] = v.y;
        col[2 * N + p] = v.z;
        lum[p] = __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, v.x), __fmul_rn(0.7152f, v.y)), __fmul_rn(0.0722f, v.z));
    }
    __syncthreads();

    // 2. the reference's Sobel: gx[y][x] = sum over the taps (dy, dx) whose slices reach (y, x)
    //    of k[dy][dx] * lum[y-1][x-1]; rows reached: dy 0 -> 1..TS-2, 1 -> 1..TS-1, 2 -> 2..TS-1
    //    (columns alike), angle = arctan2 rounded to float32, then numpy's float32 % pi.
    //    np.gradient (template): central differences / 2 inside, one-sided at the edges.
    constexpr float KX[9] = {-1, 0, 1, -2, 0, 2, -1, 0, 1};
    constexpr float KY[9] = {-1, -2, -1, 0, 0, 0, 1, 2, 1};
    const float PI32 = 3.14159274101257324f;  // float32(pi): numpy casts the Python float
    for (int p = tid; p < N; p += NT) {
        const int y = p / TS, x = p % TS;
        float gx = 0.0f, gy = 0.0f;
        if (y >= 1 && x >= 1) {
            const float L = lum[(y - 1) * TS + (x - 1)];
#pragma unroll
            for (int dy = 0; dy < 3; ++dy) {
                const bool row = dy == 0 ? (y <= TS - 2) : dy == 1 ? true : (y >= 2);
#pragma unroll
                for (int dx = 0; dx < 3; ++dx) {
                    const bool cl = dx == 0 ? (x <= TS - 2) : dx == 1 ? true : (x >= 2);
                    if (row && cl) {
                        gx = __fadd_rn(gx, __fmul_rn(KX[dy * 3 + dx], L));
                        gy = __fadd_rn(gy, __fmul_rn(KY[dy * 3 + dx], L));
                    }
                }
            }
        }
        mags[p] = __fsqrt_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)));
        float ang = (float)atan2((double)gy, (double)gx);
        float m = fmodf(ang, PI32);
        if (m != 0.0f) {
            if (m < 0.0f) m = __fadd_rn(m, PI32);
        } else {
            m = 0.0f;
        }
        int b = NB;  // no bin (NaN)
        const double md = (double)m;
        for (int i = 0; i < NB; ++i)
            if (md >= tb.bin_edges[i] && md < tb.bin_edges[i + 1]) {
                b = i;
                break;
            }
        bin[p] = (uint8_t)b;
        // np.gradient along rows (gy) and columns (gx)
        const float* L = lum;
        const float ty = y == 0 ? __fsub_rn(L[TS + x], L[x])
                         : y == TS - 1 ? __fsub_rn(L[p], L[p - TS])
                                       : __fdiv_rn(__fsub_rn(L[p + TS], L[p - TS]), 2.0f);
        const float tx = x == 0 ? __fsub_rn(L[p + 1], L[p])
                         : x == TS - 1 ? __fsub_rn(L[p], L[p - 1])
                                       : __fdiv_rn(__fsub_rn(L[p + 1], L[p - 1]), 2.0f);
        magt[p] = __fsqrt_rn(__fadd_rn(__fmul_rn(tx, tx), __fmul_rn(ty, ty)));
    }
    for (int i = tid; i < 16 * NB; i += NT) (&S.wcnt[0][0])[i] = 0;
    __syncthreads();

    // 3. histogram: stable counting sort of the Sobel magnitudes by bin into skey
    if (want1) {
        constexpr int CHUNK = N / NW;
        const int lo = warp * CHUNK;
        for (int base = lo; base < lo + CHUNK; base += 32) {
            const int b = bin[base + lane];
            const unsigned m = __match_any_sync(0xffffffffu, b);
            if (lane == __ffs(m) - 1 && b < NB) S.wcnt[warp][b] += __popc(m);
            __syncwarp();
        }
        __syncthreads();
        if (tid == 0) {
            int off = 0;
            for (int b = 0; b < NB; ++b) {
                S.bin_start[b] = off;
                for (int w = 0; w < NW; ++w) {
                    const int c = S.wcnt[w][b];
                    S.wcnt[w][b] = off;
                    off += c;
                }
            }
            S.bin_start[NB] = off;
        }
        __syncthreads();
        for (int base = lo; base < lo + CHUNK; base += 32) {
            const int b = bin[base + lane];
            const unsigned m = __match_any_sync(0xffffffffu, b);
            if (b < NB) skey[S.wcnt[warp][b] + __popc(m & ((1u << lane) - 1u))] = mags[base + lane];
            __syncwarp();
            if (lane == __ffs(m) - 1 && b < NB) S.wcnt[warp][b] += __popc(m);
            __syncwarp();
        }
        __syncthreads();
        if (tid < NB) S.hist[tid] = pairwise_sum(skey + S.bin_start[tid], S.bin_start[tid + 1] - S.bin_start[tid]);
        __syncthreads();
        if (tid == 0) {
            float hmax = S.hist[0];
            for (int i = 1; i < NB; ++i) hmax = fmaxf(hmax, S.hist[i]);
            int np = 0;
            if (hmax < 1e-6f) {
                for (int i = 0; i < 4; ++i) S.peaks[np++] = NB + i;
            } else {
                const float thr = __fmul_rn(hmax, 0.2f);
                for (int i = 0; i < NB; ++i)
                    if (S.hist[i] >= thr) S.peaks[np++] = i;
            }
            S.n_peaks = np;
        }
    }

    // 4. luminance sorted by (value, index); magt copied for its own sort
    for (int p = tid; p < N; p += NT) {
        skey[p] = lum[p];
        sidx[p] = p;
        mags[p] = magt[p];
    }
    __syncthreads();
    for (int k = 2; k <= N; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < N; i += NT) {
                const int o = i ^ j;
                if (o > i) {
                    const bool up = (i & k) == 0;
                    const float a = skey[i], b = skey[o];
                    const int ia = sidx[i], ib = sidx[o];
                    const bool gt = a > b || (a == b && ia > ib);
                    if (gt == up) {
                        skey[i] = b;
                        skey[o] = a;
                        sidx[i] = ib;
                        sidx[o] = ia;
                    }
                    const float ma = mags[i], mb = mags[o];
                    if ((ma > mb) == up) {
                        mags[i] = mb;
                        mags[o] = ma;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (tid == 0) {
        S.p25 = percentile_sorted(skey, N, 25);
        S.p75 = percentile_sorted(skey, N, 75);
        S.pm75 = percentile_sorted(mags, N, 75);
        // regions, in a fixed order
        int r = 0;
        S.reg[r++] = Region{RG_ALL, 0, TS, 0, TS, make_float4(0, 0, 0, 0)};
        const int qh = TS / 2, sh = TS / 4;
        for (int a = 0; a < 2; ++a)
            for (int c = 0; c < 2; ++c)
                S.reg[r++] = Region{RG_RECT, a * qh, (a + 1) * qh, c * qh, (c + 1) * qh, make_float4(0, 0, 0, 0)};
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < 4; ++c)
                S.reg[r++] = Region{RG_RECT, a * sh, (a + 1) * sh, c * sh, (c + 1) * sh, make_float4(0, 0, 0, 0)};
        for (int k = 0; k < 3; ++k)
            for (int j = 0; j < k + 2; ++j) {
                const int* cut = tb.cuts + (si * 3 + k) * 5;
                S.reg[r++] = Region{RG_RUN, cut[j], cut[j + 1], 0, 0, make_float4(0, 0, 0, 0)};
            }
        S.reg[r++] = Region{RG_LUM_GT, 0, 0, 0, 0, make_float4(S.p75, 0, 0, 0)};
        S.reg[r++] = Region{RG_LUM_LT, 0, 0, 0, 0, make_float4(S.p25, 0, 0, 0)};
        S.reg[r++] = Region{RG_MAGT_GE, 0, 0, 0, 0, make_float4(S.pm75, 0, 0, 0)};
        if (want1) {
            for (int i = 0; i < S.n_peaks; ++i) {
                const float* m = tb.orient_mask + (si * 16 + S.peaks[i]) * 4;
                const float4 c = make_float4(m[0], m[1], m[2], m[3]);
                S.reg[r++] = Region{RG_SIDE_A, 0, 0, 0, 0, c};
                S.reg[r++] = Region{RG_SIDE_B, 0, 0, 0, 0, c};
            }
            for (int i = 0; i < tb.n_spec; ++i) {
                const float* m = tb.spec_mask + (si * WEFTK_POOL_MAX_SPECS + i) * 4;
                const float4 c = make_float4(m[0], m[1], m[2], m[3]);
                S.reg[r++] = Region{RG_SIDE_A, 0, 0, 0, 0, c};
                S.reg[r++] = Region{RG_SIDE_B, 0, 0, 0, 0, c};
            }
        }
        S.n_reg = r;
    }
    __syncthreads();

    // 5. one thread per (region, channel): sequential float32 sum in the reference's order
    for (int ch = tid; ch < S.n_reg * 3; ch += NT) {
        const int ri = ch / 3, c = ch % 3;
        const Region R = S.reg[ri];
        const float* pl = col + c * N;
        float s = 0.0f;
        int cnt = 0;
        switch (R.type) {
            case RG_ALL:
            case RG_RECT:
                for (int y = R.a; y < R.b; ++y)
                    for (int x = R.c; x < R.d; ++x) s = __fadd_rn(s, pl[y * TS + x]);
                cnt = (R.b - R.a) * (R.d - R.c);
                break;
            case RG_RUN:
                for (int k = R.a; k < R.b; ++k) s = __fadd_rn(s, pl[sidx[k]]);
                cnt = R.b - R.a;
                break;
            case RG_LUM_GT:
                for (int p = 0; p < N; ++p)
                    if (lum[p] > R.coef.x) {
                        s = __fadd_rn(s, pl[p]);
                        ++cnt;
                    }
                break;
            case RG_LUM_LT:
                for (int p = 0; p < N; ++p)
                    if (lum[p] < R.coef.x) {
                        s = __fadd_rn(s, pl[p]);
                        ++cnt;
                    }
                break;
            case RG_MAGT_GE:
                for (int p = 0; p < N; ++p)
                    if (magt[p] >= R.coef.x) {
                        s = __fadd_rn(s, pl[p]);
                        ++cnt;
                    }
                break;
            default: {
                const bool want_a = R.type == RG_SIDE_A;
                for (int y = 0; y < TS; ++y)
                    for (int x = 0; x < TS; ++x)
                        if (side_a(R.coef, x, y) == want_a) {
                            s = __fadd_rn(s, pl[y * TS + x]);
                            ++cnt;
                        }
            }
        }
        S.rsum[ri][c] = s;
        if (c == 0) S.rcnt[ri] = cnt;
    }
    __syncthreads();

    // 6. palettes (one thread; a handful of means and distance tests), then the candidate list's
    //    segment sizes: the list is (edge pool) palette x 4 alphas, quadrants x 2, orientations x 5,
    //    (template pool) palette x 4, quadrants x 2, blocks, splits x 3 or x 1, so candidate i is
    //    a function of i that any thread can evaluate (cand_at below)
    if (tid == 0) {
        float avg[3];
        for (int c = 0; c < 3; ++c) avg[c] = clamp01(__fdiv_rn(S.rsum[0][c], (float)S.rcnt[0]));
        int npal = 1;
        for (int c = 0; c < 3; ++c) S.pal[0][c] = avg[c];
        for (int r = 21; r < 33; ++r) {
            if (r == 30) S.npal_e = npal;  // the template palette adds bright / dark / edge colours
            const Region R = S.reg[r];
            float m[3];
            if (r < 30 && R.b <= R.a) {
                const int p = sidx[min(R.a, N - 1)];
                for (int c = 0; c < 3; ++c) m[c] = col[c * N + p];
            } else if (S.rcnt[r] > 0) {
                for (int c = 0; c < 3; ++c) m[c] = __fdiv_rn(S.rsum[r][c], (float)S.rcnt[r]);
            } else {
                for (int c = 0; c < 3; ++c) m[c] = avg[c];
            }
            for (int c = 0; c < 3; ++c) m[c] = clamp01(m[c]);
            if (!near_any(m, S.pal, npal) && npal < MAXPAL) {
                for (int c = 0; c < 3; ++c) S.pal[npal][c] = m[c];
                ++npal;
            }
        }
        S.npal_t = npal;
        const int sz[7] = {want0 ? S.npal_e * 4 : 0, want0 ? 8 : 0, want1 ? S.n_peaks * 5 : 0,
                           want0 ? S.npal_t * 4 : 0, want0 ? 8 : 0, want0 ? 16 : 0,
                           want1 ? tb.n_centre * 3 + (tb.n_spec - tb.n_centre) : 0};
        S.seg[0] = 0;
        for (int k = 0; k < 7; ++k) S.seg[k + 1] = S.seg[k] + sz[k];
        S.n_cand = min(S.seg[7], MAXC);
        if (S.seg[7] > MAXC) atomicCAS(&g_device_status, 0, WEFTK_E_RANGE);
    }
    __syncthreads();

    // candidate i: kind, float64 geometry (the reference's Python values), colours, alpha
    auto cand_at = [&](int i, int& kind, double (&g)[4], float (&c0)[3], float (&c1)[3], double& alpha) {
        const double A4[4] = {1.0, 0.7, 0.4, 0.2};
        const double A3[3] = {1.0, 0.7, 0.4};
        auto mean_clamped = [&](int r, float (&m)[3]) {
            for (int c = 0; c < 3; ++c) m[c] = clamp01(__fdiv_rn(S.rsum[r][c], (float)S.rcnt[r]));
        };
        kind = 0;
        for (int k = 0; k < 4; ++k) g[k] = 0.0;
        for (int c = 0; c < 3; ++c) c1[c] = 0.0f;
        int k = 0;
        while (i >= S.seg[k + 1]) ++k;
        const int j = i - S.seg[k];
        switch (k) {
            case 0:
            case 3:  // palette colour x alphas 1, .7, .4, .2
                for (int c = 0; c < 3; ++c) c0[c] = S.pal[j >> 2][c];
                alpha = A4[j & 3];
                break;
            case 1:
            case 4:  // quadrant mean x alphas .5, .3
                mean_clamped(1 + (j >> 1), c0);
                alpha = (j & 1) ? 0.3 : 0.5;
                break;
            case 2: {  // orientation split: centre x 1, .7, .4, offsets at 0.25 and 0.75 x .5
                const int pk = j / 5, m = j - pk * 5, r = 33 + 2 * pk;
                float avg[3];
                for (int c = 0; c < 3; ++c) avg[c] = clamp01(__fdiv_rn(S.rsum[0][c], (float)S.rcnt[0]));
                if (S.rcnt[r] > 0) mean_clamped(r, c0);
                else
                    for (int c = 0; c < 3; ++c) c0[c] = avg[c];
                if (S.rcnt[r + 1] > 0) mean_clamped(r + 1, c1);
                else
                    for (int c = 0; c < 3; ++c) c1[c] = avg[c];
                const double* gg = tb.orient_geom + ((size_t)(si * 16 + S.peaks[pk]) * 3 + (m < 3 ? 0 : m - 2)) * 4;
                for (int q = 0; q < 4; ++q) g[q] = gg[q];
                alpha = m < 3 ? A3[m] : 0.5;
                kind = 1;
                break;
            }
            case 5:  // 4x4 block mean x .25
                mean_clamped(5 + j, c0);
                alpha = 0.25;
                break;
            default: {  // template split: batched side means, not clamped; an empty side takes the
                        // (unclamped) tile mean
                const int sp = j < tb.n_centre * 3 ? j / 3 : tb.n_centre + (j - tb.n_centre * 3);
                alpha = j < tb.n_centre * 3 ? A3[j % 3] : 0.5;
                const int r = 33 + 2 * S.n_peaks + 2 * sp;
                for (int c = 0; c < 3; ++c) {
                    const float fb = __fdiv_rn(S.rsum[0][c], (float)S.rcnt[0]);
                    c0[c] = S.rcnt[r] > 0 ? __fdiv_rn(S.rsum[r][c], (float)S.rcnt[r]) : fb;
                    c1[c] = S.rcnt[r + 1] > 0 ? __fdiv_rn(S.rsum[r + 1][c], (float)S.rcnt[r + 1]) : fb;
                }
                const double* gg = tb.spec_geom + (size_t)(si * WEFTK_POOL_MAX_SPECS + sp) * 4;
                for (int q = 0; q < 4; ++q) g[q] = gg[q];
                kind = 1;
            }
        }
    };
    // the reference's coarse de-duplication key: kind, geometry x4, colour0 x64, alpha x32,
    // colour1 x64 for a linear patch (each int(v * s + 0.5), truncating toward zero)
    auto key_of = [&](int i, int (&key)[KEYS]) {
        int kind;
        double g[4], alpha;
        float c0[3], c1[3];
        cand_at(i, kind, g, c0, c1, alpha);
        key[0] = kind;
        for (int j = 0; j < 4; ++j) key[1 + j] = kind == 1 ? qkey(g[j], 4.0) : 0;
        for (int j = 0; j < 3; ++j) key[5 + j] = qkey((double)c0[j], 64.0);
        key[8] = qkey(alpha, 32.0);
        for (int j = 0; j < 3; ++j) key[9 + j] = kind == 1 ? qkey((double)c1[j], 64.0) : 0;
    };

    // 7. first occurrences kept: 64-bit hashes of the keys, the full keys compared on a match
    const int nc = S.n_cand;
    for (int i = tid; i < nc; i += NT) {
        int key[KEYS];
        key_of(i, key);
        unsigned long long h = 0x9e3779b97f4a7c15ull;
        for (int k = 0; k < KEYS; ++k) {
            h = (h ^ (unsigned long long)(unsigned)key[k]) * 0xff51afd7ed558ccdull;
            h ^= h >> 33;
        }
        S.hash[i] = h;
    }
    __syncthreads();
    for (int i = tid; i < nc; i += NT) {
        const unsigned long long h = S.hash[i];
        bool dup = false;
        for (int j = 0; j < i && !dup; ++j) {
            if (S.hash[j] != h) continue;
            int a[KEYS], b[KEYS];
            key_of(i, a);
            key_of(j, b);
            bool same = true;
            for (int k = 0; k < KEYS; ++k) same = same && a[k] == b[k];
            dup = same;
        }
        S.keep[i] = !dup;
    }
    __syncthreads();
    if (tid == 0) {
        int n = 0;
        for (int i = 0; i < nc; ++i) {
            const int k = S.keep[i];
            S.keep[i] = k ? n : -1;  // output position, -1 = dropped
            n += k;
        }
        if (n > job.pool_cap) {
            atomicCAS(&g_device_status, 0, WEFTK_E_RANGE);
            n = job.pool_cap;
        }
        S.n_out = n;
        job.pool_cnt[t] = n;
    }
    __syncthreads();
    WeftPrim* out = job.cand + job.pool_off[t];
    for (int i = tid; i < nc; i += NT) {
        const int pos = S.keep[i];
        if (pos < 0 || pos >= S.n_out) continue;
        int kind;
        double g[4], alpha;
        float c0[3], c1[3];
        cand_at(i, kind, g, c0, c1, alpha);
        WeftPrim p;
        p.kind = kind;
        for (int j = 0; j < 7; ++j) p.geom[j] = j < 4 ? (float)g[j] : 0.0f;
        for (int j = 0; j < 3; ++j) {
            p.color0[j] = c0[j];
            p.color1[j] = c1[j];
        }
        p.alpha = (float)alpha;
        out[pos] = p;
    }
}

template <int TS, int NT>
int launch_gen(const WeftPoolTables& tb, const WeftPoolJob& job, int si, cudaStream_t stream) {
    const int n = job.n_tiles[si];
    if (n == 0) return WEFTK_OK;
    constexpr int N = TS * TS;
    const size_t dyn = (pool_smem_bytes(N) + 15) / 16 * 16;
    // the static scratch and the pixel planes together exceed the default 48 KB: opt in once
    // per device (under a lock, so concurrent first calls agree)
    {
        int dev = 0;
        WEFTK_CUDA(cudaGetDevice(&dev));
        static std::mutex mu;
        static std::set<int> done;
        std::lock_guard<std::mutex> lock(mu);
        if (!done.count(dev)) {
            WEFTK_CUDA(cudaFuncSetAttribute(gen_pool_kernel<TS, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)dyn));
            done.insert(dev);
        }
    }
    gen_pool_kernel<TS, NT><<<n, NT, dyn, stream>>>(tb, job, si, 0);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}

}  // namespace
}  // namespace weftk

using namespace weftk;

// Side streams of the current device that run the larger tile classes beside the 8-px class
// (forked from and joined back into the caller's stream with events, so a captured graph gets
// parallel branches).  Created on the first call on a device.
struct SideStreams {
    cudaStream_t s[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[3] = {nullptr, nullptr, nullptr};
};

int side_streams(SideStreams** out) {
    static std::mutex mu;
    static SideStreams per_dev[64];
    int dev = 0;
    WEFTK_CUDA(cudaGetDevice(&dev));
    WEFTK_REQUIRE(dev >= 0 && dev < 64, "gen_pools: device index beyond 63");
    std::lock_guard<std::mutex> lock(mu);
    SideStreams& ss = per_dev[dev];
    if (!ss.fork) {
        for (int i = 0; i < 3; ++i) {
            WEFTK_CUDA(cudaStreamCreateWithFlags(&ss.s[i], cudaStreamNonBlocking));
            WEFTK_CUDA(cudaEventCreateWithFlags(&ss.join[i], cudaEventDisableTiming));
        }
        WEFTK_CUDA(cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming));
    }
    *out = &ss;
    return WEFTK_OK;
}

extern "C" int weftk_gen_pools(const WeftPoolTables* tables, const WeftPoolJob* job, void* stream) {
    WEFTK_REQUIRE(tables && job, "gen_pools: null argument");
    WEFTK_REQUIRE(tables->n_spec >= 0 && tables->n_spec <= WEFTK_POOL_MAX_SPECS &&
                      tables->n_centre >= 0 && tables->n_centre <= tables->n_spec,
                  "gen_pools: bad template table");
    WEFTK_REQUIRE(job->pool_cap >= WEFTK_POOL_MAX_CONST_LINEAR, "gen_pools: pool_cap below the per-tile bound");
    WEFTK_REQUIRE((job->kinds_mask & ~3) == 0, "gen_pools: only constant and linear patches are generated");
    int any = 0;
    for (int i = 0; i < 4; ++i) {
        WEFTK_REQUIRE(job->n_tiles[i] >= 0, "gen_pools: negative tile count");
        any |= job->n_tiles[i] > 0;
        WEFTK_REQUIRE(job->n_tiles[i] == 0 || job->tiles[i], "gen_pools: null tile list");
    }
    if (!any) return WEFTK_OK;
    WEFTK_REQUIRE(job->src && job->px_off && job->pool_off && job->cand && job->pool_cnt, "gen_pools: null pointer");
    WEFTK_REQUIRE(tables->bin_edges && tables->cuts && tables->orient_geom && tables->orient_mask &&
                      (tables->n_spec == 0 || (tables->spec_geom && tables->spec_mask)),
                  "gen_pools: null table");
    cudaStream_t s = (cudaStream_t)stream;
    SideStreams* ss = nullptr;
    int rc = side_streams(&ss);
    if (rc) return rc;
    // the 64-, 32- and 16-px classes (few CTAs, long ones) on side streams, the 8-px class here
    WEFTK_CUDA(cudaEventRecord(ss->fork, s));
    for (int i = 0; i < 3; ++i) WEFTK_CUDA(cudaStreamWaitEvent(ss->s[i], ss->fork, 0));
    if ((rc = launch_gen<64, 512>(*tables, *job, 3, ss->s[0]))) return rc;
    if ((rc = launch_gen<32, 256>(*tables, *job, 2, ss->s[1]))) return rc;
    if ((rc = launch_gen<16, 128>(*tables, *job, 1, ss->s[2]))) return rc;
    if ((rc = launch_gen<8, 64>(*tables, *job, 0, s))) return rc;
    for (int i = 0; i < 3; ++i) {
        WEFTK_CUDA(cudaEventRecord(ss->join[i], ss->s[i]));
        WEFTK_CUDA(cudaStreamWaitEvent(s, ss->join[i], 0));
    }
    return WEFTK_OK;
}
