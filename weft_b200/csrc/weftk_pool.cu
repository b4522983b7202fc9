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
//      divided by the count in float32 — one thread per region or split line (both of its
//      sides in one pass over the pixels, the side test read from a table built once per
//      quality), over all three channels for tiles up to 16 px and one channel above; each
//      sum divided by its count in float32 there, once per region;
//   6. the palettes (the colours' pairwise near tests in parallel, the keep walk on one
//      thread) and the candidate list's segments;
//   7. the coarse de-duplication key of every candidate, first occurrences kept through a
//      shared-memory hash table (lowest index per key), and the surviving records written to
//      the tile's slots.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <set>

#include "../../include/weftk_pool.h"
#include "weftk_common.cuh"

static_assert(sizeof(WeftPoolTables) == 64, "WeftPoolTables layout is part of the C ABI");

namespace weftk {

extern __device__ int g_device_status;

namespace {

constexpr int NB = 12;                           // orientation histogram bins
constexpr int MAXC = WEFTK_POOL_MAX_CONST_LINEAR;
constexpr int NSPL = WEFTK_POOL_SPLITS;          // split rows per tile side in the side-bit table
constexpr int NFIX = 33;                         // fixed regions (below)
constexpr int MAXPAL = 16;
constexpr int NCOL = 13;                         // palette colours tested: tile mean + regions 21..32
constexpr int KEYS = 12;
constexpr int HT = 512;                          // de-duplication hash table slots (> 2 * MAXC)

// Fixed regions whose means are taken: 0 the tile, 1..4 its quadrants, 5..20 its 4x4 blocks
// (row-major), 21..29 the palette runs of the luminance order (2, 3 and 4 equal runs), 30
// luminance above its 75th percentile, 31 below its 25th, 32 np.gradient magnitude at or above
// its 75th.  Split lines (both sides) are kept apart: the dominant orientations' centre lines,
// then the template lines.

// per-tile scratch besides the pixel planes (static part of the shared memory)
struct Scratch {
    float rmean[NFIX][3];     // sum / count in float32 (0 for an empty region)
    int rcnt[NFIX];
    float smean[NSPL][2][3];  // per split line in use: side a, side b (0 for an empty side)
    int scnt[NSPL];           // pixels on side a
    double edges[NB + 1];
    float hist[NB];
    int bin_start[NB + 1];
    int peaks[NB];
    int n_peaks, n_split;
    float p25, p75, pm75;
    unsigned tmask[3][128];  // pixels above the 75th / below the 25th luminance percentile, gradient >= its 75th
    // palettes (the template palette extends the edge palette) and the candidate list's segments
    float cpal[NCOL][3];
    unsigned near_mask[NCOL];
    float pal[MAXPAL][3];
    int npal_e, npal_t;
    int seg[8];
    int n_cand;
    unsigned long long hash[MAXC];
    unsigned long long klo[MAXC], khi[MAXC];
    unsigned long long ht_hash[HT];
    int ht_idx[HT];
    unsigned keepw[(MAXC + 31) / 32];
    int keep_pre[(MAXC + 31) / 32];
    int n_out;
    int wcnt[16][NB];
};

__device__ __forceinline__ float clamp01(float v) { return fmaxf(0.0f, fminf(1.0f, v)); }

// numpy's pairwise float32 summation of x[0..n) (the contiguous add-reduce loop: fewer than 8
// sequentially, up to 128 with 8 accumulators combined pairwise, larger halves split at a
// multiple of 8), each addition rounded on its own.  The split tree is walked with an explicit
// stack (no recursion, so the kernel's stack size stays static): depth 6 covers n <= 8192.
__device__ float pairwise_block(const float* x, int n) {
    if (n < 8) {
        float r = -0.0f;
        for (int i = 0; i < n; ++i) r = __fadd_rn(r, x[i]);
        return r;
    }
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

// numpy's split tree over n elements, post-order: leaf(off, len) gives a leaf's sum (len <= 128),
// the two halves of an inner node are added left + right
template <class Leaf>
__device__ float pairwise_tree(int n, Leaf leaf) {
    constexpr int DEPTH = 8;
    int off[DEPTH], len[DEPTH], state[DEPTH];
    float left[DEPTH];
    int sp = 0;
    off[0] = 0;
    len[0] = n;
    state[0] = 0;
    float ret = 0.0f;
    while (sp >= 0) {
        const int m = len[sp];
        if (m <= 128 || sp == DEPTH - 1) {  // a leaf (n <= 8192 never reaches the depth bound)
            ret = leaf(off[sp], m);
            --sp;
            continue;
        }
        int m2 = m / 2;
        m2 -= m2 % 8;
        if (state[sp] == 0) {  // left half first
            state[sp] = 1;
            off[sp + 1] = off[sp];
            len[sp + 1] = m2;
            state[sp + 1] = 0;
            ++sp;
        } else if (state[sp] == 1) {  // then the right half
            left[sp] = ret;
            state[sp] = 2;
            off[sp + 1] = off[sp] + m2;
            len[sp + 1] = m - m2;
            state[sp + 1] = 0;
            ++sp;
        } else {
            ret = __fadd_rn(left[sp], ret);
            --sp;
        }
    }
    return ret;
}

__device__ float pairwise_sum(const float* x, int n) {
    return pairwise_tree(n, [&](int o, int m) { return pairwise_block(x + o, m); });
}

// the same sum by a whole warp (every lane gets it): the tree's leaves listed in order in lw
// (3 * cap words: offsets, lengths, sums; cap >= the leaf count), summed by the lanes in
// parallel, then the tree combined in numpy's order
__device__ float warp_pairwise_sum(const float* x, int n, int* lw, int cap, int lane) {
    int nl = 0;
    pairwise_tree(n, [&](int o, int m) {
        if (lane == 0) {
            lw[nl] = o;
            lw[cap + nl] = m;
        }
        ++nl;
        return 0.0f;
    });
    __syncwarp();
    float* sums = reinterpret_cast<float*>(lw + 2 * cap);
    for (int k = lane; k < nl; k += 32) sums[k] = pairwise_block(x + lw[k], lw[cap + k]);
    __syncwarp();
    int k = 0;
    const float r = pairwise_tree(n, [&](int, int) { return sums[k++]; });
    __syncwarp();
    return r;
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
__device__ bool near_pair(const float* c, const float* p) {
    double s = 0.0;
    for (int k = 0; k < 3; ++k) {
        const double d = __dsub_rn((double)c[k], (double)p[k]);
        s = __dadd_rn(s, __dmul_rn(d, d));
    }
    return s < 0.002;
}

__device__ __forceinline__ int qkey(double v, double s) { return (int)(long long)__dadd_rn(__dmul_rn(v, s), 0.5); }

// Dynamic shared memory of one tile of N pixels: seven float planes (r, g, b, luminance, the
// np.gradient magnitude, the Sobel magnitude, a sort key), the sorted pixel indices, the bins.
constexpr size_t POOL_FLOAT_PLANES = 7;
__host__ __device__ constexpr size_t pool_smem_bytes(int n) {
    return (size_t)n * (POOL_FLOAT_PLANES * sizeof(float) + sizeof(int) + sizeof(uint8_t));
}

// words of the side-bit table before tile side TS (8, 16, 32, 64), per split row
template <int TS>
__host__ __device__ constexpr int side_words_before() {
    return TS == 8 ? 0 : TS == 16 ? 2 : TS == 32 ? 10 : 42;
}

// run [a, b) of the luminance order behind palette region r (21..29: 2, 3 and 4 equal runs)
__device__ __forceinline__ void run_bounds(const int32_t* cuts, int si, int r, int& a, int& b) {
    const int j = r - 21;
    const int k = j < 2 ? 0 : j < 5 ? 1 : 2;
    const int jj = j - (k == 0 ? 0 : k == 1 ? 2 : 5);
    const int32_t* cut = cuts + (si * 3 + k) * 5;
    a = cut[jj];
    b = cut[jj + 1];
}

// the 12 key fields packed into 123 bits when each lies in its field's range (kind 1 bit, alpha
// 6, geometry 11 each, colours 12 each, signed by offset); bit 63 of hi marks a key that does
// not pack, whose equality is then decided on the unpacked fields
__device__ void pack_key(const int (&key)[KEYS], unsigned long long& lo, unsigned long long& hi) {
    bool ok = key[0] >= 0 && key[0] <= 1 && key[8] >= 0 && key[8] < 64;
    auto field = [&](int v, int bits) -> unsigned long long {
        const int off = 1 << (bits - 1);
        ok = ok && v >= -off && v < off;
        return (unsigned long long)(unsigned)(v + off) & ((1ull << bits) - 1ull);
    };
    lo = (unsigned long long)key[0] | ((unsigned long long)(key[8] & 63) << 1);
    for (int j = 0; j < 4; ++j) lo |= field(key[1 + j], 11) << (7 + 11 * j);
    lo |= field(key[5], 12) << 51;
    hi = field(key[6], 12) | (field(key[7], 12) << 12);
    for (int j = 0; j < 3; ++j) hi |= field(key[9 + j], 12) << (24 + 12 * j);
    if (!ok) hi |= 1ull << 63;
}

template <int TS, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) gen_pool_kernel(WeftPoolTables tb, WeftPoolJob job, int si) {
    constexpr int N = TS * TS;
    constexpr int NW = NT / 32;
    constexpr int WPS = N / 32;             // side-bit words per split row
    constexpr int CH = TS <= 16 ? 3 : 1;    // channels summed by one thread
    constexpr int G = 3 / CH;
    constexpr int LOG_TS = TS == 8 ? 3 : TS == 16 ? 4 : TS == 32 ? 5 : 6;
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
    static_assert(N % 32 == 0 && NT % 32 == 0, "whole words and warps");
    __shared__ Scratch S;

    const int t = job.tiles[si][blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool want0 = job.kinds_mask & 1, want1 = job.kinds_mask & 2;

    // 1. pixels and luminance 0.2126 r + 0.7152 g + 0.0722 b (float32, left to right)
    if (tid <= NB) S.edges[tid] = tb.bin_edges[tid];
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
            if (md >= S.edges[i] && md < S.edges[i + 1]) {
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
    if (tid == 0) S.n_peaks = 0;
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
        if (N <= 128) {  // every bin is one leaf
            if (tid < NB) S.hist[tid] = pairwise_sum(skey + S.bin_start[tid], S.bin_start[tid + 1] - S.bin_start[tid]);
        } else {  // a warp per bin; its leaf list in the Sobel-magnitude plane (free until step 4)
            constexpr int CAP = N / 64;  // leaves of numpy's tree for n <= N
            int* lw = reinterpret_cast<int*>(mags) + warp * 3 * CAP;
            static_assert(NW * 3 * CAP <= N, "leaf lists fit the plane");
            for (int b = warp; b < NB; b += NW) {
                const float h = warp_pairwise_sum(skey + S.bin_start[b], S.bin_start[b + 1] - S.bin_start[b], lw, CAP,
                                                  lane);
                if (lane == 0) S.hist[b] = h;
            }
        }
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
        S.n_split = want1 ? S.n_peaks + tb.n_spec : 0;
    }
    __syncthreads();
    // membership of the three percentile regions, one bit per pixel
    for (int base = warp * 32; base < N; base += NT) {
        const int p = base + lane;
        const float l = lum[p], g = magt[p];
        const unsigned gt = __ballot_sync(0xffffffffu, l > S.p75);
        const unsigned lt = __ballot_sync(0xffffffffu, l < S.p25);
        const unsigned ge = __ballot_sync(0xffffffffu, g >= S.pm75);
        if (lane == 0) {
            S.tmask[0][base >> 5] = gt;
            S.tmask[1][base >> 5] = lt;
            S.tmask[2][base >> 5] = ge;
        }
    }
    __syncthreads();

    // 5. every mean's sum, as numpy takes it: a sequential float32 sum per channel in the
    //    reference's pixel order.  One thread per split line (both sides: the side test read from
    //    the side-bit table) or fixed region, over CH channels; split lines are the dominant
    //    orientations' centre lines, then the template lines.  Jobs come in three groups, each
    //    starting on a warp boundary so a warp runs one loop shape: split lines; whole-tile
    //    scans (the three percentile regions and the tile); index runs (palette runs of the
    //    luminance order, quadrants, 4x4 blocks).  Adding +0.0f for a pixel outside a region
    //    leaves a sum that starts at +0.0f unchanged (round to nearest never makes it -0.0f), so
    //    the scans run without per-pixel branches.
    {
        const int nsplit = S.n_split;
        constexpr int NSCAN = 4, NRUN = NFIX - NSCAN;
        const int la = (nsplit * G + 31) & ~31, lb = (NSCAN * G + 31) & ~31, lc = (NRUN * G + 31) & ~31;
        const uint32_t* sbits = tb.side_bits + side_words_before<TS>() * NSPL;
        for (int slot = tid; slot < la + lb + lc; slot += NT) {
            const int grp = slot < la ? 0 : slot < la + lb ? 1 : 2;
            const int j = slot - (grp == 0 ? 0 : grp == 1 ? la : la + lb);
            const int nj = grp == 0 ? nsplit : grp == 1 ? NSCAN : NRUN;
            if (j >= nj * G) continue;  // padding up to the warp boundary
            const int cg = j / nj, u = j - cg * nj, c0 = cg * CH;  // channel-major with one channel per thread
            float sa[CH], sb[CH];
#pragma unroll
            for (int c = 0; c < CH; ++c) sa[c] = sb[c] = 0.0f;
            if (grp == 0) {
                const int row = u < S.n_peaks ? S.peaks[u] : 16 + (u - S.n_peaks);
                const uint32_t* m = sbits + row * WPS;
                int ca = 0;
                uint32_t next = __ldg(m);
                for (int w = 0; w < WPS; ++w) {
                    const uint32_t word = next;
                    if (w + 1 < WPS) next = __ldg(m + w + 1);
                    ca += __popc(word);
#pragma unroll 8
                    for (int b = 0; b < 32; ++b) {
                        const int p = w * 32 + b;
                        const bool in_a = (word >> b) & 1u;
#pragma unroll
                        for (int c = 0; c < CH; ++c) {
                            const float v = col[(c0 + c) * N + p];
                            sa[c] = __fadd_rn(sa[c], in_a ? v : 0.0f);
                            sb[c] = __fadd_rn(sb[c], in_a ? 0.0f : v);
                        }
                    }
                }
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    S.smean[u][0][c0 + c] = ca > 0 ? __fdiv_rn(sa[c], (float)ca) : 0.0f;
                    S.smean[u][1][c0 + c] = ca < N ? __fdiv_rn(sb[c], (float)(N - ca)) : 0.0f;
                }
                if (c0 == 0) S.scnt[u] = ca;
            } else if (grp == 1) {  // above the 75th / below the 25th luminance percentile, gradient
                                    // at or above its 75th, the whole tile: raster order
                const int r = u < 3 ? 30 + u : 0;
                int cnt = 0;
                for (int w = 0; w < WPS; ++w) {
                    const uint32_t word = r == 0 ? 0xffffffffu : S.tmask[r - 30][w];
                    cnt += __popc(word);
#pragma unroll 8
                    for (int b = 0; b < 32; ++b) {
                        const bool in = (word >> b) & 1u;
#pragma unroll
                        for (int c = 0; c < CH; ++c) {
                            const float v = col[(c0 + c) * N + w * 32 + b];
                            sa[c] = __fadd_rn(sa[c], in ? v : 0.0f);
                        }
                    }
                }
#pragma unroll
                for (int c = 0; c < CH; ++c) S.rmean[r][c0 + c] = cnt > 0 ? __fdiv_rn(sa[c], (float)cnt) : 0.0f;
                if (c0 == 0) S.rcnt[r] = cnt;
            } else {  // palette run [a, b) of the luminance order, or a quadrant / 4x4 block row by row
                const int r = u < 9 ? 21 + u : u - 8;
                const bool run = r >= 21;
                int a = 0, len, y0 = 0, x0 = 0, lg = 0;
                if (run) {
                    int b;
                    run_bounds(tb.cuts, si, r, a, b);
                    len = b > a ? b - a : 0;
                } else {
                    lg = r <= 4 ? LOG_TS - 1 : LOG_TS - 2;  // side TS/2 or TS/4
                    const int q = r <= 4 ? r - 1 : r - 5, per = r <= 4 ? 2 : 4;
                    y0 = (q / per) << lg;
                    x0 = (q % per) << lg;
                    len = 1 << (2 * lg);
                }
                const int msk = (1 << lg) - 1;
#pragma unroll 4
                for (int k = 0; k < len; ++k) {
                    const int ps = sidx[a + k];  // in range for a rect too (a = 0, len <= N / 4)
                    const int p = run ? ps : (y0 + (k >> lg)) * TS + x0 + (k & msk);
#pragma unroll
                    for (int c = 0; c < CH; ++c) sa[c] = __fadd_rn(sa[c], col[(c0 + c) * N + p]);
                }
#pragma unroll
                for (int c = 0; c < CH; ++c) S.rmean[r][c0 + c] = len > 0 ? __fdiv_rn(sa[c], (float)len) : 0.0f;
                if (c0 == 0) S.rcnt[r] = len;
            }
        }
    }
    __syncthreads();

    // 6. palettes: the 13 colours (tile mean, then regions 21..32 in order), their pairwise
    //    near tests in parallel, then one thread keeps each colour that is not near one kept
    //    before it; then the candidate list's segment sizes: the list is (edge pool) palette x 4
    //    alphas, quadrants x 2, orientations x 5, (template pool) palette x 4, quadrants x 2,
    //    blocks, splits x 3 or x 1, so candidate i is a function of i that any thread can
    //    evaluate (cand_at below)
    if (tid < NCOL) {
        float m[3];
        const int r = 20 + tid;
        int a = 0, b = 1;
        if (tid >= 1 && r < 30) run_bounds(tb.cuts, si, r, a, b);
        if (tid >= 1 && r < 30 && b <= a) {
            const int p = sidx[min(a, N - 1)];
            for (int c = 0; c < 3; ++c) m[c] = col[c * N + p];
        } else if (tid >= 1 && S.rcnt[r] > 0) {
            for (int c = 0; c < 3; ++c) m[c] = S.rmean[r][c];
        } else {
            for (int c = 0; c < 3; ++c) m[c] = S.rmean[0][c];
        }
        for (int c = 0; c < 3; ++c) S.cpal[tid][c] = clamp01(m[c]);
    }
    __syncthreads();
    if (tid < NCOL) {
        unsigned near = 0;
        for (int a = 0; a < tid; ++a)
            if (near_pair(S.cpal[tid], S.cpal[a])) near |= 1u << a;
        S.near_mask[tid] = near;
    }
    __syncthreads();
    if (tid == 0) {
        unsigned kept = 1u;
        int npal = 1;
        for (int c = 0; c < 3; ++c) S.pal[0][c] = S.cpal[0][c];
        for (int i = 1; i < NCOL; ++i) {
            if (i == 10) S.npal_e = npal;  // the template palette adds bright / dark / edge colours
            if (!(S.near_mask[i] & kept) && npal < MAXPAL) {
                kept |= 1u << i;
                for (int c = 0; c < 3; ++c) S.pal[npal][c] = S.cpal[i][c];
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
    for (int i = tid; i < HT; i += NT) {
        S.ht_hash[i] = 0ull;
        S.ht_idx[i] = 0x7fffffff;
    }
    __syncthreads();

    // candidate i: kind, float64 geometry (the reference's Python values), colours, alpha
    auto cand_at = [&](int i, int& kind, double (&g)[4], float (&c0)[3], float (&c1)[3], double& alpha) {
        auto a4 = [](int q) { return q == 0 ? 1.0 : q == 1 ? 0.7 : q == 2 ? 0.4 : 0.2; };
        kind = 0;
        for (int k = 0; k < 4; ++k) g[k] = 0.0;
        for (int c = 0; c < 3; ++c) c1[c] = 0.0f;
        int k = 0;
        while (k < 6 && i >= S.seg[k + 1]) ++k;
        const int j = i - S.seg[k];
        switch (k) {
            case 0:
            case 3:  // palette colour x alphas 1, .7, .4, .2
                for (int c = 0; c < 3; ++c) c0[c] = S.pal[j >> 2][c];
                alpha = a4(j & 3);
                break;
            case 1:
            case 4: {  // quadrant mean x alphas .5, .3
                const int r = 1 + (j >> 1);
                for (int c = 0; c < 3; ++c) c0[c] = clamp01(S.rmean[r][c]);
                alpha = (j & 1) ? 0.3 : 0.5;
                break;
            }
            case 2: {  // orientation split: centre x 1, .7, .4, offsets at 0.25 and 0.75 x .5
                const int pk = j / 5, m = j - pk * 5;
                const int na = S.scnt[pk], nb = N - na;
                for (int c = 0; c < 3; ++c) {
                    const float avg = clamp01(S.rmean[0][c]);
                    c0[c] = na > 0 ? clamp01(S.smean[pk][0][c]) : avg;
                    c1[c] = nb > 0 ? clamp01(S.smean[pk][1][c]) : avg;
                }
                const double* gg = tb.orient_geom + ((size_t)(si * 16 + S.peaks[pk]) * 3 + (m < 3 ? 0 : m - 2)) * 4;
                for (int q = 0; q < 4; ++q) g[q] = gg[q];
                alpha = m < 3 ? a4(m) : 0.5;
                kind = 1;
                break;
            }
            case 5:  // 4x4 block mean x .25
                for (int c = 0; c < 3; ++c) c0[c] = clamp01(S.rmean[5 + j][c]);
                alpha = 0.25;
                break;
            default: {  // template split: batched side means, not clamped; an empty side takes the
                        // (unclamped) tile mean
                const int sp = j < tb.n_centre * 3 ? j / 3 : tb.n_centre + (j - tb.n_centre * 3);
                alpha = j < tb.n_centre * 3 ? a4(j % 3) : 0.5;
                const int u = S.n_peaks + sp;
                const int na = S.scnt[u], nb = N - na;
                for (int c = 0; c < 3; ++c) {
                    const float fb = S.rmean[0][c];
                    c0[c] = na > 0 ? S.smean[u][0][c] : fb;
                    c1[c] = nb > 0 ? S.smean[u][1][c] : fb;
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
    auto same_key = [&](int i, int j) {
        const bool pi = !(S.khi[i] >> 63), pj = !(S.khi[j] >> 63);
        if (pi && pj) return S.klo[i] == S.klo[j] && S.khi[i] == S.khi[j];
        if (pi != pj) return false;  // a field in range against one out of range
        int a[KEYS], b[KEYS];
        key_of(i, a);
        key_of(j, b);
        bool same = true;
        for (int k = 0; k < KEYS; ++k) same = same && a[k] == b[k];
        return same;
    };

    // 7. first occurrences kept: every candidate's key, its 64-bit hash entered in a shared
    //    hash table that keeps the lowest candidate index per hash; a candidate is a repeat when
    //    that index is lower than its own and the keys agree (on a bare hash match, every earlier
    //    candidate of the hash is compared)
    const int nc = S.n_cand;
    for (int i = tid; i < nc; i += NT) {
        int key[KEYS];
        key_of(i, key);
        unsigned long long h = 0x9e3779b97f4a7c15ull;
        for (int k = 0; k < KEYS; ++k) {
            h = (h ^ (unsigned long long)(unsigned)key[k]) * 0xff51afd7ed558ccdull;
            h ^= h >> 33;
        }
        h |= h == 0ull;  // 0 marks an empty slot
        S.hash[i] = h;
        pack_key(key, S.klo[i], S.khi[i]);
        int s = (int)(h & (HT - 1));
        for (int probe = 0; probe < HT; ++probe) {  // the table holds at most MAXC < HT hashes
            const unsigned long long prev = atomicCAS(&S.ht_hash[s], 0ull, h);
            if (prev == 0ull || prev == h) {
                atomicMin(&S.ht_idx[s], i);
                break;
            }
            s = (s + 1) & (HT - 1);
        }
    }
    __syncthreads();
    for (int base = 0; base < nc; base += NT) {  // every lane of a warp reaches the ballot
        const int i = base + tid;
        bool keep = false;
        if (i < nc) {
            const unsigned long long h = S.hash[i];
            int s = (int)(h & (HT - 1));
            for (int probe = 0; probe < HT && S.ht_hash[s] != h; ++probe) s = (s + 1) & (HT - 1);
            const int j = S.ht_idx[s];
            keep = true;
            if (j < i) {
                if (same_key(i, j)) {
                    keep = false;
                } else {
                    for (int j2 = 0; j2 < i; ++j2)
                        if (S.hash[j2] == h && same_key(i, j2)) {
                            keep = false;
                            break;
                        }
                }
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (lane == 0 && base + warp * 32 < nc) S.keepw[(base + warp * 32) >> 5] = bal;
    }
    __syncthreads();
    if (tid == 0) {
        int n = 0;
        for (int w = 0; w < (nc + 31) / 32; ++w) {
            S.keep_pre[w] = n;
            n += __popc(S.keepw[w]);
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
        const unsigned w = S.keepw[i >> 5];
        if (!((w >> (i & 31)) & 1u)) continue;
        const int pos = S.keep_pre[i >> 5] + __popc(w & ((1u << (i & 31)) - 1u));
        if (pos >= S.n_out) continue;
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

// the side test of every split row over every tile side's pixel grid, one thread per word
__global__ void side_bits_kernel(WeftPoolTables tb, uint32_t* out) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= WEFTK_POOL_SIDE_WORDS) return;
    int si = 0;
    while (si < 3 && gid >= (si == 0 ? 2 : si == 1 ? 10 : 42) * NSPL) ++si;
    const int before = si == 0 ? 0 : si == 1 ? 2 : si == 2 ? 10 : 42;
    const int ts = 8 << si, wps = ts * ts / 32;
    const int local = gid - before * NSPL, row = local / wps, w = local - row * wps;
    const float* m = row < 16 ? tb.orient_mask + (si * 16 + row) * 4
                     : row - 16 < tb.n_spec ? tb.spec_mask + (si * WEFTK_POOL_MAX_SPECS + (row - 16)) * 4
                                            : nullptr;
    uint32_t word = 0;
    if (m) {
        const float4 c = make_float4(m[0], m[1], m[2], m[3]);
        for (int b = 0; b < 32; ++b) {
            const int p = w * 32 + b;
            if (side_a(c, p % ts, p / ts)) word |= 1u << b;
        }
    }
    out[gid] = word;
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
    gen_pool_kernel<TS, NT><<<n, NT, dyn, stream>>>(tb, job, si);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}

}  // namespace
}  // namespace weftk

using namespace weftk;

// Side streams of the current device that run the larger tile classes beside the 8-px class
// (forked from and joined back into the caller's stream with events, so a captured graph gets
// parallel branches).  Created on a host thread's first call on a device and kept for the life of
// the process; per host thread, so concurrent callers never share the events.
struct SideStreams {
    cudaStream_t s[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[3] = {nullptr, nullptr, nullptr};
};

int side_streams(SideStreams** out) {
    thread_local SideStreams per_dev[64];
    int dev = 0;
    WEFTK_CUDA(cudaGetDevice(&dev));
    WEFTK_REQUIRE(dev >= 0 && dev < 64, "gen_pools: device index beyond 63");
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

extern "C" int weftk_pool_side_bits(const WeftPoolTables* tables, uint32_t* d_bits, void* stream) {
    WEFTK_REQUIRE(tables && d_bits, "pool_side_bits: null argument");
    WEFTK_REQUIRE(tables->n_spec >= 0 && tables->n_spec <= WEFTK_POOL_MAX_SPECS, "pool_side_bits: bad template table");
    WEFTK_REQUIRE(tables->orient_mask && (tables->n_spec == 0 || tables->spec_mask), "pool_side_bits: null table");
    constexpr int block = 256;
    side_bits_kernel<<<(WEFTK_POOL_SIDE_WORDS + block - 1) / block, block, 0, (cudaStream_t)stream>>>(*tables, d_bits);
    WEFTK_CUDA(cudaGetLastError());
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
                      tables->side_bits && (tables->n_spec == 0 || (tables->spec_geom && tables->spec_mask)),
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
