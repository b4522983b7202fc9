// weftk_reseed.cu — device re-seeding of stalled tiles with residual-targeted candidates.
//
// Follows the reference's _generate_residual_candidates (src/weft/encoder.py:1255-1366):
// with err = src - clip(composite) and e = mean_channel |err|, pixels with e at or above
// the 60th percentile of e (numpy's linear interpolation) form the high-error set H;
// the candidates are constant patches in H's mean colours, two-colour linear patches
// split along the mean gradient of e, lines through H's centroid, a quadratic curve
// through H's leftmost, median-by-x and rightmost points, and triangles over H's
// extent — the same kinds, parameters and order as the reference, de-duplicated
// with the reference's coarse key.
//
// One 256-thread CTA per tile.  The percentile comes from a bitonic sort of e in
// shared memory; means are accumulated in float64 and rounded to float32 (numpy
// accumulates these means in float32, so values agree to rounding).  Ties in the
// x-ordering of H are broken by raster order (numpy's default sort leaves that to
// the platform's sort implementation).
#include <cuda_runtime.h>

#include <mutex>
#include <set>

#include <climits>

#include "../../include/weftk_fit.h"
#include "weftk_common.cuh"
#include "weftk_prim.cuh"

namespace weftk {

extern __device__ int g_device_status;

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_MAX_CANDS = 128;
constexpr int KEY_LEN = 16;
constexpr int NV = 36;  // reduced values of the main pass

struct RsShared {
    double red[RS_WARPS][NV];
    double res[NV];
    int colcnt[64], colminy[64], colmaxy[64], rowcnt[64], rowminx[64];
    WeftPrim cand[RS_MAX_CANDS];
    int key[RS_MAX_CANDS][KEY_LEN];
    int keep[RS_MAX_CANDS];
    int n_cand;
    float thresh;
    double lines[4][4];  // x0 y0 x1 y1 of the four linear patches (float64, as the reference computes them)
    float lf[4][4];      // X0 Y0 DY DX rounded to float32 for the side test
};

// Sum NV per-thread values over the CTA (fixed order); result in s.res.
__device__ void block_sum(double (&v)[NV], RsShared& s) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
        if (lane == 0) s.red[warp][k] = x;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double x = 0.0;
        for (int w = 0; w < RS_WARPS; ++w) x += s.red[w][threadIdx.x];
        s.res[threadIdx.x] = x;
    }
    __syncthreads();
}

__device__ __forceinline__ int qkey(double v, double scale) { return (int)(v * scale + 0.5); }

__device__ __forceinline__ float clip01d(double v) { return (float)fmin(1.0, fmax(0.0, v)); }

// Append one candidate with its dedup key (thread 0 only).
__device__ void add_cand(RsShared& s, int kind, const double* g, int ng, const float* c0, const float* c1,
                         double alpha) {
    const int i = s.n_cand;
    if (i >= RS_MAX_CANDS) return;
    WeftPrim& p = s.cand[i];
    p.kind = kind;
    for (int k = 0; k < 7; ++k) p.geom[k] = k < ng ? (float)g[k] : 0.0f;
    for (int k = 0; k < 3; ++k) {
        p.color0[k] = c0[k];
        p.color1[k] = c1 ? c1[k] : 0.0f;
    }
    p.alpha = (float)alpha;
    int* key = s.key[i];
    int n = 0;
    key[n++] = kind;
    for (int k = 0; k < ng; ++k) key[n++] = qkey(g[k], 4.0);
    for (int k = 0; k < 3; ++k) key[n++] = qkey((double)c0[k], 64.0);
    key[n++] = qkey(alpha, 32.0);
    if (c1)
        for (int k = 0; k < 3; ++k) key[n++] = qkey((double)c1[k], 64.0);
    while (n < KEY_LEN) key[n++] = INT_MIN;
    s.n_cand = i + 1;
}

__global__ void __launch_bounds__(RS_THREADS) fit_reseed_kernel(WeftFitState st, const int* gate) {
    extern __shared__ float dyn[];
    __shared__ RsShared s;
    const int t = blockIdx.x;
    if (t >= st.n_tiles) return;
    if (gate != nullptr && *gate == 0) return;  // device-driven fit: no stall this round
    if (!(st.flags[t] & WEFTK_TILE_COMPLEX) || st.n_sel[t] >= st.cap[t]) return;
    const int ts = st.size[t], n = ts * ts, tid = threadIdx.x;
    const double wf = ts - 1, hf = ts - 1;
    const float4* src = reinterpret_cast<const float4*>(st.src) + st.px_off[t];
    const float4* bg = reinterpret_cast<const float4*>(st.bg) + st.px_off[t];
    float* el = dyn;
    float* srt = dyn + n;

    for (int p = tid; p < n; p += RS_THREADS) {
        const float4 a = src[p], g = bg[p];
        const float e = __fdiv_rn(__fadd_rn(__fadd_rn(fabsf(a.x - clamp01(g.x)), fabsf(a.y - clamp01(g.y))),
                                            fabsf(a.z - clamp01(g.z))), 3.0f);
        el[p] = e;
        srt[p] = e;
    }
    if (tid < 64) {
        s.colcnt[tid] = 0;
        s.rowcnt[tid] = 0;
        s.colminy[tid] = INT_MAX;
        s.colmaxy[tid] = -1;
        s.rowminx[tid] = INT_MAX;
    }
    __syncthreads();
    // bitonic sort (n is a power of two)
    for (int k = 2; k <= n; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < n; i += RS_THREADS) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const float a = srt[i], b = srt[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        srt[i] = b;
                        srt[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (tid == 0) {
        // numpy percentile of a float32 array, linear method, all in float32:
        // q = 60/100, virtual index (n-1)*q, lerp from the far end when gamma >= 0.5
        const float q = __fdiv_rn(60.0f, 100.0f);
        const float vi = __fmul_rn((float)(n - 1), q);
        const int lo = (int)floorf(vi), hi = min(lo + 1, n - 1);
        const float g = __fsub_rn(vi, (float)lo), a = srt[lo], b = srt[hi], d = __fsub_rn(b, a);
        s.thresh = (g >= 0.5f) ? __fsub_rn(b, __fmul_rn(d, __fsub_rn(1.0f, g))) : __fadd_rn(a, __fmul_rn(d, g));
    }
    __syncthreads();
    const float thr = s.thresh;
    const int qh = ts / 2;

    // main pass: counts and sums over H, quadrants, the gradient of e, the tile mean
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = 0.0;
    for (int p = tid; p < n; p += RS_THREADS) {
        const int x = p % ts, y = p / ts;
        const float4 a = src[p], g4 = bg[p];
        const float pr[3] = {clamp01(g4.x), clamp01(g4.y), clamp01(g4.z)};
        const float sv[3] = {a.x, a.y, a.z};
        v[33] += sv[0];
        v[34] += sv[1];
        v[35] += sv[2];
        // np.gradient: central differences inside, one-sided at the borders
        const float* row = el + y * ts;
        const float gx = (x == 0) ? __fsub_rn(row[1], row[0])
                         : (x == ts - 1) ? __fsub_rn(row[ts - 1], row[ts - 2])
                                         : __fdiv_rn(__fsub_rn(row[x + 1], row[x - 1]), 2.0f);
        const float gy = (y == 0) ? __fsub_rn(el[ts + x], el[x])
                         : (y == ts - 1) ? __fsub_rn(el[(ts - 1) * ts + x], el[(ts - 2) * ts + x])
                                         : __fdiv_rn(__fsub_rn(el[(y + 1) * ts + x], el[(y - 1) * ts + x]), 2.0f);
        v[31] += gx;
        v[32] += gy;
        if (el[p] >= thr) {
            v[0] += 1.0;
            for (int c = 0; c < 3; ++c) {
                v[1 + c] += sv[c];
                v[4 + c] += pr[c];
                v[7 + c] += __fsub_rn(sv[c], pr[c]);
            }
            v[10] += x;
            v[11] += y;
            const int q = (y >= qh ? 2 : 0) + (x >= qh ? 1 : 0);
            v[12 + q] += 1.0;
            for (int c = 0; c < 3; ++c) v[16 + 3 * q + c] += sv[c];
            atomicAdd(&s.colcnt[x], 1);
            atomicMin(&s.colminy[x], y);
            atomicMax(&s.colmaxy[x], y);
            atomicAdd(&s.rowcnt[y], 1);
            atomicMin(&s.rowminx[y], x);
        }
    }
    block_sum(v, s);
    const double m = s.res[0];
    if (m == 0.0) return;  // uniform across the CTA

    // direction of the mean error gradient, and the four linear-patch lines
    if (tid == 0) {
        const double mx = (double)(float)(s.res[31] / (double)n), my = (double)(float)(s.res[32] / (double)n);
        const double nrm = sqrt(mx * mx + my * my) + 1e-8;
        const double vx = mx / nrm, vy = my / nrm;
        const double offs[3] = {0.5, 0.3, 0.7};
        for (int L = 0; L < 3; ++L) {
            const double cx = wf * offs[L], cy = hf * offs[L];
            s.lines[L][0] = cx - vx * wf * 0.6;
            s.lines[L][1] = cy - vy * hf * 0.6;
            s.lines[L][2] = cx + vx * wf * 0.6;
            s.lines[L][3] = cy + vy * hf * 0.6;
        }
        const double cx = wf * 0.5, cy = hf * 0.5;
        s.lines[3][0] = cx + vy * wf * 0.6;
        s.lines[3][1] = cy - vx * hf * 0.6;
        s.lines[3][2] = cx - vy * wf * 0.6;
        s.lines[3][3] = cy + vx * hf * 0.6;
        for (int L = 0; L < 4; ++L) {
            s.lf[L][0] = (float)s.lines[L][0];
            s.lf[L][1] = (float)s.lines[L][1];
            s.lf[L][2] = (float)(s.lines[L][3] - s.lines[L][1]);
            s.lf[L][3] = (float)(s.lines[L][2] - s.lines[L][0]);
        }
    }
    __syncthreads();
    // side means for the four lines (integer pixel coordinates, float32 side test)
    double w2[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) w2[k] = 0.0;
    for (int p = tid; p < n; p += RS_THREADS) {
        const float xf = (float)(p % ts), yf = (float)(p / ts);
        const float4 a = src[p];
#pragma unroll
        for (int L = 0; L < 4; ++L) {
            const float side = __fsub_rn(__fmul_rn(__fsub_rn(xf, s.lf[L][0]), s.lf[L][2]),
                                         __fmul_rn(__fsub_rn(yf, s.lf[L][1]), s.lf[L][3]));
            const int o = L * 8 + (side >= 0.0f ? 0 : 4);
            w2[o] += 1.0;
            w2[o + 1] += a.x;
            w2[o + 2] += a.y;
            w2[o + 3] += a.z;
        }
    }
    const double tile_mean[3] = {s.res[33] / n, s.res[34] / n, s.res[35] / n};
    double hs[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) hs[k] = s.res[k];
    __syncthreads();
    block_sum(w2, s);

    if (tid == 0) {
        s.n_cand = 0;
        float hi_col[3], corr[3];
        for (int c = 0; c < 3; ++c) {
            hi_col[c] = clip01d((double)(float)(hs[1 + c] / m));
            const float pm = (float)(hs[4 + c] / m), em = (float)(hs[7 + c] / m);
            corr[c] = clip01d((double)__fadd_rn(pm, em));
        }
        const double a_const[5] = {0.6, 0.4, 0.25, 0.15, 0.08};
        const float* cols3[3] = {hi_col, corr, hi_col};
        for (int k = 0; k < 3; ++k)
            for (int j = 0; j < 5; ++j) add_cand(s, 0, nullptr, 0, cols3[k], nullptr, a_const[j]);
        const double a_q[3] = {0.35, 0.2, 0.1};
        for (int q = 0; q < 4; ++q) {
            const double cnt = hs[12 + q];
            if (cnt > 0.0) {
                float qc[3];
                for (int c = 0; c < 3; ++c) qc[c] = clip01d((double)(float)(hs[16 + 3 * q + c] / cnt));
                for (int j = 0; j < 3; ++j) add_cand(s, 0, nullptr, 0, qc, nullptr, a_q[j]);
            }
        }
        const double a_lin[4][3] = {{0.5, 0.3, 0.15}, {0.5, 0.3, 0.15}, {0.5, 0.3, 0.15}, {0.4, 0.2, 0.0}};
        for (int L = 0; L < 4; ++L) {
            float c0[3], c1[3];
            const double ca = s.res[L * 8], cb = s.res[L * 8 + 4];
            for (int c = 0; c < 3; ++c) {
                c0[c] = ca > 0 ? (float)(s.res[L * 8 + 1 + c] / ca) : (float)tile_mean[c];
                c1[c] = cb > 0 ? (float)(s.res[L * 8 + 5 + c] / cb) : (float)tile_mean[c];
            }
            for (int j = 0; j < (L < 3 ? 3 : 2); ++j) add_cand(s, 1, s.lines[L], 4, c0, c1, a_lin[L][j]);
        }
        const double ecx = hs[10] / m, ecy = hs[11] / m;
        const double thick[5] = {0.3, 0.6, 1.0, 1.5, 2.5}, a_line[3] = {0.5, 0.3, 0.15};
        for (int i = 0; i < 5; ++i)
            for (int rep = 0; rep < 2; ++rep)
                for (int j = 0; j < 3; ++j) {
                    const double gv[5] = {ecx, 0.0, ecx, hf, thick[i]};
                    const double gh[5] = {0.0, ecy, wf, ecy, thick[i]};
                    add_cand(s, 2, gv, 5, hi_col, nullptr, a_line[j]);
                    add_cand(s, 2, gh, 5, hi_col, nullptr, a_line[j]);
                }
        for (int i = 0; i < 2; ++i) {
            const double t2 = i == 0 ? 0.5 : 1.0;
            const double d1[5] = {0.0, 0.0, wf, hf, t2}, d2[5] = {0.0, hf, wf, 0.0, t2};
            add_cand(s, 2, d1, 5, hi_col, nullptr, 0.25);
            add_cand(s, 2, d2, 5, hi_col, nullptr, 0.25);
        }
        int minx = -1, maxx = -1, miny = -1, maxy = -1;
        for (int x = 0; x < ts; ++x)
            if (s.colcnt[x]) {
                if (minx < 0) minx = x;
                maxx = x;
            }
        for (int y = 0; y < ts; ++y)
            if (s.rowcnt[y]) {
                if (miny < 0) miny = y;
                maxy = y;
            }
        const int mi = (int)m;
        if (mi >= 6) {
            // stable order by x (raster order within a column): first, middle, last
            const int r = mi / 2;
            int before = 0, X = minx;
            for (int x = 0; x < ts; ++x) {
                if (before + s.colcnt[x] > r) {
                    X = x;
                    break;
                }
                before += s.colcnt[x];
            }
            int Y = 0, seen = 0;
            for (int y = 0; y < ts; ++y) {
                if (el[y * ts + X] >= thr) {
                    if (seen == r - before) {
                        Y = y;
                        break;
                    }
                    ++seen;
                }
            }
            const double p0x = minx, p0y = s.colminy[minx], p1x = maxx, p1y = s.colmaxy[maxx];
            const double cx = fmax(0.0, fmin(wf, 2.0 * X - (p0x + p1x) / 2.0));
            const double cy = fmax(0.0, fmin(hf, 2.0 * Y - (p0y + p1y) / 2.0));
            const double tk[3] = {0.5, 1.0, 2.0};
            for (int j = 0; j < 3; ++j) {
                const double gc[7] = {p0x, p0y, cx, cy, p1x, p1y, tk[j]};
                add_cand(s, 3, gc, 7, hi_col, nullptr, 0.3);
            }
        }
        if (mi >= 3) {
            const double g1[6] = {(double)minx, (double)s.colminy[minx], (double)maxx, (double)s.colminy[maxx], ecx, ecy};
            const double g2[6] = {(double)minx, (double)miny, (double)maxx, (double)maxy, ecx, ecy};
            const double at[3] = {0.4, 0.2, 0.1};
            for (int gi = 0; gi < 2; ++gi)
                for (int j = 0; j < 3; ++j) {
                    add_cand(s, 4, gi == 0 ? g1 : g2, 6, hi_col, nullptr, at[j]);
                    add_cand(s, 4, gi == 0 ? g1 : g2, 6, hi_col, nullptr, at[j]);
                }
        }
    }
    __syncthreads();
    // keep the first candidate of each key
    const int nc = s.n_cand;
    if (tid < nc) {
        bool dup = false;
        for (int j = 0; j < tid && !dup; ++j) {
            bool same = true;
            for (int k = 0; k < KEY_LEN; ++k)
                if (s.key[j][k] != s.key[tid][k]) {
                    same = false;
                    break;
                }
            dup = same;
        }
        s.keep[tid] = dup ? 0 : 1;
    }
    __syncthreads();
    __shared__ int base_cnt, n_new, ok;
    if (tid == 0) {
        int k = 0;
        for (int i = 0; i < nc; ++i) {
            const int kp = s.keep[i];
            s.keep[i] = kp ? k : -1;
            k += kp;
        }
        n_new = k;
        base_cnt = st.pool_cnt[t];
        ok = base_cnt + k <= st.pool_cap[t];
        if (!ok) atomicCAS(&g_device_status, 0, WEFTK_E_RANGE);
    }
    __syncthreads();
    if (!ok) return;
    const long long off = st.pool_off[t];
    if (tid < nc && s.keep[tid] >= 0) {
        const long long slot = off + base_cnt + s.keep[tid];
        WeftPrim* dst = const_cast<WeftPrim*>(st.cand) + slot;
        *dst = s.cand[tid];
        Prep r = prep_prim(s.cand[tid]);
        float4* pp = reinterpret_cast<float4*>(st.prep) + slot * 4;
        pp[0] = make_float4(__int_as_float(r.kind), r.a, r.cr, r.cg);
        pp[1] = make_float4(r.cb, r.q[0], r.q[1], r.q[2]);
        pp[2] = make_float4(r.q[3], r.q[4], r.q[5], r.q[6]);
        pp[3] = make_float4(r.q[7], r.q[8], r.q[9], r.q[10]);
        st.alive[slot] = 1;
        st.kind[slot] = (uint8_t)s.cand[tid].kind;
    }
    if (tid == 0) {
        st.pool_cnt[t] = base_cnt + n_new;
        st.n_alive[t] += n_new;
    }
}

}  // namespace weftk

using namespace weftk;

int launch_fit_reseed(const WeftFitState& st, const int* gate, cudaStream_t stream) {
    if (st.n_tiles == 0) return WEFTK_OK;
    const int smem = 2 * 64 * 64 * (int)sizeof(float);
    {  // the dynamic shared-memory opt-in is per device: set it once per device, under a lock
        int dev = 0;
        WEFTK_CUDA(cudaGetDevice(&dev));
        static std::mutex mu;
        static std::set<int> done;
        std::lock_guard<std::mutex> lock(mu);
        if (!done.count(dev)) {
            WEFTK_CUDA(cudaFuncSetAttribute(fit_reseed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            done.insert(dev);
        }
    }
    fit_reseed_kernel<<<st.n_tiles, RS_THREADS, smem, stream>>>(st, gate);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}

extern "C" int weftk_fit_reseed(const WeftFitState* st, int quality, void* stream) {
    (void)quality;
    WEFTK_REQUIRE(st && st->bg, "fit_reseed: null state or no composite (bg)");
    return launch_fit_reseed(*st, nullptr, (cudaStream_t)stream);
}
