// weftk_prim.cuh — per-primitive preparation and per-pixel coverage for sm_100a.
//
// The renderer is the reference's CPU renderer (src/weft/render.py:127-234):
// back-to-front "over" compositing c = s*a + c*(1-a) from black, alpha
// clamped to [0,1], pixel-centre samples.  Arithmetic follows the reference's
// numpy dtype rules where a step function depends on it (triangle inside test:
// float64 coefficients rounded to float32, float32 products, IEEE division, no
// FMA contraction) and uses FMAs and reciprocals elsewhere (differences stay
// far below the 1/255 render tolerance).
//
// Work layout: one warp cooperates on one primitive at a time; each lane owns
// PPL pixels.  Everything per primitive that does not depend on the pixel is
// hoisted into a Prep record (64 B).  The quadratic Bezier's 32 polyline points
// are computed one per lane and exchanged with warp shuffles.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/weftk.h"

namespace weftk {

constexpr unsigned FULL = 0xffffffffu;

enum Kind : int { K_CONST = 0, K_LINEAR = 1, K_LINE = 2, K_CURVE = 3, K_TRI = 4, K_BICUBIC = 5, K_SKIP = -1 };

// Per-primitive hoisted terms.  q[] meaning by kind (U = V / (|V|^2 + 1e-8), the
// projection vector, so the clamped segment parameter is t = clamp(D . U)):
//   linear:   X0 Y0 UX UY c1r c1g c1b
//   line:     X0 Y0 VX VY UX UY K         (alpha = exp(K * d^2) * a)
//   curve:    K p0x p0y cx cy p1x p1y
//   triangle: X2 Y2 A B C D DEN 1/DEN     (a = (A dx + B dy)/DEN, b = (C dx + D dy)/DEN)
//   bicubic:  index of the 48-value control grid (as float)
struct __align__(16) Prep {
    int kind;
    float a;
    float cr, cg, cb;
    float q[11];
};
static_assert(sizeof(Prep) == 64, "Prep must be 64 bytes");

// Clamp to [0, 1] (NaN -> 0).  The saturate modifier folds into the producing FADD/FMUL/FFMA,
// so the clamp costs no instruction; same results as fminf(fmaxf(v, 0), 1).
__device__ __forceinline__ float clamp01(float v) { return __saturatef(v); }

// Gaussian falloff coefficient: -f32(1 / (2 sigma^2)), sigma = max(0.5, thickness),
// evaluated in float64 like the reference's Python scalars.
__device__ __forceinline__ float gauss_k(float thick) {
    double s = fmax(0.5, (double)thick);
    return -(float)(1.0 / (2.0 * s * s));
}

__device__ __forceinline__ Prep prep_prim(const WeftPrim& P) {
    Prep r;
    r.kind = P.kind;
    r.a = clamp01(P.alpha);
    r.cr = P.color0[0];
    r.cg = P.color0[1];
    r.cb = P.color0[2];
#pragma unroll
    for (int i = 0; i < 11; ++i) r.q[i] = 0.0f;
    const float* g = P.geom;
    switch (P.kind) {
        case K_CONST:
            break;
        case K_LINEAR:
        case K_LINE: {
            double vx = (double)g[2] - (double)g[0];
            double vy = (double)g[3] - (double)g[1];
            double den = vx * vx + vy * vy + 1e-8;
            r.q[0] = g[0];
            r.q[1] = g[1];
            if (P.kind == K_LINEAR) {
                r.q[2] = (float)(vx / den);
                r.q[3] = (float)(vy / den);
                r.q[4] = P.color1[0];
                r.q[5] = P.color1[1];
                r.q[6] = P.color1[2];
            } else {
                r.q[2] = (float)vx;
                r.q[3] = (float)vy;
                r.q[4] = (float)(vx / den);
                r.q[5] = (float)(vy / den);
                r.q[6] = gauss_k(g[4]);
            }
            break;
        }
        case K_CURVE:
            r.q[0] = gauss_k(g[6]);
#pragma unroll
            for (int i = 0; i < 6; ++i) r.q[1 + i] = g[i];
            break;
        case K_TRI: {
            double x0 = g[0], y0 = g[1], x1 = g[2], y1 = g[3], x2 = g[4], y2 = g[5];
            double den = (y1 - y2) * (x0 - x2) + (x2 - x1) * (y0 - y2);
            if (fabs(den) < 1e-6) {
                r.kind = K_SKIP;  // degenerate: coverage 0 everywhere, blend is the identity
                break;
            }
            r.q[0] = g[4];
            r.q[1] = g[5];
            r.q[2] = (float)(y1 - y2);
            r.q[3] = (float)(x2 - x1);
            r.q[4] = (float)(y2 - y0);
            r.q[5] = (float)(x0 - x2);
            r.q[6] = (float)den;
            r.q[7] = __frcp_rn((float)den);
            break;
        }
        case K_BICUBIC:
            r.q[0] = g[0];
            break;
        default:
            r.kind = K_SKIP;
    }
    return r;
}

// Point i (0..31) of the reference's curve polyline: t = float32(linspace(0,1,32))[i],
// x = u*u*p0 + 2*u*t*c + t*t*p1 evaluated in float32 without contraction
// (src/weft/render.py:98-105).
__device__ __forceinline__ float2 bezier_point(const Prep& P, int i) {
    float t = (i >= 31) ? 1.0f : (float)((double)i * (1.0 / 31.0));
    float u = __fsub_rn(1.0f, t);
    float uu = __fmul_rn(u, u), ut2 = __fmul_rn(__fmul_rn(2.0f, u), t), tt = __fmul_rn(t, t);
    float x = __fadd_rn(__fadd_rn(__fmul_rn(uu, P.q[1]), __fmul_rn(ut2, P.q[3])), __fmul_rn(tt, P.q[5]));
    float y = __fadd_rn(__fadd_rn(__fmul_rn(uu, P.q[2]), __fmul_rn(ut2, P.q[4])), __fmul_rn(tt, P.q[6]));
    return make_float2(x, y);
}

// Segment owned by this lane (lane s: point s -> point s+1); lane 31's is unused.
// (ax, ay) start, (vx, vy) direction, (ux, uy) = v / (|v|^2 + 1e-8).
struct Seg {
    float ax, ay, vx, vy, ux, uy;
};

__device__ __forceinline__ Seg lane_segment(const Prep& P, int lane) {
    float2 p = bezier_point(P, lane);
    float2 n = bezier_point(P, lane + 1 > 31 ? 31 : lane + 1);
    Seg s;
    s.ax = p.x;
    s.ay = p.y;
    s.vx = __fsub_rn(n.x, p.x);
    s.vy = __fsub_rn(n.y, p.y);
    float den = __fadd_rn(__fadd_rn(__fmul_rn(s.vx, s.vx), __fmul_rn(s.vy, s.vy)), 1e-8f);
    s.ux = __fdiv_rn(s.vx, den);
    s.uy = __fdiv_rn(s.vy, den);
    return s;
}

// Squared distance from (px,py) to the segment (ax,ay)+t(vx,vy), t = clamp((p-a).u) in [0,1].
// Every kernel uses this one formula, so cached composites equal full re-renders bit for bit.
__device__ __forceinline__ float seg_d2(float px, float py, float ax, float ay, float vx, float vy, float ux,
                                        float uy) {
    float dx = px - ax, dy = py - ay;
    float t = clamp01(fmaf(dx, ux, dy * uy));
    float ex = fmaf(-t, vx, dx), ey = fmaf(-t, vy, dy);
    return fmaf(ex, ex, ey * ey);
}

// Exact reproduction of the reference's float32 barycentric inside test:
// a = fl(num_a / den), b = fl(num_b / den), c = fl(fl(1 - a) - b), inside iff all >= 0.
// The signs of a and b are the signs of num * (1/den), so they are tested without a
// division; c is first estimated from the reciprocal products and the IEEE divisions
// are only done when the estimate is within its error bound of zero.
__device__ __forceinline__ float tri_inside(const Prep& P, float px, float py) {
    const float dx = __fsub_rn(px, P.q[0]), dy = __fsub_rn(py, P.q[1]);
    const float na = __fadd_rn(__fmul_rn(P.q[2], dx), __fmul_rn(P.q[3], dy));
    const float nb = __fadd_rn(__fmul_rn(P.q[4], dx), __fmul_rn(P.q[5], dy));
    const float ea = __fmul_rn(na, P.q[7]), eb = __fmul_rn(nb, P.q[7]);
    if (ea < 0.0f || eb < 0.0f) return 0.0f;
    const float ec = __fsub_rn(__fsub_rn(1.0f, ea), eb);
    if (fabsf(ec) > 1e-6f * (1.0f + ea + eb)) return ec >= 0.0f ? 1.0f : 0.0f;
    const float a = __fdiv_rn(na, P.q[6]), b = __fdiv_rn(nb, P.q[6]);
    const float c = __fsub_rn(__fsub_rn(1.0f, a), b);
    return (a >= 0.0f && b >= 0.0f && c >= 0.0f) ? 1.0f : 0.0f;
}

// Evaluate source colour and alpha of primitive P at this lane's PPL pixels.
// `valid` masks pixels beyond the tile (still evaluated, results ignored).
// Must be called by all 32 lanes of the warp (curves use shuffles).
template <int PPL>
__device__ __forceinline__ void prim_eval(const Prep& P, const float (&fx)[PPL], const float (&fy)[PPL],
                                          float (&a)[PPL], float (&sr)[PPL], float (&sg)[PPL], float (&sb)[PPL],
                                          int lane) {
#pragma unroll
    for (int j = 0; j < PPL; ++j) {
        sr[j] = P.cr;
        sg[j] = P.cg;
        sb[j] = P.cb;
        a[j] = 0.0f;
    }
    switch (P.kind) {
        case K_CONST:
#pragma unroll
            for (int j = 0; j < PPL; ++j) a[j] = P.a;
            break;
        case K_LINEAR:
#pragma unroll
            for (int j = 0; j < PPL; ++j) {
                float t = clamp01(fmaf(fx[j] - P.q[0], P.q[2], (fy[j] - P.q[1]) * P.q[3]));
                float u = 1.0f - t;
                sr[j] = fmaf(P.q[4], t, P.cr * u);
                sg[j] = fmaf(P.q[5], t, P.cg * u);
                sb[j] = fmaf(P.q[6], t, P.cb * u);
                a[j] = P.a;
            }
            break;
        case K_LINE:
#pragma unroll
            for (int j = 0; j < PPL; ++j) {
                float d2 = seg_d2(fx[j], fy[j], P.q[0], P.q[1], P.q[2], P.q[3], P.q[4], P.q[5]);
                a[j] = expf(d2 * P.q[6]) * P.a;
            }
            break;
        case K_CURVE: {
            Seg s = lane_segment(P, lane);
            float best[PPL];
#pragma unroll
            for (int j = 0; j < PPL; ++j) best[j] = 1e18f;
#pragma unroll 1
            for (int k = 0; k < 31; ++k) {
                float ax = __shfl_sync(FULL, s.ax, k), ay = __shfl_sync(FULL, s.ay, k);
                float vx = __shfl_sync(FULL, s.vx, k), vy = __shfl_sync(FULL, s.vy, k);
                float ux = __shfl_sync(FULL, s.ux, k), uy = __shfl_sync(FULL, s.uy, k);
#pragma unroll
                for (int j = 0; j < PPL; ++j) best[j] = fminf(best[j], seg_d2(fx[j], fy[j], ax, ay, vx, vy, ux, uy));
            }
#pragma unroll
            for (int j = 0; j < PPL; ++j) a[j] = expf(best[j] * P.q[0]) * P.a;
            break;
        }
        case K_TRI:
#pragma unroll
            for (int j = 0; j < PPL; ++j) a[j] = tri_inside(P, fx[j], fy[j]) * P.a;
            break;
        default:
            break;  // skipped primitive: a = 0, blend is the identity
    }
}

// Same as prim_eval for kind K_CURVE, with the warp's 31 segments already in shared
// memory (seg[k] = {ax, ay, vx, vy}, {ux, uy, -, -}); reads are warp-uniform broadcasts.
template <int PPL>
__device__ __forceinline__ void curve_alpha_smem(const Prep& P, const float4 (*seg)[2], const float (&fx)[PPL],
                                                 const float (&fy)[PPL], float (&a)[PPL]) {
    float best[PPL];
#pragma unroll
    for (int j = 0; j < PPL; ++j) best[j] = 1e18f;
#pragma unroll 2
    for (int k = 0; k < 31; ++k) {
        const float4 s0 = seg[k][0];
        const float4 s1 = seg[k][1];
#pragma unroll
        for (int j = 0; j < PPL; ++j)
            best[j] = fminf(best[j], seg_d2(fx[j], fy[j], s0.x, s0.y, s0.z, s0.w, s1.x, s1.y));
    }
#pragma unroll
    for (int j = 0; j < PPL; ++j) a[j] = expf(best[j] * P.q[0]) * P.a;
}

// "over" blend, identical sequence in every kernel so incremental and full renders agree bit for bit.
__device__ __forceinline__ float blend(float s, float a, float c) {
    return __fmaf_rn(s, a, __fmul_rn(c, __fsub_rn(1.0f, a)));
}

// Cubic Bernstein weights at sample i of n (t = linspace(0,1,n)[i]), float64 like the reference basis.
__device__ __forceinline__ void bernstein4(int i, int n, double (&w)[4]) {
    double t = (n > 1) ? (double)i * (1.0 / (double)(n - 1)) : 0.0;
    if (n > 1 && i == n - 1) t = 1.0;
    double u = 1.0 - t;
    w[0] = u * u * u;
    w[1] = 3.0 * u * u * t;
    w[2] = 3.0 * u * t * t;
    w[3] = t * t * t;
}

}  // namespace weftk
