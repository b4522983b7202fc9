// weftk_entropy.cu — chunked order-0 rANS decode (see include/weftk_entropy.h).
#include <cuda_runtime.h>

#include "../../include/weftk_entropy.h"
#include "weftk_common.cuh"

namespace weftk {

extern __device__ int g_device_status;

constexpr int RANS_PROB_BITS = 12;
constexpr int RANS_TOT = 1 << RANS_PROB_BITS;
constexpr unsigned RANS_L = 1u << 23;
constexpr int RD_WARPS = 4;

__device__ __forceinline__ void rans_report() { atomicCAS(&g_device_status, 0, WEFTK_E_ARG); }

__device__ __forceinline__ unsigned rd_u32(const uint8_t* p) {
    return (unsigned)p[0] | ((unsigned)p[1] << 8) | ((unsigned)p[2] << 16) | ((unsigned)p[3] << 24);
}

__device__ __forceinline__ unsigned rd_u16(const uint8_t* p) { return (unsigned)p[0] | ((unsigned)p[1] << 8); }

// One warp per chunk.  Shared memory per warp: the 4096-slot symbol table and the cumulative
// frequencies of the 256 symbols.
__global__ void __launch_bounds__(RD_WARPS * 32) rans_decode_kernel(const uint8_t* __restrict__ payload,
                                                                    long long payload_len,
                                                                    const WeftRansChunk* __restrict__ chunks,
                                                                    int n_chunks, uint8_t* __restrict__ out,
                                                                    long long out_len) {
    __shared__ uint8_t lut_all[RD_WARPS][RANS_TOT];
    __shared__ unsigned short freq_all[RD_WARPS][256];
    __shared__ unsigned short cum_all[RD_WARPS][257];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * RD_WARPS + warp;
    if (c >= n_chunks) return;
    uint8_t* lut = lut_all[warp];
    unsigned short* freq = freq_all[warp];
    unsigned short* cum = cum_all[warp];
    const WeftRansChunk ch = chunks[c];
    if (ch.coded_offset < 0 || ch.coded_length < 5 || ch.coded_offset + ch.coded_length > payload_len ||
        ch.raw_offset < 0 || ch.raw_length < 0 || ch.raw_offset + ch.raw_length > out_len) {
        if (lane == 0) rans_report();
        return;
    }
    const uint8_t* p = payload + ch.coded_offset;
    const long long len = ch.coded_length;
    uint8_t* dst = out + ch.raw_offset;
    const int mode = p[0];
    const long long n = rd_u32(p + 1);
    if (n != ch.raw_length || (mode != 0 && mode != 1)) {
        if (lane == 0) rans_report();
        return;
    }
    if (mode == 0) {  // raw
        if (5 + n != len) {
            if (lane == 0) rans_report();
            return;
        }
        for (long long i = lane; i < n; i += 32) dst[i] = p[5 + i];
        return;
    }
    if (len < 7) {
        if (lane == 0) rans_report();
        return;
    }
    const int n_sym = (int)rd_u16(p + 5);
    const long long hdr = 7 + 3LL * n_sym;
    if (n_sym > 256 || hdr + 8 > len) {
        if (lane == 0) rans_report();
        return;
    }
    for (int i = lane; i < 256; i += 32) freq[i] = 0;
    __syncwarp();
    if (lane == 0)
        for (int k = 0; k < n_sym; ++k) freq[p[7 + 3 * k]] = (unsigned short)rd_u16(p + 8 + 3 * k);
    __syncwarp();
    // cumulative frequencies: lane l sums symbols [8l, 8l + 8), then an exclusive warp scan
    unsigned loc[8], run = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        loc[j] = run;
        run += freq[lane * 8 + j];
    }
    unsigned incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const unsigned base = incl - run;
    const unsigned total = __shfl_sync(0xffffffffu, incl, 31);
    if (total != RANS_TOT) {
        if (lane == 0) rans_report();
        return;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) cum[lane * 8 + j] = (unsigned short)(base + loc[j]);
    if (lane == 0) cum[256] = RANS_TOT;
    __syncwarp();
    // symbol table: each lane fills the slots of its 8 symbols
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int s = lane * 8 + j;
        const int a = cum[s], b = a + freq[s];
        for (int k = a; k < b; ++k) lut[k] = (uint8_t)s;
    }
    __syncwarp();
    if (lane != 0) return;
    unsigned x = rd_u32(p + hdr);
    const long long m = rd_u32(p + hdr + 4);
    if (hdr + 8 + m != len) {
        rans_report();
        return;
    }
    const uint8_t* em = p + hdr + 8;
    long long ptr = m - 1;
    for (long long i = 0; i < n; ++i) {
        const unsigned slot = x & (RANS_TOT - 1);
        const unsigned s = lut[slot];
        dst[i] = (uint8_t)s;
        x = (unsigned)freq[s] * (x >> RANS_PROB_BITS) + (slot - cum[s]);
        while (x < RANS_L && ptr >= 0) {
            x = (x << 8) | em[ptr];
            --ptr;
        }
    }
}

}  // namespace weftk

using namespace weftk;

extern "C" int weftk_rans_decode_chunks(const uint8_t* d_payload, int64_t payload_len, const WeftRansChunk* d_chunks,
                                        int n_chunks, uint8_t* d_out, int64_t out_len, void* stream) {
    WEFTK_REQUIRE(n_chunks >= 0 && payload_len >= 0 && out_len >= 0, "rans_decode_chunks: negative size");
    if (n_chunks == 0) return WEFTK_OK;
    WEFTK_REQUIRE(d_payload && d_chunks && d_out, "rans_decode_chunks: null pointer");
    rans_decode_kernel<<<(n_chunks + RD_WARPS - 1) / RD_WARPS, RD_WARPS * 32, 0, (cudaStream_t)stream>>>(
        d_payload, payload_len, d_chunks, n_chunks, d_out, out_len);
    WEFTK_CUDA(cudaGetLastError());
    return WEFTK_OK;
}
