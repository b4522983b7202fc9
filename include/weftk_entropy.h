/*
 * weftk_entropy.h — chunked order-0 rANS decode of PRIM payloads on the GPU (C ABI of libweftk.so).
 *
 * Replaces the reference decoder's entropy stage for the primitive payload:
 * `decode_prim_payload` (src/weft/prim_chunks.py:80-125) over `decode_bytes` / the rANS
 * decoder (src/weft/entropy.py:121-189, mode byte and header layout :192-217), and its GPU
 * twin (src/weft/gpu_entropy.py:90-211, one thread per chunk).  Each chunk is either raw
 * (mode 0: <u8 0, u32 n, n bytes>) or rANS (mode 1: <u8 1, u32 n, u16 n_sym, n_sym x <u8 sym,
 * u16 freq>, u32 state, u32 emitted, emitted bytes>, 12-bit probabilities, state lower bound
 * 2^23, bytes consumed from the end of the emitted run).  One warp decodes one chunk: the lanes
 * build the 4096-slot symbol table together, then one lane runs the (sequential) state chain.
 * Every read stays inside its chunk's coded bytes and every write inside its raw range; a chunk
 * that does not parse is reported through weftk_device_status (WEFTK_E_ARG) and left unwritten.
 */
#ifndef WEFTK_ENTROPY_H
#define WEFTK_ENTROPY_H

#include "weftk.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One coded chunk: bytes [coded_offset, coded_offset + coded_length) of the payload decode
 * to bytes [raw_offset, raw_offset + raw_length) of the output (a CIDX entry,
 * src/weft/prim_chunks.py:23-77). */
typedef struct WeftRansChunk {
    int64_t coded_offset;
    int64_t coded_length;
    int64_t raw_offset;
    int64_t raw_length;
} WeftRansChunk;

/* Decode n_chunks chunks of d_payload (payload_len bytes) into d_out (out_len bytes). */
int weftk_rans_decode_chunks(const uint8_t* d_payload, int64_t payload_len, const WeftRansChunk* d_chunks,
                             int n_chunks, uint8_t* d_out, int64_t out_len, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WEFTK_ENTROPY_H */
