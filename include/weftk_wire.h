/*
 * weftk_wire.h — snapping fitted primitives to the bitstream's quantisation grid on the
 * device (C ABI of libweftk.so).
 *
 * The reference snaps every selected primitive before it scores the final fit and writes
 * it (_quantize_primitive, src/weft/encoder.py:211-237; the wire format of
 * encode_primitive, src/weft/primitives.py:102-177):
 *   colour channel c -> round(clamp(c, 0, 1) * 255) / 255
 *   alpha a          -> round(clamp(a, 0, 1) * 65535) / 65535
 *   coordinate v     -> round(clamp(v / 15, 0, 1) * 65535) / 65535 * 15
 *   thickness t      -> round(clamp(t / 4, 0, 1) * 65535) / 65535 * 4
 * in float64 with round-half-to-even (Python's round), then stored as float32.
 * Coordinates are geom[0..3] of a linear patch and a line (geom[4] is the line's
 * thickness), geom[0..5] of a curve (geom[6] its thickness) and of a triangle; a constant
 * patch has no geometry; bicubic rows (kind 5) and rows of kind < 0 (no layer) keep their
 * geometry.  Both entry points are device-only launches (no host synchronisation), so
 * they can sit inside a captured CUDA graph.
 */
#ifndef WEFTK_WIRE_H
#define WEFTK_WIRE_H

#include "weftk.h"

#ifdef __cplusplus
extern "C" {
#endif

struct WeftFitState;

/* Parameter rows (float[16] per row, the layout of weftk_refine.h) snapped to the wire
 * grid: d_out[r] = quantised d_params[r] by the kind d_kind[r].  Columns 14..15 are
 * copied.  d_out may equal d_params.  Replaces the per-primitive _quantize_primitive
 * calls (src/weft/encoder.py:211-237) on the selected stacks. */
int weftk_quantize_rows(const float* d_params, const int32_t* d_kind, int n_rows, float* d_out, void* stream);

/* Every tile's selected stack of a fit (weftk_fit.h), snapped to the wire grid:
 * d_rows[(t * cap_max + j) * 16 ..] = quantised parameter row of the j-th selected primitive
 * of tile t and d_kind[t * cap_max + j] its kind, for j < n_sel[t]; kind -1 and a zero row
 * for j >= n_sel[t].  d_rows holds n_tiles * cap_max rows. */
int weftk_fit_selected_rows(const struct WeftFitState* st, float* d_rows, int32_t* d_kind, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WEFTK_WIRE_H */
