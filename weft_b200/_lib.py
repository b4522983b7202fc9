"""ctypes binding of libweftk.so (the C ABI declared in include/weftk.h).

The library is loaded lazily on first use.  There is no fallback: if the
shared library is missing or no sm_100 GPU is present, the call raises.
"""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libweftk.so")


class WeftkError(RuntimeError):
    """Raised when a libweftk entry point returns a non-zero status."""


class WeftPrim(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("geom", ctypes.c_float * 7), ("color0", ctypes.c_float * 3),
                ("color1", ctypes.c_float * 3), ("alpha", ctypes.c_float)]


class WeftEval(ctypes.Structure):
    _fields_ = [("prim_offset", ctypes.c_int32), ("prim_count", ctypes.c_int32),
                ("tile_offset", ctypes.c_int32), ("tile_size", ctypes.c_int32)]


class WeftTileDecodeDesc(ctypes.Structure):
    _fields_ = [("prim_offset", ctypes.c_int32), ("prim_count", ctypes.c_int32), ("target_x0", ctypes.c_int32),
                ("target_y0", ctypes.c_int32), ("target_w", ctypes.c_int32), ("target_h", ctypes.c_int32),
                ("source_size", ctypes.c_int32), ("res1_index", ctypes.c_int32), ("res0_r", ctypes.c_float),
                ("res0_g", ctypes.c_float), ("res0_b", ctypes.c_float), ("_pad2", ctypes.c_float)]


class WeftFitState(ctypes.Structure):
    """Device pointers of a fit (include/weftk_fit.h)."""
    _fields_ = [("n_tiles", ctypes.c_int32), ("cap_max", ctypes.c_int32), ("n_slots", ctypes.c_int64)] + [
        (n, ctypes.c_void_p) for n in ("src", "bg", "px_off", "size", "cap", "pool_off", "pool_cnt", "pool_cap", "n_alive",
                                       "n_sel", "sel_bits", "flags", "cur_obj", "sel", "cand", "prep", "alive", "kind",
                                       "partial", "status", "work")] + [
        ("variant", ctypes.c_int32 * 3), ("_pad", ctypes.c_int32), ("moments", ctypes.c_void_p),
        ("queue", ctypes.c_void_p), ("queue_ctl", ctypes.c_void_p)]

FIT_VARIANTS = 3


class WeftStackSet(ctypes.Structure):
    """Device pointers of a set of per-tile stacks (include/weftk_refine.h)."""
    _fields_ = [("n_tiles", ctypes.c_int32), ("max_prims", ctypes.c_int32)] + [
        (n, ctypes.c_void_p) for n in ("src", "px_off", "size", "prim_off", "kind", "order")] + [
        ("n_big", ctypes.c_int32), ("n_mid", ctypes.c_int32), ("n_s16", ctypes.c_int32),
        ("kinds_mask", ctypes.c_int32), ("moments", ctypes.c_void_p)]


class WeftRefineParams(ctypes.Structure):
    """Parameters of a per-image refiner (include/weftk_pipeline.h)."""
    _fields_ = [("cap", ctypes.c_int32), ("steps", ctypes.c_int32), ("min_tile", ctypes.c_int32),
                ("max_tile", ctypes.c_int32), ("chunk", ctypes.c_int32 * 3), ("variant", ctypes.c_int32 * 3),
                ("lr", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("eps", ctypes.c_float),
                ("threshold", ctypes.c_double), ("lam", ctypes.c_double), ("complex_threshold", ctypes.c_double),
                ("tables", ctypes.c_void_p), ("srgb_lut", ctypes.c_void_p)]


assert ctypes.sizeof(WeftRefineParams) == 96


# numpy mirrors of the C structs (same byte layout)
PRIM_DTYPE = np.dtype([("kind", np.int32), ("geom", np.float32, 7), ("color0", np.float32, 3),
                       ("color1", np.float32, 3), ("alpha", np.float32)])
EVAL_DTYPE = np.dtype([("prim_offset", np.int32), ("prim_count", np.int32), ("tile_offset", np.int32),
                       ("tile_size", np.int32)])
TILE_DECODE_DTYPE = np.dtype([("prim_offset", np.int32), ("prim_count", np.int32), ("target_x0", np.int32),
                              ("target_y0", np.int32), ("target_w", np.int32), ("target_h", np.int32),
                              ("source_size", np.int32), ("res1_index", np.int32), ("res0_r", np.float32),
                              ("res0_g", np.float32), ("res0_b", np.float32), ("_pad2", np.float32)])
assert PRIM_DTYPE.itemsize == ctypes.sizeof(WeftPrim) == 60
assert EVAL_DTYPE.itemsize == ctypes.sizeof(WeftEval) == 16
FIT_ITEM_DTYPE = np.dtype([("tile", np.int32), ("block", np.int32), ("first", np.int32), ("count", np.int32)])
assert TILE_DECODE_DTYPE.itemsize == ctypes.sizeof(WeftTileDecodeDesc) == 48
# WeftDctTile (include/weftk_dct.h)
DCT_TILE_DTYPE = np.dtype([("x", np.int32), ("y", np.int32), ("size", np.int32), ("_pad", np.int32),
                           ("step_scale", np.float64), ("coef_base", np.int64, 3), ("coef_stride", np.int32, 3),
                           ("_pad2", np.int32)])
assert DCT_TILE_DTYPE.itemsize == 64
assert ctypes.sizeof(WeftFitState) == 16 + 21 * 8 + 16 + 8 + 16

_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64

# name -> argtypes; every entry point returns int status
SIGNATURES: dict[str, list] = {
    "weftk_version": [],
    "weftk_last_error": [ctypes.c_char_p, ctypes.c_size_t],
    "weftk_init": [_I],
    "weftk_device_status": [_P],
    "weftk_score_evals": [_P, _I, _P, _P, _P, _I, _P],
    "weftk_score_evals_host": [_P, _I, _P, _I, _P, _I64, _P, _I],
    "weftk_render_tiles": [_P, _I, _P, _I, _P, _P, _I, _P, _I, _P, _I, _I, _I, _P],
    "weftk_render_tiles_host": [_P, _I, _P, _I, _P, _I, _P, _I, _P, _I, _I, _I],
    "weftk_fit_prepare": [_P, _P, _P],
    "weftk_fit_reset": [_P, _P, _P],
    "weftk_build_residuals": [_P, _P, _I, _P, _P, _I, _P, _P, _P],
    "weftk_fit_moments": [_P, _P, _P],
    "weftk_rans_decode_chunks": [_P, ctypes.c_int64, _P, _I, _P, ctypes.c_int64, _P],
    "weftk_fit_run": [_P, _I, ctypes.c_double, ctypes.c_double, _P, _P, _I, _P, _I, _P, _I, _P, _P],
    "weftk_refine_start": [_P, _P, _I, _P, _P, _P, _P, _P],
    "weftk_fit_round": [_P, _I, ctypes.c_double, ctypes.c_double, _P, _P, _I, _P, _I, _P, _I, _P],
    "weftk_fit_timing": [_I, _P, _P],
    "weftk_fit_round_static": [_P, _I, ctypes.c_double, ctypes.c_double, _P, _P, _I, _P, _I, _P, _I, _P],
    "weftk_fit_reseed": [_P, _I, _P],
    "weftk_stack_loss": [_P, _P, _P, _I, _P],
    "weftk_stack_loss_backward": [_P, _P, _P, _P, _P, _I, _P],
    "weftk_adam_step": [_P, _P, _P, _P, _P, _I, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, _P,
                        _P],
    "weftk_refine_steps": [_P, _I, _P, _P, _P, _P, _P, _P, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                           ctypes.c_float, _I, _P],
    "weftk_refine_step": [_P, _P, _P, _P, _P, _P, _P, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                          ctypes.c_float, _I, _P],
    "weftk_measure_fp32_peak": [_P],
    "weftk_fit_variant": [_I, _I, _P, _P, _P],
    "weftk_dct_apply": [_P, _I, _P, _I64, _I, _I, ctypes.c_float, ctypes.c_float, _I, _P, _I, _I, _I, _P],
    "weftk_raster_resize": [_P, _I, _I, _P, _I, _I, _P, _P],
    "weftk_quantize_rows": [_P, _P, _I, _P, _P],
    "weftk_fit_selected_rows": [_P, _P, _P, _P],
    "weftk_pool_side_bits": [_P, _P, _P],
    "weftk_gen_pools": [_P, _P, _P],
    "weftk_quadtree_work_bytes": [_I, _I, _I, _I, _P],
    "weftk_quadtree_variance": [_P, _I, _I, ctypes.c_double, _I, _I, _P, _I, _P, _P, _P],
    "weftk_extract_tiles": [_P, _I, _I, _P, _P, _I, _P, _P, _P],
    "weftk_refiner_create": [_P, _P],
    "weftk_refiner_destroy": [_P],
    "weftk_refine_image": [_P, _P, _I, _I, _P, _P, _P, _I, _P, _P],
    "weftk_bicubic_swap": [_P, _P, _P, _I, _P, _I, _P, _P, ctypes.c_double, _P, _P, _P, _P],
}

_lock = threading.Lock()
_lib = None
_inited_devices: set[int] = set()


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libweftk.so and bind its entry points (no GPU needed)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise WeftkError(f"libweftk.so not found at {path}; run `python -m weft_b200.build`")
        lib = ctypes.CDLL(path)
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        _lib = lib
        return lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    load().weftk_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int, what: str) -> None:
    if rc != 0:
        raise WeftkError(f"{what} failed with status {rc}: {last_error()}")


def lib_for_device(device: int = 0) -> ctypes.CDLL:
    """The bound library with `device` initialised (raises without an sm_100 GPU)."""
    lib = load()
    if device not in _inited_devices:
        check(lib.weftk_init(int(device)), "weftk_init")
        _inited_devices.add(device)
    return lib


def ptr(a) -> int:
    """Address of a numpy array or torch tensor (0 for None)."""
    if a is None:
        return 0
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())
