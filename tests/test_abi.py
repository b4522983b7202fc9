"""The C-ABI library loads without a GPU and exports every symbol include/*.h declares."""

from __future__ import annotations

import ctypes
import glob
import os
import re

import numpy as np

from weft_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points() -> list[str]:
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*int\s+(weftk_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_builds_and_loads():
    from weft_b200 import build

    build.build()
    lib = _lib.load()
    assert lib.weftk_version() >= 10000


def test_every_declared_symbol_is_exported_and_bound():
    lib = _lib.load()
    names = declared_entry_points()
    assert "weftk_score_evals" in names and "weftk_render_tiles" in names
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, f"{n} declared in include/ but not bound in _lib.SIGNATURES"


def test_struct_layouts_match_reference_records():
    assert ctypes.sizeof(_lib.WeftPrim) == 60
    assert ctypes.sizeof(_lib.WeftEval) == 16
    assert ctypes.sizeof(_lib.WeftTileDecodeDesc) == 48
    # byte offsets of the reference dtypes (src/weft/gpu_render.py:241-247, :578-591)
    assert [_lib.PRIM_DTYPE.fields[k][1] for k in ("kind", "geom", "color0", "color1", "alpha")] == [0, 4, 32, 44, 56]
    assert [_lib.TILE_DECODE_DTYPE.fields[k][1] for k in ("res0_r", "res0_g", "res0_b")] == [32, 36, 40]


def test_last_error_is_empty_or_text():
    assert isinstance(_lib.last_error(), str)


def test_host_entry_points_reject_bad_descriptors_without_gpu_work():
    """Argument checks run on the host before any device call."""
    lib = _lib.load()
    ev = np.zeros(1, _lib.EVAL_DTYPE)
    ev["tile_size"] = 0  # invalid
    out = np.zeros(1, np.float32)
    tiles = np.zeros(3, np.float32)
    prims = np.zeros(1, _lib.PRIM_DTYPE)
    rc = lib.weftk_score_evals_host(_lib.ptr(ev), 1, _lib.ptr(prims), 1, _lib.ptr(tiles), 3, _lib.ptr(out), 0)
    assert rc == -1 and "out of range" in _lib.last_error()
