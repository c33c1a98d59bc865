"""The C ABI library loads and exports every entry point include/wos_b200.h
declares, with the layouts the Python binding assumes.  No compute calls:
these run without a GPU."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "wos_b200.h"


def declared():
    src = HEADER.read_text()
    return sorted(set(re.findall(r"WOS_API\s+[\w\s\*]*?\b(wos_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    for n in ("wos_scene_create", "wos_solve", "wos_adjoint", "wos_closest_point", "wos_walk_records",
              "wos_normal_derivative", "wos_largest_inscribed_ball"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from wos import _lib
    L = _lib.lib()
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from wos import _lib
    assert set(declared()) <= set(_lib.SIGNATURES), set(declared()) - set(_lib.SIGNATURES)


def test_struct_layouts():
    from wos import _lib
    assert ctypes.sizeof(_lib.WosParams) == 64
    assert _lib.WosParams.seed.offset == 40
    assert ctypes.sizeof(_lib.WosAdjointParams) == 32
    assert ctypes.sizeof(_lib.WosLaunchConfig) == 16


def test_oracle_params_match_library_params():
    from oracle import oracle as O
    from wos import _lib
    assert [f[0] for f in O.Params._fields_] == [f[0] for f in _lib.WosParams._fields_]
    assert [f[0] for f in O.AdjParams._fields_] == [f[0] for f in _lib.WosAdjointParams._fields_]
    assert [f[0] for f in O.Detector._fields_] == [f[0] for f in _lib.WosDetector._fields_]
    assert ctypes.sizeof(O.Detector) == ctypes.sizeof(_lib.WosDetector) == 52


def test_argument_validation_without_gpu():
    from wos import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.wos_scene_create(4, None, 1, None, 1, None, 0, None, None, ctypes.byref(h)) == _lib.WOS_ERR_INVALID_ARGUMENT
    assert b"dim" in L.wos_last_error_string()
    assert L.wos_scene_create(2, None, 0, None, 0, None, 0, None, None, ctypes.byref(h)) == _lib.WOS_ERR_EMPTY_SCENE
    assert L.wos_scene_create(3, None, 3, None, 1, None, 1, None, None, ctypes.byref(h)) == _lib.WOS_ERR_UNSUPPORTED
    assert L.wos_scene_create(2, None, 3, None, 1, None, 7, None, None, ctypes.byref(h)) == \
        _lib.WOS_ERR_INVALID_ARGUMENT
    p = _lib.WosParams(0, 32, 1e-3, 0, 0, 0, 0, 0, 1, 0, 0)
    assert L.wos_solve(ctypes.c_void_p(1), None, 10, ctypes.byref(p), None, None, None, 0, None) == \
        _lib.WOS_ERR_INVALID_ARGUMENT
    assert b"nwalks" in L.wos_last_error_string()
    assert L.wos_solve_workspace_size(10, ctypes.byref(_lib.WosParams(4, 32, 1e-3))) >= 10 * 4 * 4
    assert L.wos_sdf(None, None, 1, 1, None, None) == _lib.WOS_ERR_INVALID_ARGUMENT
    bt = (ctypes.c_int32 * 1)(100)
    ch = (ctypes.c_int32 * 1)(16)
    assert L.wos_batch_autotune(None, bt, ch, 1, 1, None, None, None) == _lib.WOS_ERR_INVALID_ARGUMENT
    assert L.wos_batch_autotune(ctypes.c_void_p(1), bt, ch, 0, 1, None, None, None) == _lib.WOS_ERR_INVALID_ARGUMENT
    assert L.wos_batch_autotune(ctypes.c_void_p(1), bt, ch, 1, 1, None, None, None) == _lib.WOS_ERR_INVALID_ARGUMENT
    assert b"candidate 0" in L.wos_last_error_string()
    bs = (ctypes.c_int32 * 1)(0)
    assert L.wos_batch_autotune_slots(None, bt, bs, ch, 1, 1, 1.0, None, None, None) == _lib.WOS_ERR_INVALID_ARGUMENT
    assert L.wos_batch_autotune_slots(ctypes.c_void_p(1), bt, bs, ch, 1, 1, 0.0, None, None, None) == \
        _lib.WOS_ERR_INVALID_ARGUMENT
    assert b"sample" in L.wos_last_error_string()
    assert L.wos_batch_get_launch(ctypes.c_void_p(1), 4, 0, (ctypes.c_int32 * 3)()) == _lib.WOS_ERR_INVALID_ARGUMENT
    assert L.wos_version() >= 100


def test_launch_config_roundtrip():
    import wos
    old = wos.get_launch_config(2)
    try:
        wos.set_launch_config(2, block_threads=128, chunk=16, smem_nodes=0)
        c = wos.get_launch_config(2)
        assert (c.block_threads, c.chunk, c.smem_nodes) == (128, 16, 0)
        with pytest.raises(wos.WosError):
            wos.set_launch_config(2, block_threads=100)
    finally:
        wos.set_launch_config(2, old.block_threads, old.blocks_per_sm, old.chunk, old.smem_nodes)
