"""ctypes binding of libwos_b200.so (the C ABI in include/wos_b200.h).

The library holds every compute path; this module only loads it, declares the
signatures and turns error codes into exceptions.  There is no fallback: if
the library or a CUDA device is missing, the calls raise.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("WOS_B200_LIB") or _HERE.parent / "lib" / "libwos_b200.so")

WOS_OK = 0
WOS_ERR_INVALID_ARGUMENT = -1
WOS_ERR_CUDA = -2
WOS_ERR_EMPTY_SCENE = -3
WOS_ERR_UNSUPPORTED = -4
WOS_ERR_WORKSPACE = -5

STATUS_STACK_OVERFLOW = 1
STATUS_BAD_PRIM = 2
STATUS_NONFINITE = 4
STATUS_QUEUE_LIMIT = 8


class WosError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"wos_b200 error {code}: {msg}")
        self.code = code


class WosParams(ctypes.Structure):
    _fields_ = [
        ("nwalks", ctypes.c_int32),
        ("nsteps", ctypes.c_int32),
        ("epsilon", ctypes.c_float),
        ("double_sided", ctypes.c_int32),
        ("prevent_fd_artifacts", ctypes.c_int32),
        ("use_IS_for_greens", ctypes.c_int32),
        ("include_source", ctypes.c_int32),
        ("project_unterminated", ctypes.c_int32),
        ("use_bvh", ctypes.c_int32),
        ("walk_offset", ctypes.c_uint32),
        ("seed", ctypes.c_uint64),
        ("jitter", ctypes.c_float * 3),
    ]


class WosAdjointParams(ctypes.Structure):
    _fields_ = [
        ("epsilon2", ctypes.c_float),
        ("clamping", ctypes.c_float),
        ("control_variates", ctypes.c_int32),
        ("source_in_normal_derivative", ctypes.c_int32),
        ("ball_epsilon", ctypes.c_float),
        ("want_dV", ctypes.c_int32),
        ("want_dg", ctypes.c_int32),
        ("want_dsrc", ctypes.c_int32),
    ]


class WosSceneInfo(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32),
        ("n_vertices", ctypes.c_int32),
        ("n_faces", ctypes.c_int32),
        ("n_nodes", ctypes.c_int32),
        ("bvh_depth", ctypes.c_int32),
        ("source_type", ctypes.c_int32),
        ("aabb_min", ctypes.c_float * 3),
        ("aabb_max", ctypes.c_float * 3),
        ("source_params", ctypes.c_float * 5),
    ]


class WosLaunchConfig(ctypes.Structure):
    _fields_ = [
        ("block_threads", ctypes.c_int32),
        ("blocks_per_sm", ctypes.c_int32),
        ("chunk", ctypes.c_int32),
        ("smem_nodes", ctypes.c_int32),
    ]


class WosDetector(ctypes.Structure):
    _fields_ = [
        ("vmin", ctypes.c_float * 2),
        ("vmax", ctypes.c_float * 2),
        ("res", ctypes.c_int32 * 2),
        ("axis_u", ctypes.c_int32),
        ("axis_v", ctypes.c_int32),
        ("slab_axis", ctypes.c_int32),
        ("slab_center", ctypes.c_float),
        ("slab_half_width", ctypes.c_float),
        ("size", ctypes.c_float),
        ("flags", ctypes.c_int32),
    ]


WOS_DETECTOR_REFERENCE_AREA_PDF = 1


class WosBatchItem(ctypes.Structure):
    _fields_ = [
        ("scene", ctypes.c_void_p),
        ("P", ctypes.c_void_p),
        ("n", ctypes.c_int32),
        ("loss_kind", ctypes.c_int32),
        ("target_or_dLdu", ctypes.c_void_p),
        ("params", WosParams),
    ]


_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_S = ctypes.c_size_t

# name -> (restype, argtypes); every pointer is passed as an integer address.
SIGNATURES = {
    "wos_version": (_I, []),
    "wos_last_error_string": (ctypes.c_char_p, []),
    "wos_device_status": (_I, [_I, ctypes.POINTER(ctypes.c_int32)]),
    "wos_scene_create": (_I, [_I, _P, _I, _P, _I, _P, _I, _P, _P, ctypes.POINTER(_P)]),
    "wos_scene_destroy": (_I, [_P, _P]),
    "wos_scene_update_values": (_I, [_P, _P, _P]),
    "wos_scene_update_vertices": (_I, [_P, _P, _P]),
    "wos_scene_set_source": (_I, [_P, _I, _P]),
    "wos_scene_get_info": (_I, [_P, ctypes.POINTER(WosSceneInfo)]),
    "wos_scene_get_normals": (_I, [_P, _P, _P]),
    "wos_closest_point": (_I, [_P, _P, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P]),
    "wos_sdf": (_I, [_P, _P, _I, _I, _P, _P]),
    "wos_largest_inscribed_ball": (_I, [_P, _P, _P, _P, _I, _F, _I, _P, _P]),
    "wos_walk_records": (_I, [_P, _P, _I, ctypes.POINTER(WosParams), _P, _P, _P, _P, _P, _P, _P]),
    "wos_walk_values": (_I, [_P, _P, _I, ctypes.POINTER(WosParams), _P, _P, _P]),
    "wos_walk_values_plain": (_I, [_P, _P, _I, ctypes.POINTER(WosParams), _P, _P]),
    "wos_solve_workspace_size": (_S, [_I, ctypes.POINTER(WosParams)]),
    "wos_solve": (_I, [_P, _P, _I, ctypes.POINTER(WosParams), _P, _P, _P, _S, _P]),
    "wos_normal_derivative": (
        _I,
        [_P, _P, _P, _P, _P, _P, _I, ctypes.POINTER(WosParams), ctypes.POINTER(WosAdjointParams), _P, _P],
    ),
    "wos_normal_derivative_radius": (
        _I,
        [_P, _P, _P, _P, _P, _P, _P, _I, ctypes.POINTER(WosParams), ctypes.POINTER(WosAdjointParams), _P, _P],
    ),
    "wos_adjoint_workspace_size": (_S, [_P]),
    "wos_adjoint_records_workspace_size": (_S, [_P, _I, ctypes.POINTER(WosParams)]),
    "wos_adjoint": (
        _I,
        [_P, _P, _I, ctypes.POINTER(WosParams), ctypes.POINTER(WosAdjointParams), _P, _P, _P, _P, _P, _S, _P],
    ),
    "wos_walk_record_bytes": (_S, [_I]),
    "wos_solve_records": (_I, [_P, _P, _I, ctypes.POINTER(WosParams), _P, _P, _P, _P, _P, _S, _P]),
    "wos_adjoint_records": (
        _I,
        [_P, _P, _I, ctypes.POINTER(WosParams), ctypes.POINTER(WosAdjointParams), _P, _P, _P, _P, _P, _P, _P, _S,
         _P],
    ),
    "wos_solve_adjoint_workspace_size": (_S, [_P, _I, ctypes.POINTER(WosParams), ctypes.POINTER(WosAdjointParams)]),
    "wos_soft_walk_workspace_size": (_S, [_I, ctypes.POINTER(WosParams)]),
    "wos_soft_walk": (_I, [_P, _P, _I, ctypes.POINTER(WosParams), _P, _P, _P, _P, _P, _P, _P, _S, _P]),
    "wos_soft_walk_adjoint": (_I, [_P, _P, _I, ctypes.POINTER(WosParams), _P, _P, _P, _P]),
    "wos_boundary_term": (_I, [_P, ctypes.POINTER(WosDetector), _I, ctypes.c_uint64, _P, _P, _P, _P, _P]),
    "wos_solve_tangent_workspace_size": (_S, [_P, _I, ctypes.POINTER(WosParams), ctypes.POINTER(WosAdjointParams)]),
    "wos_solve_tangent": (
        _I,
        [_P, _P, _I, ctypes.POINTER(WosParams), ctypes.POINTER(WosAdjointParams), _P, _P, _P, _P, _P, _P, _P, _P, _S,
         _P],
    ),
    "wos_solve_adjoint": (
        _I,
        [_P, _P, _I, ctypes.POINTER(WosParams), ctypes.POINTER(WosAdjointParams), _I, _P, _P, _P, _P, _P, _P, _P,
         _P, _S, _P],
    ),
    "wos_solve_noalloc": (_I, [_P, _P, _I, ctypes.POINTER(WosParams), _P, _P, _P]),
    "wos_batch_create": (_I, [ctypes.POINTER(WosBatchItem), _I, ctypes.POINTER(WosAdjointParams), _I, _P,
                              ctypes.POINTER(_P)]),
    "wos_batch_set_launch": (_I, [_P, _I, _I, _I]),
    "wos_batch_autotune": (_I, [_P, _P, _P, _I, _I, _P, _P, _P]),
    "wos_batch_autotune_slots": (_I, [_P, _P, _P, _P, _I, _I, ctypes.c_double, _P, _P, _P]),
    "wos_batch_get_launch": (_I, [_P, _I, _I, _P]),
    "wos_batch_set_launch_slot": (_I, [_P, _I, _I, _I, _I, _I]),
    "wos_batch_refresh": (_I, [_P, _P]),
    "wos_batch_run": (_I, [_P, _I, _P]),
    "wos_batch_outputs": (_I, [_P, _I, _P, _P, _P, _P, _P, _P]),
    "wos_batch_copy_outputs": (_I, [_P, _I, _P, _P, _P, _P, _P, _P, _P]),
    "wos_batch_info": (_I, [_P, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                            ctypes.POINTER(ctypes.c_int32)]),
    "wos_batch_destroy": (_I, [_P, _P]),
    "wos_set_work_counting": (_I, [_I]),
    "wos_set_sample_order": (_I, [_I]),
    "wos_work_counters": (_I, [_I, ctypes.POINTER(ctypes.c_int64)]),
    "wos_set_launch_config": (_I, [_I, ctypes.POINTER(WosLaunchConfig)]),
    "wos_get_launch_config": (_I, [_I, ctypes.POINTER(WosLaunchConfig)]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load libwos_b200.so once (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise WosError(WOS_ERR_UNSUPPORTED, f"{LIB_PATH} not built; run diff-wos_b200/build.py")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != WOS_OK:
        msg = lib().wos_last_error_string()
        raise WosError(rc, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))


def device_status(reset: bool = False) -> int:
    v = ctypes.c_int32(0)
    call("wos_device_status", int(reset), ctypes.byref(v))
    return int(v.value)


def set_work_counting(enable: bool) -> None:
    call("wos_set_work_counting", int(enable))


def set_sample_order(mode: int) -> None:
    """1: adjoint samples from records run sorted by boundary primitive; 0: in queue order."""
    call("wos_set_sample_order", int(mode))


def work_counters(reset: bool = False) -> dict:
    """Totals since the last reset: {queries, nodes, prims}."""
    v = (ctypes.c_int64 * 3)()
    call("wos_work_counters", int(reset), v)
    return dict(queries=int(v[0]), nodes=int(v[1]), prims=int(v[2]))


def get_launch_config(dim: int) -> WosLaunchConfig:
    c = WosLaunchConfig()
    call("wos_get_launch_config", dim, ctypes.byref(c))
    return c


def set_launch_config(dim: int, block_threads=0, blocks_per_sm=-1, chunk=0, smem_nodes=-1) -> None:
    c = WosLaunchConfig(block_threads, blocks_per_sm, chunk, smem_nodes)
    call("wos_set_launch_config", dim, ctypes.byref(c))
