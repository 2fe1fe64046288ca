"""ctypes binding of the C ABI in include/rtb200.h (rise_b200/_lib/librtb200.so).

There is no fallback: if the library is missing or fails to load, every
entry point raises.  Build it with `make -C rise_b200/csrc` or
`__graft_entry__.build()`.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "librtb200.so")

OK = 0
E_INVALID, E_OOM, E_BUDGET, E_TIMEOUT, E_DEVICE, E_NOT_READY, E_CANCELLED = 1, 2, 3, 4, 5, 6, 7
STATUS_NAMES = {0: "OK", 1: "E_INVALID", 2: "E_OOM", 3: "E_BUDGET", 4: "E_TIMEOUT",
                5: "E_DEVICE", 6: "E_NOT_READY", 7: "E_CANCELLED"}
BVH_F32, BVH_Q8, BVH_W8, BVH_F16 = 0, 1, 2, 3

_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_i32 = ctypes.c_int32
_pvp = ctypes.POINTER(ctypes.c_void_p)
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pf64 = ctypes.POINTER(ctypes.c_double)

# name -> (restype, argtypes); every symbol declared in include/rtb200.h.
SIGNATURES = {
    "rtb200_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_size_t, _pvp]),
    "rtb200_ctx_destroy": (ctypes.c_int, [_vp]),
    "rtb200_last_error": (ctypes.c_char_p, [_vp]),
    "rtb200_ctx_bytes_in_use": (ctypes.c_size_t, [_vp]),
    "rtb200_scene_create": (ctypes.c_int, [_vp, _pvp]),
    "rtb200_scene_add_mesh": (ctypes.c_int, [_vp, _vp, _i64, _vp, _i64, _i32, _i32]),
    "rtb200_scene_commit": (ctypes.c_int, [_vp, _i32]),
    "rtb200_scene_info": (ctypes.c_int, [_vp, _pi64, _pi64, _pi64, _pf64]),
    "rtb200_scene_destroy": (ctypes.c_int, [_vp]),
    "rtb200_bvh_host_build": (ctypes.c_int, [_vp, _i64, _i32, _pvp]),
    "rtb200_bvh_host_info": (ctypes.c_int, [_vp, _pi64, _pi64]),
    "rtb200_bvh_host_export": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "rtb200_bvh_host_destroy": (ctypes.c_int, [_vp]),
    "rtb200_bvh_host_from_risemesh": (ctypes.c_int, [_vp, ctypes.c_int32, _vp]),
    "rtb200_risemesh_parse": (ctypes.c_int, [_vp, ctypes.c_size_t, _vp]),
    "rtb200_risemesh_info": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "rtb200_risemesh_destroy": (ctypes.c_int, [_vp]),
    "rtb200_risemesh_triangles": (ctypes.c_int, [_vp, _vp]),
    "rtb200_risemesh_normals": (ctypes.c_int, [_vp, _vp]),
    "rtb200_rgb_uplift": (ctypes.c_int, [_vp, ctypes.c_int32, _vp]),
    "rtb200_rgb_uplift_table": (ctypes.c_int, [_vp]),
    "rtb200_scene_add_rgb_spectrum": (ctypes.c_int, [_vp, _vp, _vp]),
    "rtb200_scene_add_blackbody": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int32, _vp]),
    "rtb200_scene_add_point_light": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_float]),
    "rtb200_scene_add_risemesh": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, ctypes.c_int32]),
    "rtb200_scene_add_spectral_packet": (ctypes.c_int, [_vp, ctypes.c_float, ctypes.c_float, ctypes.c_int32, _vp,
                                                        _vp]),
    "rtb200_cast_closest": (ctypes.c_int, [_vp, _vp, _i64, _vp]),
    "rtb200_cast_any": (ctypes.c_int, [_vp, _vp, _i64, _vp]),
    "rtb200_cast_closest_device": (ctypes.c_int, [_vp, _vp, _i64, _vp, _vp]),
    "rtb200_cast_any_device": (ctypes.c_int, [_vp, _vp, _i64, _vp, _vp]),
    "rtb200_cast_closest_noalloc": (ctypes.c_int, [_vp, _vp, _i64, _vp, _vp]),
    "rtb200_scene_device_status": (ctypes.c_int, [_vp, _vp]),
    "rtb200_scene_add_mesh_normals": (ctypes.c_int, [_vp, _vp, _i64, _vp, _i64, _vp, _i64, _vp, ctypes.c_int32,
                                                     ctypes.c_int32]),
    "rtb200_scene_add_spectrum": (ctypes.c_int, [_vp, _vp, _vp]),
    "rtb200_scene_add_material": (ctypes.c_int, [_vp, _vp, _vp]),
    "rtb200_scene_set_environment": (ctypes.c_int, [_vp, _i32, _i32]),
    "rtb200_scene_set_environment_map": (ctypes.c_int, [_vp, _vp, _i32, _i32, ctypes.c_float, _vp, _i32]),
    "rtb200_hdr_decode": (ctypes.c_int, [_vp, _i64, _vp, _vp, _vp]),
    "rtb200_scene_set_environment_rotation": (ctypes.c_int, [_vp, _vp]),
    "rtb200_job_create": (ctypes.c_int, [_vp, _vp, _vp]),
    "rtb200_job_render": (ctypes.c_int, [_vp, _i32]),
    "rtb200_job_read_film": (ctypes.c_int, [_vp, _vp]),
    "rtb200_job_read_sample_counts": (ctypes.c_int, [_vp, _vp]),
    "rtb200_job_read_rgb": (ctypes.c_int, [_vp, _vp]),
    "rtb200_job_read_display": (ctypes.c_int, [_vp, ctypes.c_float, ctypes.c_int32, _vp]),
    "rtb200_job_stats": (ctypes.c_int, [_vp, _vp]),
    "rtb200_job_destroy": (ctypes.c_int, [_vp]),
    "rtb200_engine_create": (ctypes.c_int, [_vp, _i32, _pvp]),
    "rtb200_engine_render": (ctypes.c_int, [_vp, _vp, _vp, _i32, _i32]),
    "rtb200_engine_submit": (ctypes.c_int, [_vp, _vp, _i32]),
    "rtb200_engine_step": (ctypes.c_int, [_vp, _i32, _i32]),
    "rtb200_engine_progress": (ctypes.c_int, [_vp, _vp, _pi64, _pi64]),
    "rtb200_engine_retire": (ctypes.c_int, [_vp, _vp]),
    "rtb200_engine_cancel": (ctypes.c_int, [_vp, _vp]),
    "rtb200_job_set_progress": (ctypes.c_int, [_vp, _vp, _vp]),
    "rtb200_engine_destroy": (ctypes.c_int, [_vp]),
    "rtb200_engine_set_poll": (ctypes.c_int, [_vp, ctypes.c_int32]),
    "rtb200_job_relmse": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ctypes.c_double)]),
}
NOALLOC_SCRATCH_BYTES = 256
NOALLOC_MAX_RAYS = 2147483647

_lib = None


class RTB200Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib():
    """Load librtb200.so (raises if it is missing: no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RTB200Error(E_DEVICE, f"native library not built: {LIB_PATH} "
                                        "(run `make -C rise_b200/csrc`)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code, ctx=None):
    if code != OK:
        msg = lib().rtb200_last_error(ctx).decode() if ctx else ""
        raise RTB200Error(code, msg)
