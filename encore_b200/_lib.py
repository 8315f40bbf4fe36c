"""ctypes binding of ``include/encore_b200.h``.

The library is loaded from the package directory.  There is no fallback: if
``libencore_b200.so`` is missing or fails to load, every engine call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libencore_b200.so"

ENC_OK = 0
ENC_ERR_INVALID_ARG = 1
ENC_ERR_CUDA = 2
ENC_ERR_OUT_OF_MEMORY = 3
ENC_ERR_WATCHDOG = 4
ENC_ERR_BUDGET = 5
ENC_ERR_NOT_READY = 6
ENC_ERR_CANCELLED = 7
ENC_ERR_UNSUPPORTED = 8

ENC_ACCEL_WBVH = 0
ENC_ACCEL_KDTREE = 1
ENC_PRED_REFERENCE = 0
ENC_PRED_NOCLAMP = 1
ENC_GATHER_IGNORE_NORMAL = 1

_STATUS_NAMES = {
    1: "invalid argument", 2: "CUDA error", 3: "out of memory", 4: "watchdog",
    5: "over budget", 6: "not ready", 7: "cancelled", 8: "unsupported",
}


class EncoreError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {_STATUS_NAMES.get(status, status)} ({status}): {msg}")
        self.status = status


class BuildOpts(C.Structure):
    _fields_ = [("kind", C.c_int32), ("width", C.c_int32), ("max_leaf_tris", C.c_int32),
                ("predicate", C.c_int32)]


class LaunchOpts(C.Structure):
    _fields_ = [("block_threads", C.c_int32), ("blocks_per_sm", C.c_int32), ("chunk", C.c_int32),
                ("stack_depth", C.c_int32)]


class BinOpts(C.Structure):
    _fields_ = [("origin_bits", C.c_int32), ("dir_bits", C.c_int32), ("probe_frac", C.c_float)]


class AccelInfo(C.Structure):
    _fields_ = [("kind", C.c_int32), ("width", C.c_int32), ("predicate", C.c_int32),
                ("ntris", C.c_uint32), ("nnodes", C.c_uint32), ("node_bytes", C.c_uint64),
                ("tri_bytes", C.c_uint64), ("device_bytes", C.c_uint64),
                ("build_seconds", C.c_double), ("scene_lo", C.c_float * 3),
                ("scene_hi", C.c_float * 3)]


class BatchItem(C.Structure):
    _fields_ = [("accel", C.c_void_p), ("d_rays", C.c_void_p), ("d_hits", C.c_void_p),
                ("nrays", C.c_uint32), ("reserved", C.c_uint32)]


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("slots", C.c_uint32), ("slot_rays", C.c_uint64),
                ("budget_bytes", C.c_uint64), ("launch", LaunchOpts)]


class RequestInfo(C.Structure):
    _fields_ = [("submit_s", C.c_double), ("start_s", C.c_double), ("done_s", C.c_double),
                ("nrays", C.c_uint64), ("status", C.c_int32), ("kind", C.c_int32)]


class Camera(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("look", C.c_float * 3), ("up", C.c_float * 3),
                ("fov_deg", C.c_float), ("width", C.c_uint32), ("height", C.c_uint32),
                ("jitter_seed", C.c_uint32)]


class PhotonOpts(C.Structure):
    _fields_ = [("light_center", C.c_float * 3), ("light_size", C.c_float),
                ("nphotons", C.c_uint32), ("max_bounces", C.c_uint32), ("albedo", C.c_float),
                ("seed", C.c_uint32), ("emit_offset", C.c_float), ("bounce_offset", C.c_float)]


class PhotonStore(C.Structure):
    _fields_ = [("d_pos", C.c_void_p), ("d_nrm", C.c_void_p), ("d_pow", C.c_void_p),
                ("d_tag", C.c_void_p), ("capacity", C.c_uint32)]


class ModelXform(C.Structure):
    _fields_ = [("center", C.c_float * 3), ("size", C.c_float), ("angle_deg", C.c_float),
                ("axis", C.c_float * 3)]


class SceneDesc(C.Structure):
    _fields_ = [("ntris", C.c_uint32), ("nprims", C.c_uint32), ("nmodels", C.c_uint32),
                ("nmaterials", C.c_uint32), ("nlights", C.c_uint32), ("nspheres", C.c_uint32),
                ("nunknown", C.c_uint32), ("has_camera", C.c_int32), ("cam_eye", C.c_float * 3),
                ("cam_look", C.c_float * 3), ("cam_up", C.c_float * 3), ("cam_fov_deg", C.c_float),
                ("cam_aspect", C.c_float), ("cam_near", C.c_float), ("cam_far", C.c_float),
                ("background", C.c_float * 4)]


ENC_LIGHT_RECT = 0
ENC_LIGHT_POINT = 1


class SceneLight(C.Structure):
    _fields_ = [("kind", C.c_int32), ("center", C.c_float * 3), ("size", C.c_float),
                ("color", C.c_float * 3)]


P = C.c_void_p
F = C.POINTER(C.c_float)

# name -> (restype, argtypes); every symbol include/*.h declares.
SIGNATURES = {
    "enc_abi_version": (C.c_int32, []),
    "enc_last_error": (C.c_char_p, []),
    "enc_device_count": (C.c_int32, [C.POINTER(C.c_int32)]),
    "enc_scene_create": (C.c_int32, [P, C.c_uint32, C.POINTER(P)]),
    "enc_scene_destroy": (C.c_int32, [P]),
    "enc_scene_load_ply": (C.c_int32, [C.c_char_p, C.POINTER(ModelXform), C.POINTER(P)]),
    "enc_scene_load_file": (C.c_int32, [C.c_char_p, C.c_char_p, C.POINTER(P)]),
    "enc_scene_desc_get": (C.c_int32, [P, C.POINTER(SceneDesc)]),
    "enc_scene_tris": (C.c_int32, [P, P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "enc_scene_prims": (C.c_int32, [P, P, P, C.c_uint32]),
    "enc_scene_materials": (C.c_int32, [P, P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "enc_scene_lights": (C.c_int32, [P, C.POINTER(SceneLight), C.c_uint32, C.POINTER(C.c_uint32)]),
    "enc_accel_build": (C.c_int32, [P, C.POINTER(BuildOpts), C.c_int32, C.POINTER(P)]),
    "enc_accel_destroy": (C.c_int32, [P]),
    "enc_accel_refit": (C.c_int32, [P, P, C.c_uint32]),
    "enc_accel_serialize": (C.c_int32, [P, P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "enc_accel_deserialize": (C.c_int32, [P, C.c_size_t, C.c_int32, C.POINTER(P)]),
    "enc_accel_info_get": (C.c_int32, [P, C.POINTER(AccelInfo)]),
    "enc_intersect_closest": (C.c_int32, [P, P, C.c_size_t, P, C.POINTER(LaunchOpts), P]),
    "enc_intersect_closest_od": (C.c_int32, [P, P, C.c_size_t, P, C.POINTER(LaunchOpts), P]),
    "enc_intersect_closest_device": (C.c_int32, [P, P, C.c_size_t, P, C.POINTER(LaunchOpts), P]),
    "enc_bin_scratch_bytes": (C.c_int32, [C.c_size_t, C.POINTER(BinOpts),
                                          C.POINTER(C.c_size_t)]),
    "enc_bin_rays": (C.c_int32, [P, P, C.c_size_t, P, C.c_size_t, C.POINTER(BinOpts),
                                 C.POINTER(C.c_void_p), P]),
    "enc_intersect_closest_device_ordered": (C.c_int32, [P, P, C.c_size_t, P, P,
                                                         C.POINTER(LaunchOpts), P]),
    "enc_intersect_closest_device_binned": (C.c_int32, [P, P, C.c_size_t, P, P, C.c_size_t,
                                                        C.POINTER(BinOpts),
                                                        C.POINTER(LaunchOpts), P]),
    "enc_intersect_any": (C.c_int32, [P, P, C.c_size_t, P, C.POINTER(LaunchOpts), P]),
    "enc_intersect_any_device": (C.c_int32, [P, P, C.c_size_t, P, C.POINTER(LaunchOpts), P]),
    "enc_accel_check": (C.c_int32, [P, P]),
    "enc_accel_count_visits": (C.c_int32, [P, P, C.c_size_t, P, P]),
    "enc_intersect_closest_noalloc": (C.c_int32, [P, P, C.c_size_t, P, P]),
    "enc_batch_create": (C.c_int32, [C.POINTER(BatchItem), C.c_uint32, C.POINTER(LaunchOpts),
                                     C.POINTER(P)]),
    "enc_batch_launch": (C.c_int32, [P, P]),
    "enc_batch_launch_graph": (C.c_int32, [P, P]),
    "enc_batch_check": (C.c_int32, [P, P]),
    "enc_batch_destroy": (C.c_int32, [P]),
    "enc_server_create": (C.c_int32, [C.POINTER(ServerOpts), C.POINTER(P)]),
    "enc_server_add_scene": (C.c_int32, [P, P, C.POINTER(C.c_uint32)]),
    "enc_server_submit": (C.c_int32, [P, C.c_uint32, C.c_int32, P, C.c_uint64, P,
                                      C.POINTER(C.c_uint64)]),
    "enc_server_wait": (C.c_int32, [P, C.c_uint64, C.c_double, C.POINTER(RequestInfo)]),
    "enc_server_cancel": (C.c_int32, [P, C.c_uint64]),
    "enc_server_now": (C.c_double, []),
    "enc_server_destroy": (C.c_int32, [P]),
    "enc_camera_rays_device": (C.c_int32, [C.POINTER(Camera), P, P]),
    "enc_hit_surface_device": (C.c_int32, [P, P, C.c_size_t, P, P, P]),
    "enc_diffuse_rays_device": (C.c_int32, [P, P, P, C.c_size_t, C.c_uint32, C.c_uint32,
                                            C.c_float, P, P]),
    "enc_photons_trace_device": (C.c_int32, [P, C.POINTER(PhotonOpts), P, P, P, C.c_uint32,
                                             C.POINTER(C.c_uint32), P]),
    "enc_photons_trace_maps_device": (C.c_int32, [P, C.POINTER(PhotonOpts), C.c_float, C.c_int32,
                                                  C.POINTER(PhotonStore), C.POINTER(PhotonStore),
                                                  C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), P]),
    "enc_photons_trace_maps": (C.c_int32, [P, C.POINTER(PhotonOpts), C.c_float, C.c_int32,
                                           C.POINTER(PhotonStore), C.POINTER(PhotonStore),
                                           C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), P]),
    "enc_photonmap_create_device": (C.c_int32, [P, P, P, C.c_size_t, C.c_int32, C.c_int32,
                                                C.POINTER(P)]),
    "enc_photonmap_create": (C.c_int32, [P, P, P, C.c_size_t, C.c_int32, C.c_int32, C.POINTER(P)]),
    "enc_photonmap_destroy": (C.c_int32, [P]),
    "enc_photonmap_serialize": (C.c_int32, [P, P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "enc_photonmap_deserialize": (C.c_int32, [P, C.c_size_t, C.c_int32, C.POINTER(P)]),
    "enc_photonmap_check": (C.c_int32, [P, P]),
    "enc_photonmap_radiance": (C.c_int32, [P, P, P, C.c_size_t, C.c_int32, C.c_float, C.c_int32, P, P]),
    "enc_photonmap_radiance_device": (C.c_int32, [P, P, P, C.c_size_t, C.c_int32, C.c_float, C.c_int32, P, P]),
    "enc_photonmap_count_visits": (C.c_int32, [P, P, P, C.c_size_t, C.c_int32, C.c_float,
                                               C.c_int32, P, P, P]),
    "enc_photonmap_nearest": (C.c_int32, [P, P, P, C.c_size_t, C.c_int32, C.c_float, C.c_int32, P, P, P, P]),
}

_lib = None
_lock = threading.Lock()


def load(path: os.PathLike | None = None):
    """Loads (once) and returns the engine library; raises if it is missing."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = Path(path or os.environ.get("ENC_LIB_PATH") or LIB_PATH)
        if not p.exists():
            raise RuntimeError(
                f"{p} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                "(the engine has no CPU fallback)")
        lib = C.CDLL(str(p))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(status: int, where: str) -> None:
    if status != ENC_OK:
        msg = load().enc_last_error()
        raise EncoreError(status, where, msg.decode() if msg else "")


def ptr(a) -> int | None:
    """Address of a numpy array, torch tensor or raw int pointer."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data
