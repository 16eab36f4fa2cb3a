"""ctypes binding of libvmap_b200.so (include/vmap_c.h).

The library is built in-tree (``python -m voxelmapping_b200.build``); importing
this module without it raises ImportError - there is no fallback
implementation.
"""
import ctypes as C
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libvmap_b200.so"

VMAP_OK = 0
STATUS_NAMES = {0: "VMAP_OK", 1: "VMAP_ERR_INVALID_ARG", 2: "VMAP_ERR_CUDA", 3: "VMAP_ERR_OUT_OF_MEMORY",
                4: "VMAP_ERR_POOL_FULL", 5: "VMAP_ERR_HASH_FULL", 6: "VMAP_ERR_RANGE",
                7: "VMAP_ERR_BUFFER_FULL", 8: "VMAP_ERR_NO_DEVICE"}

FLAG_POOL_FULL, FLAG_HASH_FULL, FLAG_RANGE, FLAG_BUFFER_FULL, FLAG_BAD_SNAPSHOT, FLAG_STEP_STALLED = 1, 2, 4, 8, 16, 32

VOXEL_REF, VOXEL_F32, VOXEL_F16, VOXEL_I16 = 0, 1, 2, 3
FORMAT_NAMES = {"ref": VOXEL_REF, "f32": VOXEL_F32, "f16": VOXEL_F16, "i16": VOXEL_I16}
DEPTH_F32, DEPTH_U16 = 0, 1
STAGES = ["alloc", "visibility", "fuse", "zrange", "raycast", "normals", "mesh"]


class VmapError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = "%s (%d)" % (STATUS_NAMES.get(status, "?"), status)
        if what:
            msg += " in " + what
        detail = lib().vmap_last_error().decode() if status in (2, 3, 8) else ""
        if detail:
            msg += ": " + detail
        super().__init__(msg)


class Config(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int),
                ("fx", C.c_float), ("fy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
                ("num_entries", C.c_int), ("num_blocks", C.c_int), ("voxel_size", C.c_float),
                ("num_buckets", C.c_int), ("truncation", C.c_float), ("voxel_format", C.c_int),
                ("max_weight", C.c_int), ("with_color", C.c_int), ("raycast_mode", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("allocated_blocks", C.c_uint32), ("capacity_blocks", C.c_uint32),
                ("visible_blocks", C.c_uint32), ("error_flags", C.c_uint32),
                ("failed_allocs", C.c_uint32), ("last_triangles", C.c_uint32),
                ("pool_bytes", C.c_uint64), ("device_bytes", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class HostFrame(C.Structure):
    """vmap_host_frame: one frame for vmap_frame_host_async."""
    _fields_ = [("depth_host", C.c_void_p), ("depth_type", C.c_int), ("depth_scale", C.c_float),
                ("rgb_host", C.c_void_p), ("pose", C.c_double * 16), ("vmap_host", C.c_void_p),
                ("nmap_host", C.c_void_p)]


class LaunchConfig(C.Structure):
    """vmap_launch_config: grid of every stage in CTAs per SM (0 = default)."""
    _fields_ = [("alloc_ctas_per_sm", C.c_int), ("visibility_ctas_per_sm", C.c_int), ("fuse_ctas_per_sm", C.c_int),
                ("zrange_ctas_per_sm", C.c_int), ("raycast_ctas_per_sm", C.c_int), ("normals_ctas_per_sm", C.c_int),
                ("mesh_ctas_per_sm", C.c_int), ("raycast_tile_order", C.c_int),
                ("raycast_tile_width", C.c_int), ("raycast_threads_per_cta", C.c_int),
                ("batch_schedule", C.c_int)]


class SnapshotHeader(C.Structure):
    """vmap_snapshot_header: the first 64 bytes of a vmap_snapshot_save image."""
    _fields_ = [("magic", C.c_char * 8), ("version", C.c_uint32), ("header_bytes", C.c_uint32),
                ("voxel_format", C.c_int32), ("with_color", C.c_int32), ("block_bytes", C.c_uint32),
                ("n_blocks", C.c_uint32), ("voxel_size", C.c_float), ("truncation", C.c_float),
                ("max_weight", C.c_int32), ("error_flags", C.c_uint32), ("keys_offset", C.c_uint64),
                ("pool_offset", C.c_uint64)]


class BatchFrame(C.Structure):
    _fields_ = [("depth_dev", C.c_void_p), ("depth_type", C.c_int), ("depth_pitch", C.c_size_t),
                ("depth_scale", C.c_float), ("rgb_dev", C.c_void_p), ("rgb_pitch", C.c_size_t),
                ("pose", C.c_double * 16), ("vmap_dev", C.c_void_p), ("vmap_pitch", C.c_size_t),
                ("nmap_dev", C.c_void_p), ("nmap_pitch", C.c_size_t)]


P = C.c_void_p
SZ = C.c_size_t
DBL16 = C.POINTER(C.c_double)

# name -> (restype, argtypes); every symbol include/vmap_c.h declares
SIGNATURES = {
    "vmap_create": (C.c_int, [C.POINTER(Config), C.POINTER(P)]),
    "vmap_destroy": (C.c_int, [P]),
    "vmap_reset": (C.c_int, [P, P]),
    "vmap_get_config": (C.c_int, [P, C.POINTER(Config)]),
    "vmap_fuse_depth": (C.c_int, [P, P, C.c_int, SZ, C.c_float, DBL16, P]),
    "vmap_fuse_depth_rgb": (C.c_int, [P, P, C.c_int, SZ, C.c_float, P, SZ, DBL16, P]),
    "vmap_fuse_host": (C.c_int, [P, P, C.c_int, C.c_float, P, DBL16, P]),
    "vmap_check_visible_blocks": (C.c_int, [P, DBL16, P]),
    "vmap_render_scene": (C.c_int, [P, DBL16, P, SZ, P, SZ, P]),
    "vmap_render_scene_host": (C.c_int, [P, DBL16, P, P, P]),
    "vmap_compute_normal": (C.c_int, [P, SZ, P, SZ, C.c_int, C.c_int, P]),
    "vmap_render_phong": (C.c_int, [P, SZ, P, SZ, P, SZ, C.c_int, C.c_int, P]),
    "vmap_polygonize": (C.c_int, [P, P, P, C.c_uint32, P, P]),
    "vmap_polygonize_host": (C.c_int, [P, C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.POINTER(C.c_float)),
                                       C.POINTER(C.c_uint32), P]),
    "vmap_surface_points": (C.c_int, [P, C.c_uint32, P, P]),
    "vmap_batch_create": (C.c_int, [C.POINTER(P), C.c_int, C.POINTER(P)]),
    "vmap_batch_destroy": (C.c_int, [P]),
    "vmap_batch_step": (C.c_int, [P, C.POINTER(BatchFrame), P]),
    "vmap_batch_stall_probe": (C.c_int, [P, C.POINTER(BatchFrame), C.c_uint32, P]),
    "vmap_get_stats": (C.c_int, [P, P, C.POINTER(Stats)]),
    "vmap_clear_errors": (C.c_int, [P, P]),
    "vmap_export_blocks": (C.c_int, [P, P, P, P, P, C.c_uint32, C.POINTER(C.c_uint32), P]),
    "vmap_copy_counters": (C.c_int, [P, P, P]),
    "vmap_export_blocks_static": (C.c_int, [P, C.c_uint32, C.c_uint32, P, P, P, P, C.POINTER(C.c_uint32), P]),
    "vmap_required_bytes": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_uint64)]),
    "vmap_create_in": (C.c_int, [C.POINTER(Config), P, C.c_uint64, P, C.POINTER(P)]),
    "vmap_batch_create_slots": (C.c_int, [C.c_int, C.c_int, C.POINTER(P)]),
    "vmap_batch_set_map": (C.c_int, [P, C.c_int, P]),
    "vmap_frame_host_async": (C.c_int, [P, C.POINTER(HostFrame), P]),
    "vmap_host_wait": (C.c_int, [P, P]),
    "vmap_get_launch_config": (C.c_int, [P, C.POINTER(LaunchConfig)]),
    "vmap_set_launch_config": (C.c_int, [P, C.POINTER(LaunchConfig)]),
    "vmap_batch_get_launch_config": (C.c_int, [P, C.POINTER(LaunchConfig)]),
    "vmap_batch_set_launch_config": (C.c_int, [P, C.POINTER(LaunchConfig)]),
    "vmap_snapshot_save": (C.c_int, [P, P, C.c_uint64, C.POINTER(C.c_uint64), P]),
    "vmap_snapshot_load": (C.c_int, [P, P, C.c_uint64, P]),
    "vmap_timing_enable": (C.c_int, [P, C.c_uint32]),
    "vmap_timing_read": (C.c_int, [P, C.POINTER(C.c_double), C.POINTER(C.c_uint32)]),
    "vmap_pose_inverse": (None, [DBL16, DBL16]),
    "vmap_block_hash": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int]),
    "vmap_block_hash_device": (C.c_int, [P, C.c_uint32, C.c_int, P, P]),
    "vmap_block_bytes": (SZ, [C.c_int, C.c_int]),
    "vmap_status_string": (C.c_char_p, [C.c_int]),
    "vmap_last_error": (C.c_char_p, []),
    "vmap_abi_version": (C.c_int, []),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError("%s is missing: build it with `python -m voxelmapping_b200.build` "
                              "(no CPU fallback exists)" % LIB_PATH)
        h = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


def check(status, what=""):
    if status != VMAP_OK:
        raise VmapError(status, what)


def pose_arg(pose):
    """Row-major 4x4 camera-to-world pose -> ctypes double[16]."""
    import numpy as np
    a = np.ascontiguousarray(np.asarray(pose, dtype=np.float64).reshape(16))
    return (C.c_double * 16)(*a.tolist())
