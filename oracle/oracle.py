"""ctypes wrapper of the CPU oracle (libvmap_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU
baseline leg of bench.py, never by the product. See vmap_oracle.h for what it
restates and how far parity is pinned.
"""
import ctypes as C
import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libvmap_oracle.so"
GOLDEN = HERE.parent / "tests" / "golden"

FP32, FP64 = 0, 1
STORE = {"ref": 0, "f32": 1, "f16": 2, "i16": 3}


class OrcConfig(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("fx", C.c_float), ("fy", C.c_float),
                ("cx", C.c_float), ("cy", C.c_float), ("num_blocks", C.c_int), ("voxel_size", C.c_float),
                ("truncation", C.c_float), ("precision", C.c_int), ("storage", C.c_int),
                ("max_weight", C.c_int), ("with_color", C.c_int)]


_lib = None
_tables = False
D16 = C.POINTER(C.c_double)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError("oracle not built: make -C oracle")
        h = C.CDLL(str(LIB_PATH))
        sig = {
            "orc_set_mc_tables": (None, [C.POINTER(C.c_int)]),
            "orc_create": (C.c_void_p, [C.POINTER(OrcConfig)]),
            "orc_destroy": (None, [C.c_void_p]),
            "orc_reset": (None, [C.c_void_p]),
            "orc_set_threads": (None, [C.c_int]),
            "orc_get_threads": (C.c_int, []),
            "orc_fuse": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, D16, C.POINTER(C.c_int),
                                   C.POINTER(C.c_int)]),
            "orc_allocate": (C.c_int, [C.c_void_p, C.c_void_p, D16, C.POINTER(C.c_int)]),
            "orc_raycast": (C.c_int, [C.c_void_p, D16, C.c_void_p]),
            "orc_compute_normal": (None, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
            "orc_render_phong": (None, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
            "orc_polygonize": (C.c_long, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_long]),
            "orc_surface_points": (None, [C.c_void_p, C.c_long, C.c_void_p]),
            "orc_num_blocks": (C.c_int, [C.c_void_p]),
            "orc_last_raycast_blocks": (C.c_int, [C.c_void_p]),
            "orc_last_alloc_blocks": (C.c_int, [C.c_void_p]),
            "orc_probe": (None, [C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
            "orc_export": (None, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
            "orc_hash": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int]),
            "orc_pose_inverse": (None, [D16, D16]),
            "orc_constants": (None, [C.POINTER(C.c_int)]),
        }
        for k, (r, a) in sig.items():
            f = getattr(h, k)
            f.restype, f.argtypes = r, a
        _lib = h
    return _lib


def load_tables():
    global _tables
    if not _tables:
        tri = np.asarray(json.loads((GOLDEN / "mc_tables.json").read_text())["triTable"], dtype=np.int32)
        lib().orc_set_mc_tables(np.ascontiguousarray(tri).ctypes.data_as(C.POINTER(C.c_int)))
        _tables = True


def _pose(p):
    a = np.ascontiguousarray(np.asarray(p, np.float64).reshape(16))
    return a, a.ctypes.data_as(D16)


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class OracleMap:
    def __init__(self, width, height, K, num_blocks, voxel_size, truncation=None, precision=FP32,
                 storage="ref", max_weight=255, with_color=False):
        K = np.asarray(K, np.float64)
        self.width, self.height, self.with_color = width, height, with_color
        cfg = OrcConfig(width, height, K[0, 0], K[1, 1], K[0, 2], K[1, 2], num_blocks, voxel_size,
                        np.float32(voxel_size) * np.float32(4) if truncation is None else truncation,
                        precision, STORE[storage], max_weight, int(with_color))
        self._h = lib().orc_create(C.byref(cfg))
        if not self._h:
            raise ValueError("bad oracle config")

    def __del__(self):
        try:
            lib().orc_destroy(self._h)
        except Exception:
            pass

    def reset(self):
        lib().orc_reset(self._h)

    def fuse(self, depth_m, rgb, pose):
        d = np.ascontiguousarray(depth_m, np.float32)
        c = np.ascontiguousarray(rgb, np.uint8) if rgb is not None else None
        _, pp = _pose(pose)
        nn, nf = C.c_int(), C.c_int()
        nvis = lib().orc_fuse(self._h, _ptr(d), _ptr(c), pp, C.byref(nn), C.byref(nf))
        return {"visible": nvis, "new": nn.value, "failed": nf.value}

    def allocate(self, depth_m, pose):
        d = np.ascontiguousarray(depth_m, np.float32)
        _, pp = _pose(pose)
        nf = C.c_int()
        n = lib().orc_allocate(self._h, _ptr(d), pp, C.byref(nf))
        return n, nf.value

    def raycast(self, pose):
        v = np.empty((self.height, self.width, 4), np.float32)
        _, pp = _pose(pose)
        lib().orc_raycast(self._h, pp, _ptr(v))
        return v

    def num_blocks(self):
        return lib().orc_num_blocks(self._h)

    def last_alloc_blocks(self):
        """Unique blocks the last fused frame's allocation touched (its A)."""
        return lib().orc_last_alloc_blocks(self._h)

    def last_raycast_blocks(self):
        """Unique allocated blocks the last raycast read (its U)."""
        return lib().orc_last_raycast_blocks(self._h)

    def export(self):
        n = self.num_blocks()
        coords = np.zeros((n, 3), np.int32)
        tsdf = np.zeros((n, 512), np.float64)
        w = np.zeros((n, 512), np.float64)
        rgb = np.zeros((n, 512, 3), np.uint8) if self.with_color else None
        lib().orc_export(self._h, _ptr(coords), _ptr(tsdf), _ptr(w), _ptr(rgb))
        return {"coords": coords, "tsdf": tsdf, "weight": w, "rgb": rgb}

    def polygonize(self, max_tris=None):
        load_tables()
        n = lib().orc_polygonize(self._h, None, None, 0)
        k = n if max_tris is None else min(n, max_tris)
        v = np.zeros((k, 9), np.float32)
        nm = np.zeros((k, 9), np.float32)
        lib().orc_polygonize(self._h, _ptr(v), _ptr(nm), k)
        return n, v, nm


def compute_normal(vmap):
    v = np.ascontiguousarray(vmap, np.float32)
    h, w = v.shape[:2]
    n = np.empty_like(v)
    lib().orc_compute_normal(_ptr(v), w, h, _ptr(n))
    return n


def render_phong(vmap, nmap):
    v = np.ascontiguousarray(vmap, np.float32)
    n = np.ascontiguousarray(nmap, np.float32)
    h, w = v.shape[:2]
    out = np.empty((h, w, 4), np.uint8)
    lib().orc_render_phong(_ptr(v), _ptr(n), w, h, _ptr(out))
    return out


def surface_points(verts):
    v = np.ascontiguousarray(verts, np.float32)
    out = np.empty((v.shape[0], 3), np.float32)
    lib().orc_surface_points(_ptr(v), v.shape[0], _ptr(out))
    return out


def probe(which, inputs):
    """The reference build's arithmetic probe shape `which` (an index of
    oracle.refbuild.PROBES) on each row of `inputs` (n, <=20) float32,
    through the oracle's FP32 helpers; returns (n, 4) float32."""
    x = np.zeros((len(inputs), 20), np.float32)
    x[:, :inputs.shape[1]] = inputs
    out = np.empty((len(inputs), 4), np.float32)
    lib().orc_probe(int(which), _ptr(x), len(inputs), _ptr(out))
    return out


def set_threads(n):
    lib().orc_set_threads(int(n))


def get_threads():
    return lib().orc_get_threads()


def block_hash(x, y, z, nb):
    return lib().orc_hash(x, y, z, nb)


def pose_inverse(p):
    a, pp = _pose(p)
    out = np.zeros(16, np.float64)
    lib().orc_pose_inverse(pp, out.ctypes.data_as(D16))
    return out.reshape(4, 4)


def constants():
    out = (C.c_int * 9)()
    lib().orc_constants(out)
    keys = ["block", "min_depth_mm", "max_depth_mm", "trunc_factor", "weight_cap", "p0", "p1", "p2", "subsample"]
    return dict(zip(keys, list(out)))
