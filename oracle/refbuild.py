"""ctypes binding of the reference's own CUDA build (oracle/_ref/libvmap_ref.so).

TEST INFRASTRUCTURE ONLY: the reference's src/*.cu compiled unchanged against
the Eigen/OpenCV subsets in oracle/ref_shim/ (recipe: `make -C oracle ref`,
harness: oracle/ref_harness.cu). Imported by tests/ and by bench.py's
reference arm, never by the product. Device buffers are torch tensors.
"""
import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libvmap_ref.so"

# include/map_struct.h:17-42 (HashEntry 20 B; Voxel 4 B with one pad byte;
# VoxelRGB 6 B)
HASH_DT = np.dtype([("ptr", "<i4"), ("offset", "<i4"), ("pos", "<i4", (3,))])
VOXEL_DT = np.dtype([("sdf", "<i2"), ("wt", "u1"), ("pad", "u1")])
VOXEL_RGB_DT = np.dtype([("sdf", "<i2"), ("wt", "u1"), ("rgb", "u1", (3,))])

SYMBOLS = {
    "ref_last_error": (C.c_char_p, []),
    "ref_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_float), C.c_int, C.c_int, C.c_float, C.c_int,
                             C.POINTER(C.c_void_p)]),
    "ref_destroy": (None, [C.c_void_p]),
    "ref_reset": (C.c_int, [C.c_void_p]),
    "ref_fuse": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.POINTER(C.c_float), C.c_int,
                           C.POINTER(C.c_int)]),
    "ref_render": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_float)]),
    "ref_compute_normal": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_int, C.c_int]),
    "ref_render_phong": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_int,
                                   C.c_int]),
    "ref_polygonize": (C.c_long, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.POINTER(C.c_uint)]),
    "ref_surface_points": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint]),
    "ref_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "ref_copy_map": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "ref_probe": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "ref_sync": (C.c_int, []),
}

_lib = None


def available():
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError("reference build missing: make -C oracle ref (needs the reference sources)")
        h = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SYMBOLS.items():
            f = getattr(h, name)
            f.restype, f.argtypes = res, args
        _lib = h
    return _lib


def _check(rc, what):
    if rc < 0:
        raise RuntimeError("%s: %s" % (what, lib().ref_last_error().decode()))
    return rc


def _mat(a, n):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(n))
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


def hash_bucket(coords, n_bucket):
    """The reference's bucket function (include/map_struct.h:104-109) with
    int32 wrap-around, vectorised."""
    c = np.asarray(coords, dtype=np.int64)
    primes = np.array([73856093, 19349669, 83492791], dtype=np.int64)
    p = (c * primes) & 0xFFFFFFFF
    p = np.where(p >= 1 << 31, p - (1 << 32), p).astype(np.int32)
    h = (p[..., 0] ^ p[..., 1] ^ p[..., 2]).astype(np.int64)
    r = np.fmod(h, n_bucket)
    return np.where(r < 0, r + n_bucket, r)


class RefMap:
    """One map of the reference build: VoxelMapping's CreateMap / FuseDepth /
    FuseDepthAndImage / RenderScene / Polygonize (src/vmapping.cpp), with the
    harness changes stated in oracle/ref_harness.cu."""

    def __init__(self, width, height, K, num_entries, num_voxels, voxel_size, with_color=False):
        self.width, self.height, self.with_color = width, height, with_color
        self._K, kp = _mat(K, 9)
        h = C.c_void_p()
        _check(lib().ref_create(width, height, kp, num_entries, num_voxels, voxel_size, int(with_color), C.byref(h)),
               "ref_create")
        self._h = h

    def close(self):
        if self._h:
            lib().ref_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self):
        _check(lib().ref_reset(self._h), "ref_reset")

    def fuse(self, depth, pose, rgb=None, complete=False):
        """depth: cuda float32 (H, W) metres; rgb: cuda uint8 (H, W, 3) or
        None; pose: camera-to-world 4x4 (rounded to float32). Returns
        (visible blocks, extra allocation passes)."""
        _, pp = _mat(pose, 16)
        passes = C.c_int(0)
        vis = lib().ref_fuse(self._h, depth.data_ptr(), depth.stride(0) * 4,
                             rgb.data_ptr() if rgb is not None else None,
                             rgb.stride(0) if rgb is not None else 0, pp, int(complete), C.byref(passes))
        return _check(vis, "ref_fuse"), passes.value

    def render(self, pose, out=None):
        """Vertex map (H, W, 4) float32 at the pose, NaN where the reference
        writes nothing; synchronised."""
        import torch
        if out is None:
            out = torch.full((self.height, self.width, 4), float("nan"), dtype=torch.float32, device="cuda")
        else:
            out.fill_(float("nan"))
        _, pp = _mat(pose, 16)
        torch.cuda.synchronize()
        _check(lib().ref_render(self._h, out.data_ptr(), self.width * 16, pp), "ref_render")
        _check(lib().ref_sync(), "ref_sync")
        return out

    def info(self):
        a = (C.c_int * 7)()
        _check(lib().ref_info(self._h, a), "ref_info")
        keys = ("entries", "buckets", "pool_blocks", "allocated", "excess_used", "hash_entry_bytes", "voxel_bytes")
        return dict(zip(keys, list(a)))

    def polygonize(self, max_tris):
        """(triangle count, vertices (n, 9), face normals (n, 9), blocks)."""
        import torch
        v = torch.empty((max(max_tris, 1), 9), dtype=torch.float32, device="cuda")
        n = torch.empty_like(v)
        blocks = C.c_uint(0)
        cnt = _check(lib().ref_polygonize(self._h, v.data_ptr(), n.data_ptr(), max_tris, C.byref(blocks)),
                     "ref_polygonize")
        return cnt, v[:cnt].cpu().numpy(), n[:cnt].cpu().numpy(), blocks.value

    def export(self):
        """Every live hash entry (ptr >= 0), duplicates included, with its
        block's voxels: coords (n, 3) int32, tsdf (n, 512) float32
        (= code / 32767, unpackFloat), weight (n, 512) float32, rgb
        (n, 512, 3) uint8 or None, and 'codes' (n, 512) int16."""
        inf = self.info()
        table = np.empty(inf["entries"], HASH_DT)
        dt = VOXEL_RGB_DT if self.with_color else VOXEL_DT
        assert dt.itemsize == inf["voxel_bytes"] and HASH_DT.itemsize == inf["hash_entry_bytes"]
        nb = max(inf["allocated"], 0)
        pool = np.empty(max(nb, 1) * 512, dt)
        _check(lib().ref_copy_map(self._h, table.ctypes.data, pool.ctypes.data, nb), "ref_copy_map")
        live = table[table["ptr"] >= 0]
        blk = live["ptr"] // 512
        assert (live["ptr"] % 512 == 0).all() and (blk < max(nb, 1)).all()
        vox = pool.reshape(-1, 512)[blk] if nb else pool[:0].reshape(0, 512)
        codes = vox["sdf"].astype(np.int16)
        return {"coords": live["pos"].astype(np.int32), "codes": codes,
                "tsdf": codes.astype(np.float32) / np.float32(32767.0),
                "weight": vox["wt"].astype(np.float32),
                "rgb": vox["rgb"].copy() if self.with_color else None}


def compute_normal(vmap, nmap=None):
    """computeNormal (src/image_proc.cu:74-104) on a cuda (H, W, 4) vertex
    map; entries it leaves unwritten (last row and column) are NaN."""
    import torch
    h, w = vmap.shape[:2]
    if nmap is None:
        nmap = torch.full_like(vmap, float("nan"))
    _check(lib().ref_compute_normal(vmap.data_ptr(), w * 16, nmap.data_ptr(), w * 16, w, h), "ref_compute_normal")
    _check(lib().ref_sync(), "ref_sync")
    return nmap


def render_phong(vmap, nmap):
    import torch
    h, w = vmap.shape[:2]
    img = torch.zeros((h, w, 4), dtype=torch.uint8, device="cuda")
    _check(lib().ref_render_phong(vmap.data_ptr(), w * 16, nmap.data_ptr(), w * 16, img.data_ptr(), w * 4, w, h),
           "ref_render_phong")
    _check(lib().ref_sync(), "ref_sync")
    return img


PROBES = {"xform": 0, "unproject_world": 1, "project": 2, "squared_norm": 3, "norm": 4, "normalized": 5,
          "cross": 6, "dot": 7, "lerp": 8, "running_average": 9, "rgb_blend": 10, "ray_step": 11, "phong": 12,
          "mc_interp": 13}


def probe(name, inputs):
    """Evaluate one of the reference's expression shapes (PROBES) on the GPU
    for each row of `inputs` (n, <=20) float32; returns (n, 4) float32."""
    import torch
    x = np.zeros((len(inputs), 20), np.float32)
    x[:, :inputs.shape[1]] = inputs
    xi = torch.from_numpy(x).cuda()
    out = torch.full((len(inputs), 4), float("nan"), dtype=torch.float32, device="cuda")
    _check(lib().ref_probe(PROBES[name], xi.data_ptr(), len(inputs), out.data_ptr()), "ref_probe")
    return out.cpu().numpy()
