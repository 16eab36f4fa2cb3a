"""Synthetic RGB-D sequences (ctypes over libvmap_synth.so) and the workload
definitions the tests and the benchmark use.

Workloads (seeded, no external data):
  room_small : 320x240, f 262.5, c (159.5, 119.5), 100 poses on a 1 m circle at
               1.5 m looking at the room centre; 8 mm voxels, 2^20 entries,
               2^18 blocks; reference voxel format (int16 TSDF, uint8 weight).
  room_full  : 640x480, f 525, c (319.5, 239.5), 500 poses on a figure-8;
               5 mm voxels, 2^21 entries, 2^20 blocks; FP32 TSDF + float
               weight + uint8x3 colour.
  uneven_workloads(n): n maps of uneven extent, voxel size and resolution.
Scene: 4 x 4 x 3 m box room seen from inside + 8 spheres, radius U(0.1, 0.5) m;
depth uint16 mm with N(0, 0.0012 + 0.0019 (z - 0.4)^2) m noise and 2 % dropouts.
"""
import ctypes as C
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
SYNTH_PATH = _PKG / "libvmap_synth.so"
TRAJ_CIRCLE, TRAJ_FIGURE8 = 0, 1


class SceneDesc(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("size", C.c_double * 3), ("n_spheres", C.c_int),
                ("cam_radius", C.c_double), ("cam_height", C.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not SYNTH_PATH.exists():
            raise ImportError("%s missing: run `python -m voxelmapping_b200.build`" % SYNTH_PATH)
        h = C.CDLL(str(SYNTH_PATH))
        h.vmap_synth_scene_create.argtypes = [C.POINTER(SceneDesc), C.POINTER(C.c_void_p)]
        h.vmap_synth_scene_create.restype = C.c_int
        h.vmap_synth_scene_destroy.argtypes = [C.c_void_p]
        h.vmap_synth_scene_destroy.restype = None
        h.vmap_synth_scene_spheres.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        h.vmap_synth_scene_spheres.restype = C.c_int
        h.vmap_synth_trajectory.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_double)]
        h.vmap_synth_trajectory.restype = C.c_int
        h.vmap_synth_render.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_int, C.c_double, C.c_double,
                                        C.c_double, C.c_double, C.c_uint64, C.c_int, C.c_double, C.c_void_p,
                                        C.c_void_p, C.c_void_p]
        h.vmap_synth_render.restype = C.c_int
        _lib = h
    return _lib


@dataclass
class Workload:
    name: str
    width: int
    height: int
    fx: float
    fy: float
    cx: float
    cy: float
    n_poses: int
    trajectory: int
    voxel_size: float
    num_entries: int
    num_blocks: int
    voxel_format: str
    with_color: bool
    max_weight: int = 255
    room: tuple = (4.0, 4.0, 3.0)
    n_spheres: int = 8
    cam_radius: float = 1.0
    cam_height: float = 1.5
    seed: int = 0
    noisy: bool = True
    dropout: float = 0.02
    depth_scale: float = 0.001
    extra: dict = field(default_factory=dict)

    @property
    def K(self):
        return np.array([[self.fx, 0, self.cx], [0, self.fy, self.cy], [0, 0, 1]], np.float64)


WORKLOADS = {
    "room_small": Workload("room_small", 320, 240, 262.5, 262.5, 159.5, 119.5, 100, TRAJ_CIRCLE, 0.008,
                           1 << 20, 1 << 18, "ref", False),
    "room_full": Workload("room_full", 640, 480, 525.0, 525.0, 319.5, 239.5, 500, TRAJ_FIGURE8, 0.005,
                          1 << 21, 1 << 20, "f32", True),
}


RESOLUTIONS = ((320, 240), (640, 480), (1280, 720))
VOXEL_SIZES = (0.004, 0.008, 0.012, 0.016)


def uneven_workloads(n, seed=0, voxel_format="f16", with_color=True):
    """n independent map workloads of uneven size (the batching / serving mix):
    room extent U(1, 8) m, voxel size from {4, 8, 12, 16} mm, depth resolution
    from {320x240, 640x480, 1280x720} (focal length 0.82 x width, principal
    point at the centre), each its own seeded scene and trajectory. The pool
    is the power of two (clamped to 2^14 .. 2^19 blocks) above 1.5x the
    room's surface area in block faces."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        e = float(rng.uniform(1.0, 8.0))
        room = (e, e * float(rng.uniform(0.6, 1.0)), min(3.0, max(1.0, 0.6 * e)))
        vs = float(VOXEL_SIZES[rng.integers(len(VOXEL_SIZES))])
        w, h = RESOLUTIONS[rng.integers(len(RESOLUTIONS))]
        f = 0.8203125 * w
        area = 2.0 * (room[0] * room[1] + room[0] * room[2] + room[1] * room[2])
        est = 1.5 * area / (8 * vs) ** 2
        blocks = 1 << int(min(19, max(14, int(np.ceil(np.log2(est))))))
        out.append(Workload("uneven%d" % i, w, h, f, f, (w - 1) / 2.0, (h - 1) / 2.0, 100,
                            TRAJ_FIGURE8 if i % 2 else TRAJ_CIRCLE, vs, 4 * blocks, blocks, voxel_format,
                            with_color, max_weight=128, room=room,
                            cam_radius=0.25 * min(room[0], room[1]), cam_height=0.5 * room[2],
                            seed=int(seed) * 100003 + 17 + i))
    return out


class Scene:
    """A seeded room scene with a trajectory; renders frames on demand."""

    def __init__(self, wl: Workload):
        self.wl = wl
        d = SceneDesc(wl.seed, (C.c_double * 3)(*wl.room), wl.n_spheres, wl.cam_radius, wl.cam_height)
        h = C.c_void_p()
        if lib().vmap_synth_scene_create(C.byref(d), C.byref(h)) != 0:
            raise ValueError("bad scene description")
        self._h = h
        self.poses = np.zeros((wl.n_poses, 4, 4), np.float64)
        lib().vmap_synth_trajectory(wl.trajectory, wl.n_poses, wl.cam_radius, wl.cam_height,
                                    self.poses.ctypes.data_as(C.POINTER(C.c_double)))

    def __del__(self):
        try:
            lib().vmap_synth_scene_destroy(self._h)
        except Exception:
            pass

    def spheres(self):
        out = np.zeros((16, 4), np.float64)
        n = lib().vmap_synth_scene_spheres(self._h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out[:n]

    def render(self, i, noisy=None, dropout=None, want_true=False):
        """Frame i: (depth uint16 mm (h, w), rgb uint8 (h, w, 3), pose (4, 4)[, true depth float32])."""
        wl = self.wl
        pose = np.ascontiguousarray(self.poses[i % wl.n_poses])
        depth = np.zeros((wl.height, wl.width), np.uint16)
        rgb = np.zeros((wl.height, wl.width, 3), np.uint8)
        true = np.zeros((wl.height, wl.width), np.float32) if want_true else None
        lib().vmap_synth_render(self._h, pose.ctypes.data_as(C.POINTER(C.c_double)), wl.width, wl.height,
                                wl.fx, wl.fy, wl.cx, wl.cy, i, int(wl.noisy if noisy is None else noisy),
                                wl.dropout if dropout is None else dropout, depth.ctypes.data_as(C.c_void_p),
                                rgb.ctypes.data_as(C.c_void_p),
                                true.ctypes.data_as(C.c_void_p) if true is not None else None)
        if want_true:
            return depth, rgb, pose, true
        return depth, rgb, pose


def depth_to_metres(depth_u16, scale=0.001):
    """The library's uint16 -> metres conversion: float32(d) * float32(scale)."""
    return depth_u16.astype(np.float32) * np.float32(scale)
