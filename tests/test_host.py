"""Host-side checks that need no GPU: the C ABI library loads and exports what
include/vmap_c.h declares, hash and pose math agree between library and
oracle, argument validation, and the synthetic scene generator."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from voxelmapping_b200 import _lib as L
from voxelmapping_b200 import synth

ROOT = Path(__file__).resolve().parent.parent


def declared(header):
    text = (ROOT / "include" / header).read_text()
    return sorted(set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(vmap_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    h = C.CDLL(str(L.LIB_PATH))
    names = declared("vmap_c.h")
    assert len(names) >= 20
    for n in names:
        assert hasattr(h, n), n
    assert set(names) <= set(L.SIGNATURES), set(names) - set(L.SIGNATURES)


def test_abi_basics():
    lib = L.lib()
    assert lib.vmap_abi_version() == 1
    assert lib.vmap_block_bytes(L.VOXEL_REF, 0) == 512 * 4
    assert lib.vmap_block_bytes(L.VOXEL_REF, 1) == 512 * 7
    assert lib.vmap_block_bytes(L.VOXEL_F32, 1) == 512 * 11
    assert lib.vmap_block_bytes(L.VOXEL_F16, 0) == 512 * 4
    assert lib.vmap_block_bytes(L.VOXEL_I16, 1) == 512 * 7
    assert lib.vmap_block_bytes(9, 0) == 0
    assert lib.vmap_status_string(4) == b"voxel-block pool full"


def test_create_rejects_bad_config_without_touching_the_gpu():
    lib = L.lib()
    h = C.c_void_p()
    base = dict(width=64, height=48, fx=50.0, fy=50.0, cx=32.0, cy=24.0, num_entries=0, num_blocks=1024,
                voxel_size=0.01, num_buckets=0, truncation=0.0, voxel_format=1, max_weight=0, with_color=0,
                raycast_mode=0)
    for bad in [dict(width=0), dict(num_blocks=0), dict(voxel_size=0.0), dict(voxel_format=7), dict(fx=-1.0),
                dict(max_weight=300, voxel_format=0), dict(raycast_mode=3), dict(num_entries=-1)]:
        cfg = L.Config(**{**base, **bad})
        assert lib.vmap_create(C.byref(cfg), C.byref(h)) == 1, bad
    assert lib.vmap_create(None, C.byref(h)) == 1
    assert lib.vmap_destroy(None) == 1
    assert lib.vmap_fuse_depth(None, None, 0, 0, 1.0, None, None) == 1


def int32_hash(x, y, z, nb):
    """hash (map_struct.h:104-109) with explicit int32 wrap-around."""
    w = lambda v: ((v + 2 ** 31) % 2 ** 32) - 2 ** 31
    r = w(w(x * 73856093) ^ w(y * 19349669) ^ w(z * 83492791))
    r = (abs(r) % nb) * (1 if r >= 0 else -1)  # C remainder: sign of the dividend
    return r + nb if r < 0 else r


def test_hash_library_oracle_and_restatement_agree():
    rng = np.random.default_rng(0)
    lib = L.lib()
    pts = [(0, 0, 0), (-1, -1, -1), (2 ** 20 - 1, -(2 ** 20), 7), (12345, -54321, 999)]
    pts += [tuple(int(v) for v in rng.integers(-(2 ** 20), 2 ** 20, 3)) for _ in range(2000)]
    for nb in (943718, 235929, 1, 7, 2 ** 20):
        for p in pts:
            a = lib.vmap_block_hash(*p, nb)
            assert a == O.block_hash(*p, nb) == int32_hash(*p, nb)
            assert 0 <= a < nb


def test_pose_inverse_bitwise_equal_to_oracle():
    rng = np.random.default_rng(1)
    lib = L.lib()
    for _ in range(200):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                      [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                      [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        P = np.eye(4)
        P[:3, :3] = R * rng.uniform(0.5, 2.0)
        P[:3, 3] = rng.normal(size=3) * 3
        out = (C.c_double * 16)()
        lib.vmap_pose_inverse(L.pose_arg(P), out)
        a = np.array(out[:]).reshape(4, 4)
        b = O.pose_inverse(P)
        assert np.array_equal(a, b)
        assert np.allclose(a @ P, np.eye(4), atol=1e-9)


def test_synthetic_scene_is_deterministic_and_plausible():
    wl = synth.WORKLOADS["room_small"]
    s1, s2 = synth.Scene(wl), synth.Scene(wl)
    d1, c1, p1, t1 = s1.render(3, want_true=True)
    d2, c2, p2 = s2.render(3)
    assert np.array_equal(d1, d2) and np.array_equal(c1, c2) and np.array_equal(p1, p2)
    assert not np.array_equal(d1, s1.render(4)[0])
    drop = (d1 == 0).mean()
    assert 0.01 < drop < 0.03
    ok = d1 > 0
    z = t1[ok]
    err = d1[ok] / 1000.0 - z
    sigma = 0.0012 + 0.0019 * (z - 0.4) ** 2
    assert abs(np.mean(err / sigma)) < 0.05 and 0.9 < np.std(err / sigma) < 1.1
    assert 0.3 < z.min() and z.max() < 4.0
    # poses are rigid, camera z axis looks at the room centre on the circle
    for P in s1.poses[::10]:
        R = P[:3, :3]
        assert np.allclose(R @ R.T, np.eye(3), atol=1e-12)
        to_c = np.array([0, 0, 1.5]) - P[:3, 3]
        assert np.allclose(R[:, 2], to_c / np.linalg.norm(to_c))


def test_figure8_trajectory_keeps_clear_of_spheres():
    wl = synth.WORKLOADS["room_full"]
    s = synth.Scene(wl)
    sp = s.spheres()
    for P in s.poses:
        d = np.linalg.norm(sp[:, :3] - P[:3, 3], axis=1) - sp[:, 3]
        assert d.min() > 0.1


def test_static_export_source_allocates_nothing():
    """The no-allocation export calls no allocating or freeing routine."""
    src = (Path(__file__).resolve().parent.parent / "voxelmapping_b200" / "csrc" / "export_static.cu").read_text()
    code = "\n".join(l.split("//")[0] for l in src.splitlines())
    for name in ("cudaMalloc", "cudaMallocAsync", "cudaMallocHost", "cudaHostAlloc", "cudaMallocManaged", "cudaFree",
                 "malloc(", "new "):
        assert name not in code, name
