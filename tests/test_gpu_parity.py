"""GPU parity through the C ABI against the CPU oracle (FP32 reference
arithmetic) on seeded synthetic frames.

Tolerances (stated here, checked below):
  * allocated block sets: bit-exact (compared as sets; pool order differs)
  * TSDF / weight / colour: bit-exact in every voxel format
  * visible-block counts: exact
  * raycast: hit/miss disagreement <= 0.5 % of pixels; on pixels both hit,
    >= 99.5 % of vertices within 1 mm of the oracle's and mean |dz| <= 0.05 mm
    (the product skips unallocated blocks in one jump instead of the
    reference's 1-voxel steps, so its sample positions differ by float
    rounding only)
  * normals on a given vertex map: bit-exact
  * marching cubes: identical triangle multiset (vertices and normals
    bit-exact), triangle centroids bit-exact
  * Phong preview: within 1 of 255 per channel (powf differs by ulps)
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.common import aligned_maps, block_keys, fuse_both, make_pair, raycast_stats, sorted_rows, to_gpu_depth
from voxelmapping_b200 import _lib as L
from voxelmapping_b200 import synth

pytestmark = pytest.mark.gpu

SMALL = synth.WORKLOADS["room_small"]
FULL = synth.WORKLOADS["room_full"]


@pytest.fixture(scope="module")
def small_scene():
    return synth.Scene(SMALL)


@pytest.fixture(scope="module")
def full_scene():
    return synth.Scene(FULL)


def assert_maps_equal(vm, om, color=False):
    g, o = aligned_maps(vm, om)
    assert g["coords"].shape == o["coords"].shape, (g["coords"].shape, o["coords"].shape)
    assert np.array_equal(g["coords"], o["coords"])
    assert np.array_equal(g["tsdf"], o["tsdf"].astype(np.float32)), \
        "tsdf mismatch in %d voxels" % int((g["tsdf"] != o["tsdf"].astype(np.float32)).sum())
    assert np.array_equal(g["weight"], o["weight"].astype(np.float32))
    if color:
        assert np.array_equal(g["rgb"], o["rgb"])
    return g, o


# ---------------------------------------------------------------- allocation
def test_block_set_exact_small(small_scene):
    vm, om = make_pair(SMALL)
    for i in range(3):
        d, rgb, pose = small_scene.render(i)
        st, orc = fuse_both(vm, om, d, None, pose)
        assert st["allocated_blocks"] == om.num_blocks()
        assert st["visible_blocks"] == orc["visible"]
        assert st["error_flags"] == 0
    g = vm.export_blocks()
    assert set(block_keys(g["coords"]).tolist()) == set(block_keys(om.export()["coords"]).tolist())


def test_block_set_exact_full_size(full_scene):
    vm, om = make_pair(FULL, fmt="f32", color=True)
    d, rgb, pose = full_scene.render(0)
    st, orc = fuse_both(vm, om, d, rgb, pose)
    assert st["allocated_blocks"] == om.num_blocks() > 5000
    assert st["visible_blocks"] == orc["visible"]
    assert_maps_equal(vm, om, color=True)


def test_empty_and_invalid_depth():
    vm, om = make_pair(SMALL)
    pose = synth.Scene(SMALL).poses[0]
    zero = np.zeros((SMALL.height, SMALL.width), np.uint16)
    st, orc = fuse_both(vm, om, zero, None, pose)
    assert st["allocated_blocks"] == 0 and st["visible_blocks"] == 0 and orc["visible"] == 0
    # float depth with NaN, too near, too far: all invalid
    dm = np.full((SMALL.height, SMALL.width), np.nan, np.float32)
    dm[::2] = 0.05
    dm[1::4] = 7.0
    vm.FuseDepth(torch.from_numpy(dm).cuda(), pose)
    assert vm.stats()["allocated_blocks"] == 0
    v = vm.RenderScene(None, pose).cpu().numpy()
    assert np.isnan(v).all()
    assert vm.Polygonize()[0] == 0


def test_nan_depth_float_path(small_scene):
    vm, om = make_pair(SMALL)
    d, _, pose = small_scene.render(5)
    dm = synth.depth_to_metres(d)
    rng = np.random.default_rng(0)
    dm[rng.random(dm.shape) < 0.05] = np.nan
    vm.FuseDepth(torch.from_numpy(dm).cuda(), pose)
    om.fuse(dm, None, pose)
    assert_maps_equal(vm, om)


def test_ragged_image_size(small_scene):
    K = np.array([[181.3, 0, 97.2], [0, 179.9, 55.7], [0, 0, 1]])
    w, h = 203, 117
    vm, om = make_pair(SMALL, width=w, height=h, K=K)
    s = synth.Scene(synth.Workload("ragged", w, h, K[0, 0], K[1, 1], K[0, 2], K[1, 2], 10, 0, 0.008, 1 << 16,
                                   1 << 16, "ref", False))
    for i in range(2):
        d, _, pose = s.render(i)
        fuse_both(vm, om, d, None, pose)
    assert_maps_equal(vm, om)
    v_g = vm.RenderScene(None, pose).cpu().numpy()
    r = raycast_stats(v_g, om.raycast(pose))
    assert r["mismatch"] <= 0.005 and r["frac_within_1mm"] >= 0.995, r


def test_pool_exhaustion_reports_and_keeps_valid_subset(small_scene):
    cap = 1000
    vm, _ = make_pair(SMALL, num_blocks=cap)
    _, om = make_pair(SMALL)  # unlimited oracle
    d, _, pose = small_scene.render(0)
    st, _ = fuse_both(vm, om, d, None, pose)
    assert st["allocated_blocks"] == cap
    assert st["error_flags"] & L.FLAG_POOL_FULL and st["failed_allocs"] > 0
    g = vm.export_blocks()
    o = om.export()
    okeys = block_keys(o["coords"])
    idx = {k: i for i, k in enumerate(okeys.tolist())}
    sel = np.array([idx[k] for k in block_keys(g["coords"]).tolist()])  # GPU set is a subset
    # single frame: each block's voxels depend on that block only
    assert np.array_equal(g["tsdf"], o["tsdf"][sel].astype(np.float32))
    assert np.array_equal(g["weight"], o["weight"][sel].astype(np.float32))
    vm.clear_errors()
    assert vm.stats()["error_flags"] == 0


def test_hash_full_flag():
    vm, _ = make_pair(SMALL, num_buckets=2, num_entries=8)
    d, _, pose = synth.Scene(SMALL).render(0)
    vm.FuseDepth(to_gpu_depth(d), pose)
    st = vm.stats()
    assert st["error_flags"] & L.FLAG_HASH_FULL
    assert st["allocated_blocks"] == 8  # 2 buckets x 4 slots


def test_out_of_range_coordinates_flagged():
    vm, _ = make_pair(SMALL)
    s = synth.Scene(SMALL)
    d, _, pose = s.render(0)
    far = pose.copy()
    far[0, 3] += 1.0e5  # 100 km: block coordinates beyond +-2^20
    vm.FuseDepth(to_gpu_depth(d), far)
    st = vm.stats()
    assert st["error_flags"] & L.FLAG_RANGE and st["allocated_blocks"] == 0


# -------------------------------------------------------------------- fusion
@pytest.mark.parametrize("fmt,color,wmax", [("ref", False, 255), ("ref", True, 255), ("f32", True, 255),
                                            ("f16", True, 128), ("i16", False, 128), ("f32", False, 3)])
def test_tsdf_bit_exact(small_scene, fmt, color, wmax):
    vm, om = make_pair(SMALL, fmt=fmt, color=color, max_weight=wmax)
    for i in range(0, 12, 3):
        d, rgb, pose = small_scene.render(i)
        st, orc = fuse_both(vm, om, d, rgb if color else None, pose)
        assert st["visible_blocks"] == orc["visible"]
    g, o = assert_maps_equal(vm, om, color=color)
    assert g["weight"].max() == min(wmax, 4)


def test_fusion_properties_full_size(full_scene):
    """Size-independent properties at the full 640x480 / 2^20-block config."""
    vm, _ = make_pair(FULL, fmt="f32", color=True)
    d0, c0, p0 = full_scene.render(0)
    d1, c1, p1 = full_scene.render(40)
    vm.FuseDepth(to_gpu_depth(d0), p0)
    n0 = vm.stats()["allocated_blocks"]
    vm.FuseDepth(to_gpu_depth(d0), p0)  # same frame again: nothing new
    assert vm.stats()["allocated_blocks"] == n0
    vm.FuseDepth(to_gpu_depth(d1), p1)
    set_a = set(block_keys(vm.export_blocks(with_rgb=False)["coords"]).tolist())
    vm.reset()
    st = vm.stats()
    assert st["allocated_blocks"] == 0 and st["error_flags"] == 0
    assert np.isnan(vm.RenderScene(None, p0).cpu().numpy()).all()
    vm.FuseDepth(to_gpu_depth(d1), p1)  # reversed order: same block set
    vm.FuseDepth(to_gpu_depth(d0), p0)
    set_b = set(block_keys(vm.export_blocks(with_rgb=False)["coords"]).tolist())
    assert set_a == set_b


# ------------------------------------------------------------------- raycast
@pytest.mark.parametrize("mode", [0, 1])
def test_raycast_matches_oracle(small_scene, mode):
    vm, om = make_pair(SMALL, raycast_mode=mode)
    for i in range(0, 20, 2):
        d, _, pose = small_scene.render(i)
        fuse_both(vm, om, d, None, pose)
    for k, pose in enumerate([small_scene.poses[18], small_scene.poses[7], small_scene.poses[50]]):
        v_g = vm.RenderScene(None, pose).cpu().numpy()
        v_o = om.raycast(pose)
        r = raycast_stats(v_g, v_o)
        print("raycast mode", mode, "pose", k, r)
        assert r["hits_gpu"] > 0.5 * v_g.shape[0] * v_g.shape[1] or k == 2
        assert r["mismatch"] <= 0.005, r
        assert r["frac_within_1mm"] >= 0.995 and r["dz_mean_mm"] <= 0.05, r
        assert np.all(v_g[np.isfinite(v_g[..., 0])][:, 3] == 1.0)
        assert np.isnan(v_g[~np.isfinite(v_g[..., 0])]).all()


def test_raycast_full_size_vs_fp64(full_scene):
    """Full config: GPU depth against the FP64 oracle within 1 mm."""
    vm, _ = make_pair(FULL, fmt="f32", color=True)
    o64 = O.OracleMap(FULL.width, FULL.height, FULL.K, FULL.num_blocks, FULL.voxel_size, precision=O.FP64,
                      storage="f32", with_color=False)
    for i in range(0, 6):
        d, rgb, pose = full_scene.render(i)
        vm.FuseDepthAndImage(torch.from_numpy(rgb).cuda().reshape(FULL.height, -1), to_gpu_depth(d), pose)
        o64.fuse(synth.depth_to_metres(d), None, pose)
    v_g = vm.RenderScene(None, pose).cpu().numpy()
    v_o = o64.raycast(pose)
    r = raycast_stats(v_g, v_o)
    print("full-size raycast vs FP64", r)
    assert r["mismatch"] <= 0.01, r
    assert r["frac_within_1mm"] >= 0.99 and r["dz_mean_mm"] <= 0.1, r


def test_normals_bit_exact(small_scene):
    vm, om = make_pair(SMALL)
    for i in range(4):
        d, _, pose = small_scene.render(i)
        fuse_both(vm, om, d, None, pose)
    nmap = torch.empty((SMALL.height, SMALL.width, 4), dtype=torch.float32, device="cuda")
    vmap = vm.RenderScene(None, pose, nmap=nmap)
    v = vmap.cpu().numpy()
    n_g = nmap.cpu().numpy()
    n_o = O.compute_normal(v)
    assert np.array_equal(np.isnan(n_g), np.isnan(n_o))
    ok = ~np.isnan(n_o)
    assert np.array_equal(n_g[ok], n_o[ok])
    assert ok[..., 0].mean() > 0.5
    # Phong preview of the same maps
    rgba = torch.empty((SMALL.height, SMALL.width, 4), dtype=torch.uint8, device="cuda")
    L.check(L.lib().vmap_render_phong(vmap.data_ptr(), 0, nmap.data_ptr(), 0, rgba.data_ptr(), 0, SMALL.width,
                                      SMALL.height, torch.cuda.current_stream().cuda_stream))
    p_g = rgba.cpu().numpy().astype(int)
    p_o = O.render_phong(v, n_g).astype(int)
    assert np.abs(p_g - p_o).max() <= 1


# -------------------------------------------------------------- marching cubes
@pytest.mark.parametrize("fmt", ["ref", "f32", "f16"])
def test_mesh_bit_exact(small_scene, fmt):
    vm, om = make_pair(SMALL, fmt=fmt)
    for i in range(0, 9, 3):
        d, _, pose = small_scene.render(i)
        fuse_both(vm, om, d, None, pose)
    n_g, v_g, nn_g = vm.Polygonize()
    n_o, v_o, nn_o = om.polygonize()
    assert n_g == n_o > 1000
    a = sorted_rows(np.concatenate([v_g, nn_g], axis=1))
    b = sorted_rows(np.concatenate([v_o, nn_o], axis=1))
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    pts = vm.GetSurfacePoints()
    assert pts.shape == (n_g, 3)
    assert np.array_equal(sorted_rows(pts), sorted_rows(O.surface_points(v_o)))


def test_mesh_buffer_full_flag(small_scene):
    vm, om = make_pair(SMALL)
    d, _, pose = small_scene.render(0)
    fuse_both(vm, om, d, None, pose)
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    # a counting pass (no buffers) flags nothing
    L.check(L.lib().vmap_polygonize(vm._map, None, None, 0, cnt.data_ptr(), torch.cuda.current_stream().cuda_stream))
    assert vm.stats()["error_flags"] == 0 and int(cnt.item()) > 100
    verts = torch.empty((100, 9), dtype=torch.float32, device="cuda")
    norms = torch.empty((100, 9), dtype=torch.float32, device="cuda")
    L.check(L.lib().vmap_polygonize(vm._map, verts.data_ptr(), norms.data_ptr(), 100, cnt.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream))
    st = vm.stats()
    assert int(cnt.item()) == om.polygonize(max_tris=0)[0] > 100
    assert st["error_flags"] & L.FLAG_BUFFER_FULL
    # the 100 written triangles are genuine triangles of the full mesh
    _, v_o, _ = om.polygonize()
    full = {r.tobytes() for r in v_o}
    assert all(r.tobytes() in full for r in verts.cpu().numpy())


# ------------------------------------------------------------- host-buffer API
def test_host_buffer_entry_points(small_scene):
    vm, om = make_pair(SMALL, fmt="ref", color=True)
    d, rgb, pose = small_scene.render(2)
    vm.FuseDepthAndImage(rgb, d, pose)  # numpy -> vmap_fuse_host
    om.fuse(synth.depth_to_metres(d), rgb, pose)
    assert_maps_equal(vm, om, color=True)
    vh = np.empty((SMALL.height, SMALL.width, 4), np.float32)
    nh = np.empty_like(vh)
    L.check(L.lib().vmap_render_scene_host(vm._map, L.pose_arg(pose), vh.ctypes.data, nh.ctypes.data,
                                           torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    v_d = vm.RenderScene(None, pose).cpu().numpy()
    assert np.array_equal(np.nan_to_num(vh, nan=-7), np.nan_to_num(v_d, nan=-7))
    assert np.array_equal(np.nan_to_num(nh, nan=-7), np.nan_to_num(O.compute_normal(v_d), nan=-7))
