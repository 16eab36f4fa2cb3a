"""Whole configurations through the C ABI against the CPU oracle.

room_small (320x240, 8 mm, 2^20 entries, 2^18 blocks, reference voxel
format): fuse all 100 frames, comparing the maps every 25 frames, then
raycast at the last pose and extract the mesh.
room_full (640x480, 5 mm, 2^21 entries, 2^20 blocks, FP32 TSDF + float
weight + colour): 100 frames, maps compared every 25 frames against the FP32
oracle; at the end raycast depth and the mesh against the FP64 oracle.

Bars (stated here, checked below):
  * block sets, TSDF, weight and colour: bit-exact against the FP32 oracle
    at every checkpoint
  * raycast against the FP32 oracle: hit/miss disagreement <= 0.5 %,
    >= 99.5 % of common hits within 1 mm (both march modes)
  * normals on the rendered vertex map: bit-exact
  * mesh against the FP32 oracle: identical triangle multiset
  * room_full against FP64: raycast hit/miss disagreement <= 1 %, >= 99.9 %
    within 1 mm and |dz| <= 1 mm at the 99.9th percentile, with no more pixels
    beyond 1 mm than the FP32 oracle (the reference arithmetic) has against
    FP64, + 0.02 % of the hits; mesh symmetric Hausdorff 99th percentile
    < 0.5 mm
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.common import aligned_maps, fuse_both, make_pair, raycast_stats, sorted_rows
from voxelmapping_b200 import synth

pytestmark = pytest.mark.gpu

SMALL = synth.WORKLOADS["room_small"]
FULL = synth.WORKLOADS["room_full"]


def assert_equal_maps(vm, om, color):
    g, o = aligned_maps(vm, om)
    assert np.array_equal(g["coords"], o["coords"]), (len(g["coords"]), len(o["coords"]))
    bad = g["tsdf"] != o["tsdf"].astype(np.float32)
    assert not bad.any(), "tsdf differs in %d voxels" % int(bad.sum())
    assert np.array_equal(g["weight"], o["weight"].astype(np.float32))
    if color:
        assert np.array_equal(g["rgb"], o["rgb"])
    return g


def test_room_small_all_frames_raycast_and_mesh():
    scene = synth.Scene(SMALL)
    vm, om = make_pair(SMALL, fmt="ref", raycast_mode=0)
    vm1, _ = make_pair(SMALL, fmt="ref", raycast_mode=1)
    for i in range(SMALL.n_poses):
        d, _, pose = scene.render(i)
        st, orc = fuse_both(vm, om, d, None, pose)
        assert st["visible_blocks"] == orc["visible"] and st["error_flags"] == 0
        vm1.FuseDepth(torch.from_numpy(np.ascontiguousarray(d).view(np.int16)).cuda(), pose)
        if i % 25 == 24:
            assert_equal_maps(vm, om, False)
    v_o = om.raycast(pose)
    for m in (vm, vm1):
        nmap = torch.empty((SMALL.height, SMALL.width, 4), dtype=torch.float32, device="cuda")
        vmap = m.RenderScene(None, pose, nmap=nmap)
        v = vmap.cpu().numpy()
        r = raycast_stats(v, v_o)
        print("room_small frame 99 raycast vs FP32 oracle", r)
        assert r["mismatch"] <= 0.005 and r["frac_within_1mm"] >= 0.995, r
        n_o = O.compute_normal(v)
        n_g = nmap.cpu().numpy()
        assert np.array_equal(np.isnan(n_g), np.isnan(n_o))
        ok = ~np.isnan(n_o)
        assert np.array_equal(n_g[ok], n_o[ok])
    n_g, v_g, nn_g = vm.Polygonize()
    n_o, v_oo, nn_o = om.polygonize()
    print("room_small mesh: %d triangles" % n_g)
    assert n_g == n_o > 10000
    a = sorted_rows(np.concatenate([v_g, nn_g], axis=1))
    b = sorted_rows(np.concatenate([v_oo, nn_o], axis=1))
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_room_full_100_frames_full_pool():
    from scipy.spatial import cKDTree
    scene = synth.Scene(FULL)
    vm, om = make_pair(FULL, fmt="f32", color=True)
    o64 = O.OracleMap(FULL.width, FULL.height, FULL.K, FULL.num_blocks, FULL.voxel_size, precision=O.FP64,
                      storage="f32", with_color=False)
    for i in range(100):
        d, rgb, pose = scene.render(i)
        st, orc = fuse_both(vm, om, d, rgb, pose)
        assert st["visible_blocks"] == orc["visible"] and st["error_flags"] == 0
        o64.fuse(synth.depth_to_metres(d), None, pose)
        if i % 25 == 24:
            g = assert_equal_maps(vm, om, True)
    assert len(g["coords"]) > 15000
    # raycast against FP64, beside the FP32 oracle's own distance from FP64
    v = vm.RenderScene(None, pose).cpu().numpy()
    v64 = o64.raycast(pose)
    r = raycast_stats(v, v64)
    v32 = om.raycast(pose)
    b32 = np.isfinite(v32[..., 0]) & np.isfinite(v64[..., 0])
    over32 = int((np.abs(v32[..., 2] - v64[..., 2])[b32] > 1e-3).sum())
    both = np.isfinite(v[..., 0]) & np.isfinite(v64[..., 0])
    over = int((np.abs(v[..., 2] - v64[..., 2])[both] > 1e-3).sum())
    print("room_full frame 99 raycast vs FP64", r, "pixels beyond 1 mm: library %d, FP32 oracle %d" % (over, over32))
    assert r["mismatch"] <= 0.01 and r["frac_within_1mm"] >= 0.999 and r["dz_p999_mm"] <= 1.0, r
    assert over <= 2 * over32 + 2e-4 * both.sum()
    # mesh against FP64
    n_g, v_g, _ = vm.Polygonize()
    _, v_64, _ = o64.polygonize()
    a = np.unique(v_g.reshape(-1, 3), axis=0)
    b = np.unique(v_64.reshape(-1, 3), axis=0)
    d_ab = cKDTree(b).query(a, workers=-1)[0]
    d_ba = cKDTree(a).query(b, workers=-1)[0]
    p99 = float(np.percentile(np.concatenate([d_ab, d_ba]), 99)) * 1e3
    print("room_full mesh: %d triangles, Hausdorff vs FP64 p99 %.4f mm, max %.2f mm" %
          (n_g, p99, 1e3 * max(d_ab.max(), d_ba.max())))
    assert p99 < 0.5
