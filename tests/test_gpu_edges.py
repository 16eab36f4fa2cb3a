"""Edge cases against the oracle: an empty map through every stage, the
largest image size of the uneven mix (1280x720) at the finest voxel size
(4 mm), and ray marching in every storage format against the FP32 oracle with
the same storage (same tolerances as tests/test_gpu_parity.py)."""
import dataclasses

import numpy as np
import pytest
import torch

from tests.common import aligned_maps, fuse_both, make_pair, raycast_stats, sorted_rows
from voxelmapping_b200 import MapBatch, VoxelMapping
from voxelmapping_b200 import synth

pytestmark = pytest.mark.gpu
SMALL = synth.WORKLOADS["room_small"]


def test_empty_map_through_every_stage():
    vm = VoxelMapping(SMALL.width, SMALL.height, SMALL.K, voxel_format="f16", with_color=True)
    vm.CreateMap(SMALL.num_entries, 1 << 12, SMALL.voxel_size)
    pose = synth.Scene(SMALL).poses[0]
    nm = torch.empty((SMALL.height, SMALL.width, 4), device="cuda")
    v = vm.RenderScene(None, pose, nmap=nm).cpu().numpy()
    assert np.isnan(v).all() and np.isnan(nm.cpu().numpy()).all()
    k, verts, norms = vm.Polygonize()
    assert k == 0 and verts.shape[0] == 0 and len(vm.GetSurfacePoints()) == 0
    assert vm.export_blocks()["coords"].shape == (0, 3)
    snap = vm.save_snapshot()
    other = VoxelMapping(SMALL.width, SMALL.height, SMALL.K, voxel_format="f16", with_color=True)
    other.CreateMap(SMALL.num_entries, 1 << 12, SMALL.voxel_size)
    d, c, p = synth.Scene(SMALL).render(0)
    other.FuseDepthAndImage(torch.from_numpy(c).cuda().reshape(SMALL.height, -1),
                            torch.from_numpy(d.view(np.int16)).cuda(), p)
    other.load_snapshot(snap)
    assert other.stats()["allocated_blocks"] == 0
    # a batch step over empty maps, render only
    b = MapBatch([vm, other])
    out = [torch.zeros((SMALL.height, SMALL.width, 4), device="cuda") for _ in range(2)]
    b.step([None, None], None, [pose, pose], out)
    torch.cuda.synchronize()
    assert all(np.isnan(o.cpu().numpy()).all() for o in out)
    assert vm.stats()["error_flags"] == 0 and other.stats()["error_flags"] == 0
    b.release()


def test_largest_image_finest_voxels_against_oracle():
    wl = dataclasses.replace(synth.WORKLOADS["room_full"], width=1280, height=720, fx=1050.0, fy=1050.0, cx=639.5,
                             cy=359.5, voxel_size=0.004, num_blocks=1 << 18, name="hd")
    sc = synth.Scene(wl)
    vm, om = make_pair(wl, fmt="f16", color=True, max_weight=128)
    for i in (0, 7):
        d, rgb, pose = sc.render(i)
        st, orc = fuse_both(vm, om, d, rgb, pose)
        assert st["visible_blocks"] == orc["visible"] > 5000
    g, o = aligned_maps(vm, om)
    assert np.array_equal(g["coords"], o["coords"]) and np.array_equal(g["tsdf"], o["tsdf"].astype(np.float32))
    assert np.array_equal(g["weight"], o["weight"].astype(np.float32)) and np.array_equal(g["rgb"], o["rgb"])
    r = raycast_stats(vm.RenderScene(None, pose).cpu().numpy(), om.raycast(pose))
    assert r["mismatch"] <= 0.005 and r["frac_within_1mm"] >= 0.995, r
    k, verts, norms = vm.Polygonize()
    n, v_o, n_o = om.polygonize()
    assert k == n > 100000
    assert np.array_equal(sorted_rows(np.concatenate([verts, norms], 1)), sorted_rows(np.concatenate([v_o, n_o], 1)))


@pytest.mark.parametrize("fmt,wmax", [("f32", 255), ("f16", 128), ("i16", 128)])
def test_raycast_every_storage_format(fmt, wmax):
    sc = synth.Scene(SMALL)
    vm, om = make_pair(SMALL, fmt=fmt, color=False, max_weight=wmax)
    for i in range(0, 20, 2):
        d, _, pose = sc.render(i)
        fuse_both(vm, om, d, None, pose)
    for pose in (sc.poses[18], sc.poses[7]):
        r = raycast_stats(vm.RenderScene(None, pose).cpu().numpy(), om.raycast(pose))
        assert r["hits_gpu"] > 0.5 * SMALL.width * SMALL.height
        assert r["mismatch"] <= 0.005 and r["frac_within_1mm"] >= 0.995 and r["dz_mean_mm"] <= 0.05, (fmt, r)
