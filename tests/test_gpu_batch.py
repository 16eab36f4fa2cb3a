"""Batched fuse + raycast (vmap_batch_*): a batch step over maps of different
image sizes, cameras, voxel sizes and pools must leave every map, vertex map
and normal map bit-identical to driving each map on its own. Steps run on a
side stream so the graph recording (steps 1-2) and replay (steps 3+) are both
covered."""
import dataclasses

import numpy as np
import pytest
import torch

from tests.common import block_keys
from voxelmapping_b200 import MapBatch, VoxelMapping
from voxelmapping_b200 import _lib as L
from voxelmapping_b200 import synth

pytestmark = pytest.mark.gpu


def workloads():
    small = synth.WORKLOADS["room_small"]
    full = synth.WORKLOADS["room_full"]
    return [
        dataclasses.replace(small, seed=11, voxel_format="f16", num_blocks=1 << 16, with_color=True),
        dataclasses.replace(small, name="ragged", width=203, height=117, fx=181.3, fy=179.9, cx=97.2, cy=55.7,
                            seed=12, voxel_format="f16", voxel_size=0.012, num_blocks=1 << 14, with_color=False,
                            room=(2.5, 3.0, 2.5), cam_radius=0.6, cam_height=1.2),
        dataclasses.replace(full, seed=13, voxel_format="f16", num_blocks=1 << 16, with_color=True),
    ]


def make_map(wl):
    vm = VoxelMapping(wl.width, wl.height, wl.K, voxel_format=wl.voxel_format, with_color=wl.with_color,
                      max_weight=128)
    vm.CreateMap(1 << 18, wl.num_blocks, wl.voxel_size)
    return vm


def test_batch_step_equals_single_map_calls():
    wls = workloads()
    scenes = [synth.Scene(wl) for wl in wls]
    batch_maps = [make_map(wl) for wl in wls]
    solo_maps = [make_map(wl) for wl in wls]
    batch = MapBatch(batch_maps)
    side = torch.cuda.Stream()
    for step in range(5):
        depths, rgbs, poses, vb, nb = [], [], [], [], []
        for wl, sc in zip(wls, scenes):
            d, c, p = sc.render(step * 3)
            depths.append(torch.from_numpy(d.view(np.int16)).cuda())
            rgbs.append(torch.from_numpy(c).cuda().reshape(wl.height, -1) if wl.with_color else None)
            poses.append(p)
            vb.append(torch.full((wl.height, wl.width, 4), 7.0, device="cuda"))
            nb.append(torch.full((wl.height, wl.width, 4), 7.0, device="cuda"))
        torch.cuda.synchronize()
        with torch.cuda.stream(side):
            batch.step(depths, rgbs, poses, vb, nb)
        side.synchronize()
        for i, (wl, vm) in enumerate(zip(wls, solo_maps)):
            if wl.with_color:
                vm.FuseDepthAndImage(rgbs[i], depths[i], poses[i])
            else:
                vm.FuseDepth(depths[i], poses[i])
            nm = torch.empty_like(vb[i])
            v = vm.RenderScene(None, poses[i], nmap=nm)
            torch.cuda.synchronize()
            assert np.array_equal(np.nan_to_num(v.cpu().numpy(), nan=-9.0), np.nan_to_num(vb[i].cpu().numpy(), nan=-9.0)), (step, i)
            assert np.array_equal(np.nan_to_num(nm.cpu().numpy(), nan=-9.0), np.nan_to_num(nb[i].cpu().numpy(), nan=-9.0)), (step, i)
            assert np.isfinite(v.cpu().numpy()[..., 0]).mean() > 0.3
    for wl, a, b in zip(wls, batch_maps, solo_maps):
        ea, eb = a.export_blocks(), b.export_blocks()
        ia, ib = np.argsort(block_keys(ea["coords"])), np.argsort(block_keys(eb["coords"]))
        for k in ("coords", "tsdf", "weight") + (("rgb",) if wl.with_color else ()):
            assert np.array_equal(ea[k][ia], eb[k][ib]), k
        assert a.stats()["error_flags"] == 0
    batch.release()


def test_batch_rejects_mixed_formats_and_duplicates():
    wl = synth.WORKLOADS["room_small"]
    a = VoxelMapping(wl.width, wl.height, wl.K, voxel_format="f16", with_color=False)
    a.CreateMap(1 << 14, 1 << 12, wl.voxel_size)
    b = VoxelMapping(wl.width, wl.height, wl.K, voxel_format="f32", with_color=False)
    b.CreateMap(1 << 14, 1 << 12, wl.voxel_size)
    with pytest.raises(L.VmapError):
        MapBatch([a, b])
    with pytest.raises(L.VmapError):
        MapBatch([a, a])


def test_batch_fuse_only_and_render_only_frames():
    """A step may fuse some maps, render others and leave the rest idle: the
    result equals the matching single-map calls, and idle maps keep their
    visible count."""
    wls = workloads()
    scenes = [synth.Scene(wl) for wl in wls]
    batch_maps = [make_map(wl) for wl in wls]
    solo_maps = [make_map(wl) for wl in wls]
    batch = MapBatch(batch_maps)
    side = torch.cuda.Stream()
    # (fuse, render) per map and step; step 0 fuses everything so renders see surface
    plan = [[(1, 1), (1, 1), (1, 1)], [(1, 0), (0, 1), (0, 0)], [(0, 1), (1, 0), (1, 1)],
            [(0, 0), (1, 1), (0, 1)], [(1, 0), (0, 0), (1, 0)]]
    for step, work in enumerate(plan):
        depths, rgbs, poses, vb, nb = [], [], [], [], []
        for (fu, re), wl, sc in zip(work, wls, scenes):
            d, c, p = sc.render(step * 4)
            depths.append(torch.from_numpy(d.view(np.int16)).cuda() if fu else None)
            rgbs.append(torch.from_numpy(c).cuda().reshape(wl.height, -1) if fu and wl.with_color else None)
            poses.append(p)
            vb.append(torch.full((wl.height, wl.width, 4), 7.0, device="cuda") if re else None)
            nb.append(torch.full((wl.height, wl.width, 4), 7.0, device="cuda") if re else None)
        vis_before = [m.stats()["visible_blocks"] for m in batch_maps]
        torch.cuda.synchronize()
        with torch.cuda.stream(side):
            batch.step(depths, rgbs, poses, vb, nb)
        side.synchronize()
        for i, ((fu, re), wl, vm) in enumerate(zip(work, wls, solo_maps)):
            if fu:
                if wl.with_color:
                    vm.FuseDepthAndImage(rgbs[i], depths[i], poses[i])
                else:
                    vm.FuseDepth(depths[i], poses[i])
                assert batch_maps[i].stats()["visible_blocks"] == vm.stats()["visible_blocks"], (step, i)
            else:
                assert batch_maps[i].stats()["visible_blocks"] == vis_before[i], (step, i)
            if re:
                nm = torch.empty_like(vb[i])
                v = vm.RenderScene(None, poses[i], nmap=nm)
                torch.cuda.synchronize()
                assert np.array_equal(np.nan_to_num(v.cpu().numpy(), nan=-9.0),
                                      np.nan_to_num(vb[i].cpu().numpy(), nan=-9.0)), (step, i)
                assert np.array_equal(np.nan_to_num(nm.cpu().numpy(), nan=-9.0),
                                      np.nan_to_num(nb[i].cpu().numpy(), nan=-9.0)), (step, i)
    for wl, a, b in zip(wls, batch_maps, solo_maps):
        ea, eb = a.export_blocks(), b.export_blocks()
        ia, ib = np.argsort(block_keys(ea["coords"])), np.argsort(block_keys(eb["coords"]))
        for k in ("coords", "tsdf", "weight") + (("rgb",) if wl.with_color else ()):
            assert np.array_equal(ea[k][ia], eb[k][ib]), k
        assert a.stats()["error_flags"] == 0
    batch.release()


def test_uneven_batch_equals_single_map_calls():
    """Maps of uneven extent, voxel size (4-16 mm), resolution (up to
    1280x720) and pool size in one batch."""
    # pools 4x the generator's so no allocation is refused (which blocks a full
    # pool refuses depends on scheduling order)
    wls = [dataclasses.replace(w, num_blocks=4 * w.num_blocks) for w in synth.uneven_workloads(10, seed=3)]
    assert len({(w.width, w.voxel_size, w.num_blocks) for w in wls}) >= 6
    scenes = [synth.Scene(wl) for wl in wls]
    mk = lambda wl: VoxelMapping(wl.width, wl.height, wl.K, voxel_format=wl.voxel_format, with_color=wl.with_color,
                                 max_weight=wl.max_weight)
    batch_maps, solo_maps = [mk(wl) for wl in wls], [mk(wl) for wl in wls]
    for m, wl in zip(batch_maps + solo_maps, wls + wls):
        m.CreateMap(wl.num_entries, wl.num_blocks, wl.voxel_size)
    batch = MapBatch(batch_maps)
    side = torch.cuda.Stream()
    for step in range(3):
        frames = [sc.render(step * 7) for sc in scenes]
        depths = [torch.from_numpy(d.view(np.int16)).cuda() for d, _, _ in frames]
        rgbs = [torch.from_numpy(c).cuda().reshape(wl.height, -1) for (_, c, _), wl in zip(frames, wls)]
        poses = [p for _, _, p in frames]
        vb = [torch.full((wl.height, wl.width, 4), 7.0, device="cuda") for wl in wls]
        nb = [torch.full((wl.height, wl.width, 4), 7.0, device="cuda") for wl in wls]
        torch.cuda.synchronize()
        with torch.cuda.stream(side):
            batch.step(depths, rgbs, poses, vb, nb)
        side.synchronize()
        for i, vm in enumerate(solo_maps):
            vm.FuseDepthAndImage(rgbs[i], depths[i], poses[i])
            nm = torch.empty_like(vb[i])
            v = vm.RenderScene(None, poses[i], nmap=nm)
            torch.cuda.synchronize()
            assert np.array_equal(np.nan_to_num(v.cpu().numpy(), nan=-9.0), np.nan_to_num(vb[i].cpu().numpy(), nan=-9.0)), (step, i)
            assert np.array_equal(np.nan_to_num(nm.cpu().numpy(), nan=-9.0), np.nan_to_num(nb[i].cpu().numpy(), nan=-9.0)), (step, i)
    hit = np.mean([np.isfinite(v.cpu().numpy()[..., 0]).mean() for v in vb])
    assert hit > 0.3
    for a, b in zip(batch_maps, solo_maps):
        ea, eb = a.export_blocks(), b.export_blocks()
        ia, ib = np.argsort(block_keys(ea["coords"])), np.argsort(block_keys(eb["coords"]))
        for k in ("coords", "tsdf", "weight", "rgb"):
            assert np.array_equal(ea[k][ia], eb[k][ib]), k
        assert a.stats()["error_flags"] == b.stats()["error_flags"] == 0
    batch.release()
