"""Batched fuse + raycast (vmap_batch_*): a batch step over maps of different
image sizes, cameras, voxel sizes and pools must leave every map, vertex map
and normal map bit-identical to driving each map on its own, under both
schedules (batch_schedule 1: one launch per stage; 2: one persistent launch
fed by a device-side task queue). Steps run on a side stream so the graph
recording (steps 1-2) and replay (steps 3+) are both covered."""
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


SCHEDULES = pytest.mark.parametrize("schedule", [1, 2], ids=["stages", "persistent"])


@SCHEDULES
def test_batch_step_equals_single_map_calls(schedule):
    wls = workloads()
    scenes = [synth.Scene(wl) for wl in wls]
    batch_maps = [make_map(wl) for wl in wls]
    solo_maps = [make_map(wl) for wl in wls]
    batch = MapBatch(batch_maps)
    batch.set_launch_config(batch_schedule=schedule)
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


@SCHEDULES
def test_batch_fuse_only_and_render_only_frames(schedule):
    """A step may fuse some maps, render others and leave the rest idle: the
    result equals the matching single-map calls, and idle maps keep their
    visible count."""
    wls = workloads()
    scenes = [synth.Scene(wl) for wl in wls]
    batch_maps = [make_map(wl) for wl in wls]
    solo_maps = [make_map(wl) for wl in wls]
    batch = MapBatch(batch_maps)
    batch.set_launch_config(batch_schedule=schedule)
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


@SCHEDULES
def test_uneven_batch_equals_single_map_calls(schedule):
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
    batch.set_launch_config(batch_schedule=schedule)
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


@SCHEDULES
def test_slot_batch_with_maps_in_caller_memory(schedule):
    """vmap_batch_create_slots + vmap_batch_set_map with maps built by
    vmap_create_in: maps move between slots and sit out steps (empty slot)
    while the recorded graphs are replayed; results equal single-map calls."""
    import ctypes as C
    lib = L.lib()
    wls = workloads()
    scenes = [synth.Scene(wl) for wl in wls]
    solo_maps = [make_map(wl) for wl in wls]
    slot_maps, mems = [], []
    for wl in wls:
        vm = VoxelMapping(wl.width, wl.height, wl.K, voxel_format=wl.voxel_format, with_color=wl.with_color,
                          max_weight=128)
        need = vm.required_bytes(1 << 18, wl.num_blocks, wl.voxel_size)
        mem = torch.full((need + 4096,), 0xAB, dtype=torch.uint8, device="cuda")  # dirty memory
        vm.CreateMapIn(1 << 18, wl.num_blocks, wl.voxel_size, mem)
        assert vm.stats()["device_bytes"] == need
        slot_maps.append(vm)
    with pytest.raises(L.VmapError):
        VoxelMapping(wls[0].width, wls[0].height, wls[0].K, voxel_format="f16").CreateMapIn(
            1 << 18, wls[0].num_blocks, wls[0].voxel_size, torch.empty(1000, dtype=torch.uint8, device="cuda"))
    h = C.c_void_p()
    L.check(lib.vmap_batch_create_slots(5, L.VOXEL_F16, C.byref(h)))
    cfg = L.LaunchConfig()
    L.check(lib.vmap_batch_get_launch_config(h, C.byref(cfg)))
    cfg.batch_schedule = schedule
    L.check(lib.vmap_batch_set_launch_config(h, C.byref(cfg)))
    f32 = VoxelMapping(64, 48, wls[0].K, voxel_format="f32")
    f32.CreateMap(1 << 10, 1 << 10, 0.01)
    assert lib.vmap_batch_set_map(h, 0, f32._map) == 1
    side = torch.cuda.Stream()
    # slot of each map per step (None: not in the batch this step)
    layout = [[0, 1, 2], [4, 1, 2], [4, None, 0], [3, 1, 0], [3, 2, 1], [0, 2, 1]]
    cur = [None] * 3
    frames = (L.BatchFrame * 5)()
    for step, slots in enumerate(layout):
        for i, sl in enumerate(slots):  # empty old slots first, then fill
            if cur[i] is not None and cur[i] != sl:
                L.check(lib.vmap_batch_set_map(h, cur[i], None))
        for i, sl in enumerate(slots):
            if sl is not None:
                L.check(lib.vmap_batch_set_map(h, sl, slot_maps[i]._map))
            cur[i] = sl
        for k in range(5):
            fr = frames[k]
            fr.depth_dev = fr.rgb_dev = fr.vmap_dev = fr.nmap_dev = None
        keep, outs = [], {}
        for i, (wl, sc) in enumerate(zip(wls, scenes)):
            if slots[i] is None:
                continue
            d, c, p = sc.render(step * 3)
            dt = torch.from_numpy(d.view(np.int16)).cuda()
            ct = torch.from_numpy(c).cuda().reshape(wl.height, -1) if wl.with_color else None
            vb = torch.full((wl.height, wl.width, 4), 7.0, device="cuda")
            nb = torch.full((wl.height, wl.width, 4), 7.0, device="cuda")
            keep += [dt, ct, vb, nb]
            fr = frames[slots[i]]
            fr.depth_dev, fr.depth_type, fr.depth_pitch, fr.depth_scale = dt.data_ptr(), L.DEPTH_U16, wl.width * 2, 0.001
            if ct is not None:
                fr.rgb_dev, fr.rgb_pitch = ct.data_ptr(), wl.width * 3
            fr.pose[:] = [float(x) for x in p.reshape(16)]
            fr.vmap_dev, fr.vmap_pitch, fr.nmap_dev, fr.nmap_pitch = vb.data_ptr(), wl.width * 16, nb.data_ptr(), \
                wl.width * 16
            outs[i] = (dt, ct, p, vb, nb)
        torch.cuda.synchronize()
        L.check(lib.vmap_batch_step(h, frames, C.c_void_p(side.cuda_stream)))
        side.synchronize()
        for i, (dt, ct, p, vb, nb) in outs.items():
            vm = solo_maps[i]
            if ct is not None:
                vm.FuseDepthAndImage(ct, dt, p)
            else:
                vm.FuseDepth(dt, p)
            nm = torch.empty_like(vb)
            v = vm.RenderScene(None, p, nmap=nm)
            torch.cuda.synchronize()
            assert np.array_equal(np.nan_to_num(v.cpu().numpy(), nan=-9.0), np.nan_to_num(vb.cpu().numpy(), nan=-9.0)), (step, i)
            assert np.array_equal(np.nan_to_num(nm.cpu().numpy(), nan=-9.0), np.nan_to_num(nb.cpu().numpy(), nan=-9.0)), (step, i)
    # a frame for an empty slot is refused
    for k in range(5):
        frames[k].depth_dev = frames[k].rgb_dev = frames[k].vmap_dev = frames[k].nmap_dev = None
    frames[4].vmap_dev = keep[2].data_ptr()
    assert lib.vmap_batch_step(h, frames, C.c_void_p(side.cuda_stream)) == 1
    side.synchronize()
    for wl, a, b in zip(wls, slot_maps, solo_maps):
        ea, eb = a.export_blocks(), b.export_blocks()
        ia, ib = np.argsort(block_keys(ea["coords"])), np.argsort(block_keys(eb["coords"]))
        for k in ("coords", "tsdf", "weight") + (("rgb",) if wl.with_color else ()):
            assert np.array_equal(ea[k][ia], eb[k][ib]), k
    L.check(lib.vmap_batch_destroy(h))
    for vm in slot_maps:
        vm.release()


def test_set_map_on_a_regular_batch_records_again_and_matches_single_calls():
    """vmap_batch_set_map on a batch made by vmap_batch_create (grids sized for
    its original maps): after swapping a map in, steps still equal single-map
    calls."""
    import ctypes as C
    wls = workloads()[:2]
    scenes = [synth.Scene(wl) for wl in wls]
    a, b = make_map(wls[0]), make_map(wls[1])
    c = make_map(wls[1])  # replaces b after two steps
    solo = [make_map(wls[0]), make_map(wls[1]), make_map(wls[1])]
    batch = MapBatch([a, b])
    side = torch.cuda.Stream()
    for step in range(5):
        cur = [a, b] if step < 2 else [a, c]
        if step == 2:
            L.check(L.lib().vmap_batch_set_map(batch._h, 1, c._map))
            batch.maps[1] = c
        fr = [sc.render(step * 4) for sc in scenes]
        depths = [torch.from_numpy(d.view(np.int16)).cuda() for d, _, _ in fr]
        rgbs = [torch.from_numpy(cc).cuda().reshape(wl.height, -1) if wl.with_color else None
                for (_, cc, _), wl in zip(fr, wls)]
        poses = [p for _, _, p in fr]
        vb = [torch.empty((wl.height, wl.width, 4), device="cuda") for wl in wls]
        torch.cuda.synchronize()
        with torch.cuda.stream(side):
            batch.step(depths, rgbs, poses, vb)
        side.synchronize()
        refs = [solo[0], solo[1] if step < 2 else solo[2]]
        for i, (wl, vm) in enumerate(zip(wls, refs)):
            if wl.with_color:
                vm.FuseDepthAndImage(rgbs[i], depths[i], poses[i])
            else:
                vm.FuseDepth(depths[i], poses[i])
            v = vm.RenderScene(None, poses[i])
            torch.cuda.synchronize()
            assert np.array_equal(np.nan_to_num(v.cpu().numpy(), nan=-9.0), np.nan_to_num(vb[i].cpu().numpy(), nan=-9.0)), (step, i)
    assert c.stats()["allocated_blocks"] == solo[2].stats()["allocated_blocks"] > 0
    # the same map in two slots is refused
    assert L.lib().vmap_batch_set_map(batch._h, 0, c._map) == 1
    batch.release()


def test_persistent_step_equals_stage_launches_on_many_maps():
    """40 maps (more than the task ring's first wave of openers needs), small
    and full-size images, one rendered in raycast mode 1, two left idle in
    some steps: the persistent step and the stage launches give bit-identical
    vertex maps, normal maps and voxels."""
    base = synth.WORKLOADS["room_small"]
    wls = [dataclasses.replace(base, seed=100 + i, width=96 + 8 * (i % 5), height=64 + 4 * (i % 3),
                               fx=90.0 + i, fy=90.0 + i, cx=48.0 + 4 * (i % 5), cy=32.0 + 2 * (i % 3),
                               voxel_format="f16", num_blocks=1 << 13, with_color=i % 2 == 0) for i in range(38)]
    wls += [dataclasses.replace(synth.WORKLOADS["room_full"], seed=200 + i, voxel_format="f16", num_blocks=1 << 16,
                                with_color=True) for i in range(2)]
    scenes = [synth.Scene(wl) for wl in wls]

    def mk(i, wl):
        vm = VoxelMapping(wl.width, wl.height, wl.K, voxel_format="f16", with_color=wl.with_color, max_weight=128,
                          raycast_mode=1 if i == 7 else 0)
        vm.CreateMap(1 << 15 if wl.num_blocks < (1 << 16) else 1 << 18, wl.num_blocks, wl.voxel_size)
        return vm

    maps = {s: [mk(i, wl) for i, wl in enumerate(wls)] for s in (1, 2)}
    batches = {s: MapBatch(maps[s]) for s in (1, 2)}
    for s, b in batches.items():
        b.set_launch_config(batch_schedule=s)
    side = torch.cuda.Stream()
    for step in range(4):
        fr = [sc.render(step * 5) for sc in scenes]
        idle = {3, 11} if step % 2 else set()
        depths = [None if i in idle else torch.from_numpy(d.view(np.int16)).cuda() for i, (d, _, _) in enumerate(fr)]
        rgbs = [torch.from_numpy(c).cuda().reshape(wl.height, -1) if wl.with_color and i not in idle else None
                for i, ((_, c, _), wl) in enumerate(zip(fr, wls))]
        poses = [p for _, _, p in fr]
        outs = {}
        for s, b in batches.items():
            vb = [None if i in idle else torch.full((wl.height, wl.width, 4), 7.0, device="cuda")
                  for i, wl in enumerate(wls)]
            nb = [None if v is None else torch.full_like(v, 7.0) for v in vb]
            torch.cuda.synchronize()
            with torch.cuda.stream(side):
                b.step(depths, rgbs, poses, vb, nb)
            side.synchronize()
            outs[s] = (vb, nb)
        for i in range(len(wls)):
            if i in idle:
                continue
            for k in (0, 1):
                a, c = outs[1][k][i].cpu().numpy(), outs[2][k][i].cpu().numpy()
                assert np.array_equal(np.nan_to_num(a, nan=-9.0), np.nan_to_num(c, nan=-9.0)), (step, i, k)
    hit = np.mean([np.isfinite(v.cpu().numpy()[..., 0]).mean() for v in outs[2][0] if v is not None])
    assert hit > 0.3
    for i, (a, c) in enumerate(zip(maps[1], maps[2])):
        ea, ec = a.export_blocks(), c.export_blocks()
        ia, ic = np.argsort(block_keys(ea["coords"])), np.argsort(block_keys(ec["coords"]))
        for k in ("coords", "tsdf", "weight") + (("rgb",) if wls[i].with_color else ()):
            assert np.array_equal(ea[k][ia], ec[k][ic]), (i, k)
        assert a.stats()["visible_blocks"] == c.stats()["visible_blocks"], i
        assert a.stats()["error_flags"] == c.stats()["error_flags"] == 0, i
    for b in batches.values():
        b.release()


def test_persistent_step_wait_is_bounded():
    """The persistent step's waits end on their own. With one task-ring entry
    that nothing writes (vmap_batch_stall_probe), every warp gives up once the
    stall limit passes without progress: the launch ends, every map carries
    VMAP_FLAG_STEP_STALLED, and the context stays usable (the reset maps then
    step normally and equal single-map calls)."""
    import time
    wls = workloads()[:2]
    scenes = [synth.Scene(wl) for wl in wls]
    maps = [make_map(wl) for wl in wls]
    solo = [make_map(wl) for wl in wls]
    batch = MapBatch(maps)
    batch.set_launch_config(batch_schedule=2)
    side = torch.cuda.Stream()

    def frame(step):
        fr = [sc.render(step) for sc in scenes]
        depths = [torch.from_numpy(d.view(np.int16)).cuda() for d, _, _ in fr]
        rgbs = [torch.from_numpy(c).cuda().reshape(wl.height, -1) if wl.with_color else None
                for (_, c, _), wl in zip(fr, wls)]
        vb = [torch.full((wl.height, wl.width, 4), 7.0, device="cuda") for wl in wls]
        return depths, rgbs, [p for _, _, p in fr], vb

    depths, rgbs, poses, vb = frame(0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with torch.cuda.stream(side):
        batch.stall_probe(depths, rgbs, poses, vb, stall_ms=200)
    side.synchronize()
    dt = time.perf_counter() - t0
    assert 0.15 < dt < 10.0, dt
    for m in maps:
        assert m.stats()["error_flags"] & L.FLAG_STEP_STALLED
        m.clear_errors()
        m.reset()
    depths, rgbs, poses, vb = frame(3)
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        batch.step(depths, rgbs, poses, vb)
    side.synchronize()
    for i, (wl, vm) in enumerate(zip(wls, solo)):
        if wl.with_color:
            vm.FuseDepthAndImage(rgbs[i], depths[i], poses[i])
        else:
            vm.FuseDepth(depths[i], poses[i])
        v = vm.RenderScene(None, poses[i])
        torch.cuda.synchronize()
        assert np.array_equal(np.nan_to_num(v.cpu().numpy(), nan=-9.0), np.nan_to_num(vb[i].cpu().numpy(), nan=-9.0))
        assert maps[i].stats()["error_flags"] == 0
    batch.release()
