"""Launch shapes (vmap_launch_config) change only the time: maps and batches
run with extreme grids give bit-identical maps, vertex/normal maps and meshes;
invalid shapes are refused; the autotuner runs and applies its choice."""
import dataclasses

import numpy as np
import pytest
import torch

from tests.common import block_keys, sorted_rows
from voxelmapping_b200 import MapBatch, VoxelMapping
from voxelmapping_b200 import _lib as L
from voxelmapping_b200 import autotune as AT
from voxelmapping_b200 import synth

pytestmark = pytest.mark.gpu
WL = synth.WORKLOADS["room_small"]
GRIDS = [f for f in AT.FIELDS if f.endswith("_ctas_per_sm")]
SHAPES = [{}, dict({f: 1 for f in GRIDS}, raycast_tile_order=1, raycast_tile_width=16, raycast_threads_per_cta=128),
          dict({f: 32 for f in GRIDS}, raycast_tile_order=2, raycast_tile_width=4, raycast_threads_per_cta=256)]


def new_map(**shape):
    vm = VoxelMapping(WL.width, WL.height, WL.K, voxel_format="f16", with_color=True)
    vm.CreateMap(WL.num_entries, 1 << 16, WL.voxel_size)
    if shape:
        vm.set_launch_config(**shape)
    return vm


def test_map_results_do_not_depend_on_launch_shape():
    sc = synth.Scene(WL)
    frames = [sc.render(i) for i in range(0, 24, 3)]
    outs = []
    for shape in SHAPES:
        vm = new_map(**shape)
        got = vm.get_launch_config()
        for f, v in shape.items():
            assert got[f] == v
        nm = torch.empty((WL.height, WL.width, 4), device="cuda")
        for d, c, p in frames:
            vm.FuseDepthAndImage(torch.from_numpy(c).cuda().reshape(WL.height, -1),
                                 torch.from_numpy(d.view(np.int16)).cuda(), p)
            v = vm.RenderScene(None, p, nmap=nm)
        e = vm.export_blocks()
        i = np.argsort(block_keys(e["coords"]))
        k, verts, norms = vm.Polygonize()
        outs.append(({x: e[x][i] for x in ("coords", "tsdf", "weight", "rgb")}, np.nan_to_num(v.cpu().numpy(), nan=-9),
                     np.nan_to_num(nm.cpu().numpy(), nan=-9), sorted_rows(np.concatenate([verts, norms], 1))))
    for o in outs[1:]:
        for x in ("coords", "tsdf", "weight", "rgb"):
            assert np.array_equal(o[0][x], outs[0][0][x]), x
        for a, b in zip(o[1:], outs[0][1:]):
            assert np.array_equal(a, b)


def test_invalid_shapes_are_refused():
    vm = new_map()
    for bad in ({"fuse_ctas_per_sm": 65}, {"raycast_ctas_per_sm": -1}, {"raycast_tile_order": 3},
                {"raycast_tile_width": 5}, {"raycast_threads_per_cta": 64}):
        with pytest.raises(L.VmapError):
            vm.set_launch_config(**bad)
    vm.set_launch_config(**{f: 0 for f in AT.FIELDS})  # 0 = defaults
    assert vm.get_launch_config()["fuse_ctas_per_sm"] == 16 and vm.get_launch_config()["raycast_ctas_per_sm"] == 0


def test_batch_results_do_not_depend_on_launch_shape_and_tuner_runs():
    wls = [dataclasses.replace(WL, seed=s, voxel_format="f16", with_color=True, num_blocks=1 << 15) for s in (1, 2, 3)]
    scenes = [synth.Scene(w) for w in wls]
    side = torch.cuda.Stream()
    results = []
    for shape in SHAPES:
        maps = [VoxelMapping(w.width, w.height, w.K, voxel_format="f16", with_color=True) for w in wls]
        for m, w in zip(maps, wls):
            m.CreateMap(w.num_entries, w.num_blocks, w.voxel_size)
        b = MapBatch(maps)
        if shape:
            b.set_launch_config(**shape)
        vb = [torch.empty((w.height, w.width, 4), device="cuda") for w in wls]
        for step in range(4):
            fr = [sc.render(step * 5) for sc in scenes]
            with torch.cuda.stream(side):
                b.step([torch.from_numpy(d.view(np.int16)).cuda() for d, _, _ in fr],
                       [torch.from_numpy(c).cuda().reshape(w.height, -1) for (_, c, _), w in zip(fr, wls)],
                       [p for _, _, p in fr], vb)
            side.synchronize()
        results.append([np.nan_to_num(v.cpu().numpy(), nan=-9) for v in vb])
        b.release()
    for r in results[1:]:
        for a, c in zip(r, results[0]):
            assert np.array_equal(a, c)
    # the tuner on a small map: picks a candidate for every stage and applies it
    sc = scenes[0]
    frames = [sc.render(i) for i in range(6)]
    dev = [(torch.from_numpy(d.view(np.int16)).cuda(), torch.from_numpy(c).cuda().reshape(WL.height, -1), p)
           for d, c, p in frames]
    vm = new_map()
    lib = L.lib()
    vout = torch.empty((WL.height, WL.width, 4), device="cuda")
    s = torch.cuda.current_stream().cuda_stream

    def step(i):
        d, c, p = dev[i % len(dev)]
        L.check(lib.vmap_fuse_depth_rgb(vm._map, d.data_ptr(), L.DEPTH_U16, WL.width * 2, 0.001, c.data_ptr(),
                                        WL.width * 3, L.pose_arg(p), s))
        L.check(lib.vmap_render_scene(vm._map, L.pose_arg(p), vout.data_ptr(), WL.width * 16, None, 0, s))
    best, table = AT.tune_map(vm, step, n_steps=2, rounds=1, warmup=1)
    # coordinate descent on whole-step time: every stage grid and the ray
    # marcher's parameters get a median per candidate, and the best is applied
    assert set(table) == set(AT.STAGE) | set(AT.RAYCAST_PARAMS)
    assert all(set(table[f]) == set(AT.CANDIDATES[f]) and best[f] in AT.CANDIDATES[f] for f in table)
    assert all(v > 0 for t in table.values() for v in t.values())
    assert vm.get_launch_config() == best
    m_best, m_table = AT.tune_mesh(vm, rounds=1)
    assert m_best in AT.CANDIDATES["mesh_ctas_per_sm"] and vm.get_launch_config()["mesh_ctas_per_sm"] == m_best
