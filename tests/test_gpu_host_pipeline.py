"""Pipelined host frames (vmap_frame_host_async / vmap_host_wait): a sequence
run through the pipeline - copies of neighbouring frames overlapping each
other's kernels, one frame fuse-only - gives every frame's vertex and normal
maps and the final map bit-identical to the synchronous host calls
(vmap_fuse_host + vmap_render_scene_host)."""
import ctypes as C

import numpy as np
import pytest
import torch

from tests.common import block_keys
from voxelmapping_b200 import VoxelMapping
from voxelmapping_b200 import _lib as L
from voxelmapping_b200 import synth

pytestmark = pytest.mark.gpu
WL = synth.WORKLOADS["room_small"]


def new_map():
    vm = VoxelMapping(WL.width, WL.height, WL.K, voxel_format="f32", with_color=True)
    vm.CreateMap(WL.num_entries, 1 << 16, WL.voxel_size)
    return vm


def test_pipeline_equals_synchronous_host_calls():
    lib = L.lib()
    sc = synth.Scene(WL)
    idx = list(range(0, 40, 4))
    frames = [sc.render(i) for i in idx]
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    depth = [pin(d.view(np.int16)) for d, _, _ in frames]
    rgb = [pin(c) for _, c, _ in frames]
    shape = (WL.height, WL.width, 4)
    fuse_only = 5

    a = new_map()
    s = torch.cuda.current_stream().cuda_stream
    ref = []
    for k, (d, c, p) in enumerate(frames):
        L.check(lib.vmap_fuse_host(a._map, C.c_void_p(depth[k].data_ptr()), L.DEPTH_U16, 0.001,
                                   C.c_void_p(rgb[k].data_ptr()), L.pose_arg(p), s))
        if k == fuse_only:
            ref.append(None)
            continue
        v = torch.empty(shape, dtype=torch.float32).pin_memory()
        n = torch.empty(shape, dtype=torch.float32).pin_memory()
        L.check(lib.vmap_render_scene_host(a._map, L.pose_arg(p), C.c_void_p(v.data_ptr()), C.c_void_p(n.data_ptr()), s))
        torch.cuda.synchronize()
        ref.append((v.numpy().copy(), n.numpy().copy()))

    b = new_map()
    side = torch.cuda.Stream()
    outs, hf = [], []
    for k, (d, c, p) in enumerate(frames):
        f = L.HostFrame()
        f.depth_host, f.depth_type, f.depth_scale = depth[k].data_ptr(), L.DEPTH_U16, 0.001
        f.rgb_host = rgb[k].data_ptr()
        f.pose[:] = [float(x) for x in p.reshape(16)]
        if k != fuse_only:
            v = torch.full(shape, 7.0).pin_memory()
            n = torch.full(shape, 7.0).pin_memory()
            f.vmap_host, f.nmap_host = v.data_ptr(), n.data_ptr()
            outs.append((v, n))
        else:
            outs.append(None)
        hf.append(f)
        L.check(lib.vmap_frame_host_async(b._map, C.byref(f), C.c_void_p(side.cuda_stream)))
    L.check(lib.vmap_host_wait(b._map, C.c_void_p(side.cuda_stream)))
    side.synchronize()
    for k, (r, o) in enumerate(zip(ref, outs)):
        if r is None:
            assert o is None
            continue
        assert np.array_equal(np.nan_to_num(r[0], nan=-9), np.nan_to_num(o[0].numpy(), nan=-9)), k
        assert np.array_equal(np.nan_to_num(r[1], nan=-9), np.nan_to_num(o[1].numpy(), nan=-9)), k
        assert np.isfinite(r[0][..., 0]).mean() > 0.3
    ea, eb = a.export_blocks(), b.export_blocks()
    ia, ib = np.argsort(block_keys(ea["coords"])), np.argsort(block_keys(eb["coords"]))
    for x in ("coords", "tsdf", "weight", "rgb"):
        assert np.array_equal(ea[x][ia], eb[x][ib]), x
    # invalid frames are refused before anything is enqueued
    bad = L.HostFrame()
    bad.depth_host, bad.depth_type, bad.depth_scale = depth[0].data_ptr(), 9, 0.001
    bad.pose[:] = [float(x) for x in frames[0][2].reshape(16)]
    assert lib.vmap_frame_host_async(b._map, C.byref(bad), None) == 1
    bad.depth_type, bad.nmap_host = L.DEPTH_U16, outs[0][1].data_ptr()  # normals without a vertex map
    assert lib.vmap_frame_host_async(b._map, C.byref(bad), None) == 1


def test_python_host_pipeline_wrapper():
    from voxelmapping_b200 import HostPipeline
    sc = synth.Scene(WL)
    frames = [sc.render(i) for i in range(0, 20, 5)]
    a, b = new_map(), new_map()
    pipe = HostPipeline(b)
    outs = [pipe.submit(d, c, p) for d, c, p in frames]
    pipe.wait()
    for (d, c, p), (v, n) in zip(frames, outs):
        a.FuseDepthAndImage(c, synth.depth_to_metres(d), p)
        nm = torch.empty((WL.height, WL.width, 4), device="cuda")
        va = a.RenderScene(None, p, nmap=nm).cpu().numpy()
        assert np.array_equal(np.nan_to_num(va, nan=-9), np.nan_to_num(v, nan=-9))
        assert np.array_equal(np.nan_to_num(nm.cpu().numpy(), nan=-9), np.nan_to_num(n, nan=-9))
