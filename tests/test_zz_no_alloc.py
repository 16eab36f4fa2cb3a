"""vmap_export_blocks_static: the block export for callers that cannot allocate.

Callers running under a no-allocation policy, or inside a host application
that owns all device memory, cannot use vmap_export_blocks, which allocates
device staging on every call.
The static variant stages through a fixed device array instead. Here it must
return exactly what vmap_export_blocks returns (the export is exact, so the
tolerance is zero), on two calls in a row over the same map, and refuse
requests larger than its staging array.

This file is collected last on purpose so that a run stopping at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from voxelmapping_b200 import VoxelMapping
from voxelmapping_b200 import _lib as L
from voxelmapping_b200 import synth

pytestmark = pytest.mark.gpu

MAX_BLOCKS = 256  # VMAP_EXPORT_STATIC_MAX_BLOCKS in include/vmap_c.h


def static_export(vm, n):
    lib = L.lib()
    coords = np.zeros((n, 3), np.int32)
    tsdf = np.zeros((n, 512), np.float32)
    weight = np.zeros((n, 512), np.float32)
    rgb = np.zeros((n, 512, 3), np.uint8)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for first in range(0, n, MAX_BLOCKS):
        got = C.c_uint32()
        st = lib.vmap_export_blocks_static(vm._map, first, MAX_BLOCKS, coords[first:].ctypes.data,
                                           tsdf[first:].ctypes.data, weight[first:].ctypes.data,
                                           rgb[first:].ctypes.data, C.byref(got), stream)
        L.check(st, "vmap_export_blocks_static")
        assert got.value == min(MAX_BLOCKS, n - first)
    return {"coords": coords, "tsdf": tsdf, "weight": weight, "rgb": rgb}


def test_static_export_matches_allocating_export_on_two_calls():
    wl = synth.WORKLOADS["room_small"]
    scene = synth.Scene(wl)
    vm = VoxelMapping(wl.width, wl.height, wl.K, voxel_format="f16", with_color=True, max_weight=128)
    vm.CreateMap(wl.num_entries, wl.num_blocks, wl.voxel_size)
    for i in (0, 4, 8):
        d, rgb, pose = scene.render(i)
        vm.FuseDepthAndImage(rgb, d, pose)
    ref = vm.export_blocks()
    n = ref["coords"].shape[0]
    assert n > 2 * MAX_BLOCKS
    for _ in range(2):
        got = static_export(vm, n)
        for k in ("coords", "tsdf", "weight", "rgb"):
            assert np.array_equal(got[k], ref[k]), k
    # past the end: nothing to export
    cnt = C.c_uint32(7)
    L.check(L.lib().vmap_export_blocks_static(vm._map, n, MAX_BLOCKS, None, None, None, None, C.byref(cnt),
                                              C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    assert cnt.value == 0
    vm.release()


@pytest.mark.parametrize("fmt", ["ref", "i16"])
def test_static_export_without_colour_tsdf_only(fmt):
    """A map without colour, and only the TSDF requested (the other outputs
    NULL): the same TSDF as vmap_export_blocks, on two calls in a row."""
    wl = synth.WORKLOADS["room_small"]
    scene = synth.Scene(wl)
    vm = VoxelMapping(wl.width, wl.height, wl.K, voxel_format=fmt, with_color=False)
    vm.CreateMap(wl.num_entries, wl.num_blocks, wl.voxel_size)
    for i in (1, 5):
        d, _, pose = scene.render(i)
        vm.FuseDepth(torch.from_numpy(d.view(np.int16)).cuda(), pose)
    ref = vm.export_blocks(with_rgb=False)
    n = ref["coords"].shape[0]
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        tsdf = np.zeros((n, 512), np.float32)
        for first in range(0, n, MAX_BLOCKS):
            got = C.c_uint32()
            L.check(L.lib().vmap_export_blocks_static(vm._map, first, MAX_BLOCKS, None, tsdf[first:].ctypes.data, None,
                                                      None, C.byref(got), stream), "vmap_export_blocks_static")
            assert got.value == min(MAX_BLOCKS, n - first)
        assert np.array_equal(tsdf, ref["tsdf"])
    # colour requested from a map without colour: refused
    buf = np.zeros((1, 512, 3), np.uint8)
    got = C.c_uint32()
    assert L.lib().vmap_export_blocks_static(vm._map, 0, 1, None, None, None, buf.ctypes.data, C.byref(got),
                                             stream) == 1
    vm.release()


def test_static_export_rejects_more_than_its_staging_holds():
    wl = synth.WORKLOADS["room_small"]
    vm = VoxelMapping(wl.width, wl.height, wl.K, voxel_format="ref", with_color=False)
    vm.CreateMap(wl.num_entries, 1 << 12, wl.voxel_size)
    cnt = C.c_uint32()
    buf = np.zeros((MAX_BLOCKS + 1, 512), np.float32)
    st = L.lib().vmap_export_blocks_static(vm._map, 0, MAX_BLOCKS + 1, None, buf.ctypes.data, None, None,
                                           C.byref(cnt), None)
    assert st == 1  # VMAP_ERR_INVALID_ARG
    assert b"exceeds the staging limit" in L.lib().vmap_last_error()
    vm.release()
