"""Map snapshots (vmap_snapshot_save / vmap_snapshot_load): a map saved to host
or device memory and loaded into another map (different bucket count, stale
content) must export, render, fuse further and mesh bit-identically to the
original; invalid snapshots are refused and leave the target untouched."""
import dataclasses

import numpy as np
import pytest
import torch

from tests.common import block_keys, sorted_rows
from voxelmapping_b200 import VoxelMapping
from voxelmapping_b200 import _lib as L
from voxelmapping_b200 import synth

pytestmark = pytest.mark.gpu

WL = synth.WORKLOADS["room_small"]


def new_map(fmt="ref", color=True, blocks=1 << 16, buckets=0, vs=None):
    # num_entries 8 keeps the bucket count at `buckets` (default 0.9 * blocks)
    vm = VoxelMapping(WL.width, WL.height, WL.K, voxel_format=fmt, with_color=color, num_buckets=buckets)
    vm.CreateMap(8, blocks, vs or WL.voxel_size)
    return vm


def fuse(vm, scene, idx):
    for i in idx:
        d, c, p = scene.render(i)
        vm.FuseDepthAndImage(torch.from_numpy(c).cuda().reshape(WL.height, -1),
                             torch.from_numpy(d.view(np.int16)).cuda(), p)
    return p


def same_export(a, b, ordered=True):
    """Equal block sets; `ordered`: also in the same pool order (a load keeps
    the order, blocks allocated later take slots in scheduling order)."""
    ea, eb = a.export_blocks(), b.export_blocks()
    ia = np.arange(len(ea["coords"])) if ordered else np.argsort(block_keys(ea["coords"]))
    ib = np.arange(len(eb["coords"])) if ordered else np.argsort(block_keys(eb["coords"]))
    for k in ("coords", "tsdf", "weight", "rgb"):
        assert np.array_equal(ea[k][ia], eb[k][ib]), k


def same_render(a, b, pose):
    na, nb = (torch.empty((WL.height, WL.width, 4), device="cuda") for _ in range(2))
    va = a.RenderScene(None, pose, nmap=na).cpu().numpy()
    vb = b.RenderScene(None, pose, nmap=nb).cpu().numpy()
    assert np.array_equal(np.nan_to_num(va, nan=-9.0), np.nan_to_num(vb, nan=-9.0))
    assert np.array_equal(np.nan_to_num(na.cpu().numpy(), nan=-9.0), np.nan_to_num(nb.cpu().numpy(), nan=-9.0))
    assert np.isfinite(va[..., 0]).mean() > 0.3


@pytest.mark.parametrize("fmt", ["ref", "f16"])
def test_snapshot_round_trip_is_bit_identical(fmt):
    scene = synth.Scene(WL)
    a = new_map(fmt)
    pose = fuse(a, scene, range(0, 12, 2))
    host = a.save_snapshot()
    assert host.nbytes == a.snapshot_bytes()
    hdr = host[:64].view(np.uint32)
    n = a.stats()["allocated_blocks"]
    assert bytes(host[:8]) == b"VMAPSNAP" and hdr[2] == 1 and hdr[7] == n > 1000
    dev = torch.empty(host.nbytes + 100, dtype=torch.uint8, device="cuda")
    assert np.array_equal(a.save_snapshot(dev).cpu().numpy(), host)

    # target with 4x the buckets and stale content from another scene
    b = new_map(fmt, buckets=4 * int(0.9 * (1 << 16)) + 3)
    assert b.get_config()["num_buckets"] != a.get_config()["num_buckets"]
    fuse(b, synth.Scene(dataclasses.replace(WL, seed=5)), range(0, 40, 4))
    assert b.stats()["allocated_blocks"] > n
    b.load_snapshot(host)
    assert b.stats()["allocated_blocks"] == n and b.stats()["error_flags"] == 0
    same_export(a, b)
    same_render(a, b, pose)

    # load from device memory into a fresh map, then keep fusing all three
    c = new_map(fmt)
    c.load_snapshot(dev[:host.nbytes])
    for m in (a, b, c):
        pose = fuse(m, scene, range(13, 30, 3))
    same_export(a, b, ordered=False)
    same_export(a, c, ordered=False)
    same_render(a, c, pose)
    ka, va, na = a.Polygonize()
    kc, vc, nc = c.Polygonize()
    assert ka == kc > 1000
    assert np.array_equal(sorted_rows(np.concatenate([va, na], 1)), sorted_rows(np.concatenate([vc, nc], 1)))


def test_snapshot_refusals_leave_the_map_untouched():
    scene = synth.Scene(WL)
    a = new_map()
    fuse(a, scene, range(0, 6, 2))
    snap = a.save_snapshot()
    n = a.stats()["allocated_blocks"]

    t = new_map()
    fuse(t, scene, [20])
    before = t.export_blocks()

    def refused(target, buf, what):
        with pytest.raises(L.VmapError):
            target.load_snapshot(buf)
        if target is t:
            after = t.export_blocks()
            for k in ("coords", "tsdf", "weight", "rgb"):
                assert np.array_equal(before[k], after[k]), (what, k)

    bad = snap.copy(); bad[0] ^= 1
    refused(t, bad, "magic")
    refused(t, snap[:-1], "truncated")
    refused(t, snap[:40], "short header")
    refused(new_map(blocks=n - 1), snap, "capacity")
    refused(new_map(fmt="f16"), snap, "format")
    refused(new_map(color=False), snap, "colour")
    refused(new_map(vs=WL.voxel_size * 1.5), snap, "voxel size")

    small = np.empty(10, np.uint8)
    with pytest.raises(L.VmapError):
        a.save_snapshot(small)


def test_snapshot_with_bad_keys_or_too_few_buckets_resets_the_target():
    scene = synth.Scene(WL)
    a = new_map()
    fuse(a, scene, range(0, 6, 2))
    snap = a.save_snapshot()
    keys = snap[64:64 + 8 * 4].view(np.uint64)
    dup = snap.copy()
    dup[64 + 8:64 + 16] = dup[64:72]  # block 1 gets block 0's key
    t = new_map()
    with pytest.raises(L.VmapError):
        t.load_snapshot(dup)
    assert t.stats()["allocated_blocks"] == 0 and t.stats()["error_flags"] == 0
    assert keys[0] != keys[1]
    # 8 buckets hold at most 32 keys: the rebuild runs out of probes
    tiny = new_map(buckets=8)
    with pytest.raises(L.VmapError):
        tiny.load_snapshot(snap)
    assert tiny.stats()["allocated_blocks"] == 0
    # the reset map still works
    fuse(t, scene, [0])
    assert t.stats()["allocated_blocks"] > 0 and t.stats()["error_flags"] == 0
