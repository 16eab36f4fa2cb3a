"""Serving on the GPU (voxelmapping_b200.serving): sessions are evicted to
pinned host memory and restored while requests run; every request completes,
and each session's map and its last raycast are bit-identical to replaying
that session's fuse requests alone on a fresh map."""
import numpy as np
import pytest
import torch

from tests.common import block_keys
from voxelmapping_b200 import VoxelMapping
from voxelmapping_b200 import serving as S

pytestmark = pytest.mark.gpu


def solo_replay(wl, frames, n_fused):
    vm = VoxelMapping(wl.width, wl.height, wl.K, voxel_format=wl.voxel_format, with_color=wl.with_color,
                      max_weight=wl.max_weight)
    vm.CreateMap(wl.num_entries, wl.num_blocks, wl.voxel_size)
    for k in range(n_fused):
        d, c, _ = frames[k % len(frames)]
        vm.FuseDepthAndImage(c.cuda(), d.cuda(), frames[k % len(frames)][2])
    return vm


def test_serving_with_eviction_matches_solo_replay():
    results, ex = S.run_serving(n_sessions=6, rates=(4000.0,), count=160, budget_frac=0.4, n_frames=3, seed=2,
                                warmup=0, keep_results=True, pool_scale=4)
    try:
        summ = results[0]
        reqs = summ["_requests"]
        assert all(np.isfinite(r.done) and r.done >= r.arrival for r in reqs)
        assert summ["evictions"] > 0 and summ["restores"] > 6
        assert summ["fuse"]["n"] > 80 and summ["raycast"]["n"] > 20
        for s, wl in enumerate(ex.wls):
            n_fused = ex.next_frame[s]
            solo = solo_replay(wl, ex.frames[s], n_fused)
            if s in ex.maps:
                served = ex.maps[s]
            else:
                served = VoxelMapping(wl.width, wl.height, wl.K, voxel_format=wl.voxel_format,
                                      with_color=wl.with_color, max_weight=wl.max_weight)
                served.CreateMap(wl.num_entries, wl.num_blocks, wl.voxel_size)
                served.load_snapshot(ex.snaps[s])
            ea, eb = served.export_blocks(), solo.export_blocks()
            ia, ib = np.argsort(block_keys(ea["coords"])), np.argsort(block_keys(eb["coords"]))
            for k in ("coords", "tsdf", "weight", "rgb"):
                assert np.array_equal(ea[k][ia], eb[k][ib]), (s, k)
            assert served.stats()["error_flags"] == 0, s
            rays = [r for r in reqs if r.session == s and r.kind == "raycast"]
            if not rays:
                continue
            vmap, nmap, nf = rays[-1].result
            if nf == 0:
                assert np.isnan(vmap.numpy()[..., 0]).all()
                continue
            solo2 = solo_replay(wl, ex.frames[s], nf)
            nm = torch.empty((wl.height, wl.width, 4), device="cuda")
            v = solo2.RenderScene(None, ex.frames[s][(nf - 1) % len(ex.frames[s])][2], nmap=nm)
            torch.cuda.synchronize()
            assert np.array_equal(np.nan_to_num(v.cpu().numpy(), nan=-9.0), np.nan_to_num(vmap.numpy(), nan=-9.0)), s
            assert np.array_equal(np.nan_to_num(nm.cpu().numpy(), nan=-9.0), np.nan_to_num(nmap.numpy(), nan=-9.0)), s
    finally:
        ex.release()


def test_session_bytes_cover_the_maps():
    from voxelmapping_b200 import synth
    wls = synth.uneven_workloads(4, seed=5)
    ex = S.GpuExecutor(wls, [[] for _ in wls])
    for s, wl in enumerate(wls):
        ex.restore(s)
        st = ex.maps[s].stats()
        bufs = sum(t.numel() * t.element_size() for t in ex.bufs[s])
        assert st["device_bytes"] + bufs <= ex.session_bytes(s), (s, st["device_bytes"] + bufs, ex.session_bytes(s))
    ex.release()
