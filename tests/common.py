"""Shared helpers for the GPU parity tests: run the product (through the C ABI)
and the CPU oracle on the same seeded frames and line their maps up."""
import numpy as np

from oracle import oracle as O
from voxelmapping_b200 import VoxelMapping, synth


def block_keys(coords):
    c = coords.astype(np.int64) + (1 << 20)
    return (c[:, 0] << 42) | (c[:, 1] << 21) | c[:, 2]


def make_pair(wl, fmt="ref", color=False, num_blocks=None, raycast_mode=0, max_weight=255, num_buckets=0,
              width=None, height=None, K=None, num_entries=None):
    w = width or wl.width
    h = height or wl.height
    K = wl.K if K is None else K
    nb = num_blocks or wl.num_blocks
    vm = VoxelMapping(w, h, K, voxel_format=fmt, with_color=color, max_weight=max_weight,
                      raycast_mode=raycast_mode, num_buckets=num_buckets)
    vm.CreateMap(wl.num_entries if num_entries is None else num_entries, nb, wl.voxel_size)
    om = O.OracleMap(w, h, K, nb, wl.voxel_size, storage=fmt, max_weight=max_weight, with_color=color)
    return vm, om


def to_gpu_depth(depth_u16):
    import torch
    return torch.from_numpy(np.ascontiguousarray(depth_u16).view(np.int16)).cuda()


def fuse_both(vm, om, depth_u16, rgb, pose, scale=0.001):
    """Fuse one frame in both; returns (gpu stats, oracle result)."""
    import torch
    d = to_gpu_depth(depth_u16)
    if rgb is not None and vm.with_color:
        c = torch.from_numpy(np.ascontiguousarray(rgb)).cuda().reshape(rgb.shape[0], -1)
        vm.FuseDepthAndImage(c, d, pose, depth_scale=scale)
    else:
        vm.FuseDepth(d, pose, depth_scale=scale)
    st = vm.stats()
    orc = om.fuse(synth.depth_to_metres(depth_u16, scale), rgb if om.with_color else None, pose)
    return st, orc


def aligned_maps(vm, om):
    """GPU and oracle blocks sorted by coordinates (their pool orders differ)."""
    g = vm.export_blocks()
    o = om.export()
    gi = np.argsort(block_keys(g["coords"]))
    oi = np.argsort(block_keys(o["coords"]))
    g = {k: (v[gi] if v is not None else None) for k, v in g.items()}
    o = {k: (v[oi] if v is not None else None) for k, v in o.items()}
    return g, o


def raycast_stats(v_gpu, v_orc):
    hg = np.isfinite(v_gpu[..., 0])
    ho = np.isfinite(v_orc[..., 0])
    both = hg & ho
    dz = np.abs(v_gpu[..., 2][both] - v_orc[..., 2][both])
    dp = np.linalg.norm(v_gpu[..., :3][both] - v_orc[..., :3][both], axis=-1)
    return {"hits_gpu": int(hg.sum()), "hits_oracle": int(ho.sum()), "mismatch": float((hg ^ ho).mean()),
            "dz_max_mm": float(dz.max() * 1e3) if dz.size else 0.0,
            "dz_p999_mm": float(np.percentile(dz, 99.9) * 1e3) if dz.size else 0.0,
            "dz_mean_mm": float(dz.mean() * 1e3) if dz.size else 0.0,
            "dp_p99_mm": float(np.percentile(dp, 99) * 1e3) if dp.size else 0.0,
            "frac_within_1mm": float((dp <= 1e-3).mean()) if dp.size else 1.0}


def sorted_rows(a):
    a = np.ascontiguousarray(a)
    v = a.view(np.dtype((np.void, a.dtype.itemsize * a.shape[1]))).ravel()
    return a[np.argsort(v, kind="stable")]
