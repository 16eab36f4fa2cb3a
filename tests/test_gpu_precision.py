"""Precision sweep of the voxel storage formats against the FP64 oracle.

The 640x480 / 5 mm room sequence (24 frames) is fused into one map per format
- FP32 TSDF + float weight, FP16 TSDF + uint16 weight, int16 TSDF (x32767 of
the truncation) + uint16 weight, each with the weight capped at 128, and the
reference's own format (int16 + uint8 weight capped at 255) - all with colour.
Fusion and interpolation run in FP32 in every format. Each map is compared
with the oracle's FP64 map (same weight cap, unquantised double storage):
TSDF RMS over voxels observed in both, raycast depth error at the last pose,
symmetric Hausdorff distance between the mesh vertex sets, plus bytes per
voxel and the fuse kernel's achieved bandwidth (algorithmic bytes / time).

Set VMAP_PRECISION_OUT to a path to write the table as JSON."""
import ctypes as C
import dataclasses
import json
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.common import aligned_maps, block_keys, raycast_stats
from voxelmapping_b200 import VoxelMapping
from voxelmapping_b200 import _lib as L
from voxelmapping_b200 import synth

pytestmark = pytest.mark.gpu

WL = dataclasses.replace(synth.WORKLOADS["room_full"], num_blocks=1 << 16)
FRAMES = list(range(0, 48, 2))
FORMATS = [("f32", 128), ("f16", 128), ("i16", 128), ("ref", 255)]


def hausdorff_mm(a, b):
    from scipy.spatial import cKDTree
    a = np.unique(a.reshape(-1, 3), axis=0)
    b = np.unique(b.reshape(-1, 3), axis=0)
    d_ab = cKDTree(b).query(a, workers=-1)[0]
    d_ba = cKDTree(a).query(b, workers=-1)[0]
    return 1e3 * float(max(d_ab.max(), d_ba.max())), 1e3 * float(np.percentile(np.concatenate([d_ab, d_ba]), 99))


@pytest.fixture(scope="module")
def sweep():
    scene = synth.Scene(WL)
    frames = [scene.render(i) for i in FRAMES]
    pose = frames[-1][2]
    ref64 = {}
    for cap in sorted({c for _, c in FORMATS}):
        o = O.OracleMap(WL.width, WL.height, WL.K, WL.num_blocks, WL.voxel_size, precision=O.FP64, storage="f32",
                        max_weight=cap, with_color=False)
        for d, _, p in frames:
            o.fuse(synth.depth_to_metres(d), None, p)
        n, verts, _ = o.polygonize()
        ref64[cap] = (o, o.raycast(pose), verts)
    # the reference arithmetic itself (FP32 oracle, FP32 storage) against FP64:
    # how many pixels the algorithm in single precision puts beyond 1 mm
    o32 = O.OracleMap(WL.width, WL.height, WL.K, WL.num_blocks, WL.voxel_size, storage="f32", max_weight=128)
    for d, _, p in frames:
        o32.fuse(synth.depth_to_metres(d), None, p)
    v32 = o32.raycast(pose)
    both32 = np.isfinite(v32[..., 0]) & np.isfinite(ref64[128][1][..., 0])
    dz32 = np.abs(v32[..., 2] - ref64[128][1][..., 2])[both32]
    oracle32 = {"over_1mm": int((dz32 > 1e-3).sum()), "max_mm": float(dz32.max() * 1e3)}
    lib = L.lib()
    rows = {}
    f32_map = None  # FP32-storage export: the others minus it isolate storage quantisation
    P = WL.width * WL.height
    for fmt, cap in FORMATS:
        vm = VoxelMapping(WL.width, WL.height, WL.K, voxel_format=fmt, with_color=True, max_weight=cap)
        vm.CreateMap(WL.num_entries, WL.num_blocks, WL.voxel_size)
        L.check(lib.vmap_timing_enable(vm._map, 8 * len(frames)))
        vis = []
        for d, c, p in frames:
            vm.FuseDepthAndImage(torch.from_numpy(c).cuda().reshape(WL.height, -1),
                                 torch.from_numpy(d.view(np.int16)).cuda(), p)
            vis.append(vm.stats()["visible_blocks"])
        torch.cuda.synchronize()
        ms = (C.c_double * 7)()
        cnt = (C.c_uint32 * 7)()
        L.check(lib.vmap_timing_read(vm._map, ms, cnt))
        L.check(lib.vmap_timing_enable(vm._map, 0))
        fuse_i = L.STAGES.index("fuse")
        fuse_us = 1e3 * ms[fuse_i] / cnt[fuse_i]
        bpv = lib.vmap_block_bytes(L.FORMAT_NAMES[fmt], 1) / 512.0
        fuse_bytes = np.mean(vis) * (512 * bpv * 2 + 12) + P * 5
        o, v64, verts64 = ref64[cap]
        g, r = aligned_maps(vm, o)
        # FP32 and FP64 allocation can round a sample into a different block: compare common blocks
        _, ig, ir = np.intersect1d(block_keys(g["coords"]), block_keys(r["coords"]), return_indices=True)
        only_gpu, only_64 = len(g["coords"]) - len(ig), len(r["coords"]) - len(ir)
        gw, rw = g["weight"][ig], r["weight"][ir]
        both = (gw > 0) & (rw > 0)
        err = g["tsdf"][ig][both].astype(np.float64) - r["tsdf"][ir][both]
        mu_mm = 4 * WL.voxel_size * 1e3
        if fmt == "f32":
            f32_map = g
        qw = (g["weight"] > 0) & (f32_map["weight"] > 0)
        assert np.array_equal(g["coords"], f32_map["coords"]) and np.array_equal(g["weight"], f32_map["weight"]), fmt
        q = g["tsdf"][qw].astype(np.float64) - f32_map["tsdf"][qw]
        v = vm.RenderScene(None, pose).cpu().numpy()
        ray = raycast_stats(v, v64)
        hit2 = np.isfinite(v[..., 0]) & np.isfinite(v64[..., 0])
        over = int((np.abs(v[..., 2] - v64[..., 2])[hit2] > 1e-3).sum())
        k, verts, _ = vm.Polygonize()
        h_max, h_p99 = hausdorff_mm(verts, verts64)
        rows[fmt] = {"weight_cap": cap, "bytes_per_voxel": bpv, "blocks": int(len(g["coords"])),
                     "tsdf_rms": float(np.sqrt(np.mean(err ** 2))), "tsdf_rms_mm": float(np.sqrt(np.mean(err ** 2))) * mu_mm,
                     "tsdf_max_abs": float(np.abs(err).max()), "tsdf_p99_abs": float(np.percentile(np.abs(err), 99)),
                     "quant_rms_vs_f32_storage": float(np.sqrt(np.mean(q ** 2))),
                     "quant_max_vs_f32_storage": float(np.abs(q).max()),
                     "blocks_only_gpu": int(only_gpu), "blocks_only_fp64": int(only_64),
                     "weight_mismatch": float((gw != rw).mean()),
                     "raycast_dz_max_mm": ray["dz_max_mm"], "raycast_dz_mean_mm": ray["dz_mean_mm"],
                     "raycast_dz_p999_mm": ray["dz_p999_mm"], "raycast_within_1mm": ray["frac_within_1mm"],
                     "raycast_over_1mm": over, "raycast_hit_pixels": int(hit2.sum()),
                     "oracle_fp32_over_1mm": oracle32["over_1mm"], "oracle_fp32_dz_max_mm": oracle32["max_mm"],
                     "raycast_hit_mismatch": ray["mismatch"], "triangles": int(k),
                     "mesh_hausdorff_mm": h_max, "mesh_hausdorff_p99_mm": h_p99,
                     "fuse_us": fuse_us, "fuse_gbs": float(fuse_bytes / (fuse_us * 1e-6) / 1e9)}
        vm.release()
    print()
    for fmt, r in rows.items():
        print(fmt, {k: (round(x, 6) if isinstance(x, float) else x) for k, x in r.items()})
    out = os.environ.get("VMAP_PRECISION_OUT")
    if out:
        with open(out, "w") as f:
            json.dump({"workload": "room_full 640x480, 5 mm, frames %s, 2^16-block pool" % FRAMES, "rows": rows}, f,
                      indent=1)
    return rows


@pytest.mark.parametrize("fmt", [f for f, _ in FORMATS])
def test_raycast_depth_within_1mm_of_fp64(sweep, fmt):
    # Depth within 1 mm of FP64 at the 99.9th percentile, with no more pixels
    # beyond 1 mm than the reference arithmetic itself (the FP32 oracle) puts
    # there (+ 0.02 % of the hits): the reference's two fixed refinement
    # steps after the zero crossing (ray_tracing.cu:381-393) do not converge
    # at oblique incidence, so single precision and double precision can stop
    # on neighbouring samples and end millimetres apart on a few pixels.
    r = sweep[fmt]
    assert r["raycast_within_1mm"] >= 0.999 and r["raycast_dz_p999_mm"] <= 1.0, r
    assert r["raycast_dz_mean_mm"] <= 0.2 and r["raycast_hit_mismatch"] <= 0.01, r
    assert r["raycast_over_1mm"] <= 2 * r["oracle_fp32_over_1mm"] + 2e-4 * r["raycast_hit_pixels"], r


def test_tsdf_error_ordered_by_storage_precision(sweep):
    # Against FP64 the error is dominated by the few voxels where FP32 and FP64
    # arithmetic take different decisions (nearest pixel, truncation cut-off),
    # the same in every format. Against FP32 storage (identical arithmetic and
    # weights) only the storage quantisation remains: int16 truncates toward
    # zero to 1/32767 of the truncation distance on every update (packFloat,
    # map_struct.h:72-75), so the error drifts over a running average to a few
    # steps; FP16 rounds to nearest at 2^-11 relative.
    for fmt in ("f32", "f16", "i16", "ref"):
        assert sweep[fmt]["tsdf_rms"] < 0.01 and sweep[fmt]["tsdf_p99_abs"] < 0.01, sweep[fmt]
    assert sweep["f32"]["quant_rms_vs_f32_storage"] == 0.0
    assert 0 < sweep["i16"]["quant_rms_vs_f32_storage"] < 2e-4 and sweep["i16"]["quant_max_vs_f32_storage"] < 1e-3
    assert 0 < sweep["f16"]["quant_rms_vs_f32_storage"] < 5e-4 and sweep["f16"]["quant_max_vs_f32_storage"] < 2e-3
    for fmt in ("f32", "f16", "i16"):
        r = sweep[fmt]
        assert r["weight_mismatch"] <= 2e-3 and r["blocks_only_gpu"] + r["blocks_only_fp64"] <= 2e-3 * r["blocks"], r
        assert r["mesh_hausdorff_p99_mm"] < 0.5, (fmt, r)
