#!/usr/bin/env python
"""Fused+raycast frames/s at 640x480, 5 mm voxels (plain FP32 single map).

One step = fuse one synthetic RGB-D frame (uint16 mm depth + uint8x3 colour)
into the map and raycast the vertex + normal maps at that frame's pose,
through the library's C ABI (libvmap_b200.so).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 is launched with torch.distributed.run: every rank maps its own seeded
scene (independent maps, no collective on the data path: weak scaling) and
the timed region is the max over ranks of the summed per-step device times.
--impl reference times the reference algorithm's CPU restatement (the
reference is CUDA/Eigen/OpenCV code that cannot be built here) on the host
cores, rank 0 only.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "fused+raycast frames/s @640x480, 5mm voxels: batched vs plain B200; p99 ms"
WORKLOAD = "room_full"
FLUSH_BYTES = 256 << 20  # > 126 MB L2


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="product", choices=["product", "reference"])
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--num-blocks", type=int, default=0, help="override the block pool (small profiling runs)")
    p.add_argument("--batch", type=int, default=32, help="maps per batched step (0 skips the batched arm)")
    p.add_argument("--batch-steps", type=int, default=0, help="timed batched steps (default: --steps // 4)")
    p.add_argument("--batch-blocks", type=int, default=1 << 17, help="block pool per batched map")
    p.add_argument("--uneven", type=int, default=64, help="maps of the uneven batch (0 skips it)")
    p.add_argument("--serving", action="store_true",
                   help="also run the serving sweep (256 sessions, Poisson arrivals, 70/25/5 fuse/raycast/mesh)")
    p.add_argument("--serving-rates", default="100,200,300,400,600")
    p.add_argument("--serving-budgets", default="1.0,0.5", help="device memory budgets, fractions of all sessions' bytes")
    p.add_argument("--serving-requests", type=int, default=1500)
    p.add_argument("--autotune", action="store_true",
                   help="tune the launch shapes first (else a cached or shipped table, if any, is applied)")
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(x, device, world):
    """The maximum of a per-rank number over all ranks (the device time of the
    slowest rank bounds the job): an all-reduce MAX when world > 1."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def all_gather_objects(x, world):
    """Every rank's x, in rank order: one all_gather_object (control data only,
    e.g. free device memory or summaries); [x] on one rank."""
    if world == 1:
        return [x]
    import torch.distributed as dist
    out = [None] * world
    dist.all_gather_object(out, x)
    return out


def job_throughput(units_per_rank, max_total_ms, world):
    """Whole-job units per second: every rank processed units_per_rank units
    within the slowest rank's max_total_ms."""
    return world * units_per_rank / (max_total_ms / 1e3)


def apply_tuning(target, key, args, tune):
    """Launch shapes for `target` (a map or batch): tuned now with --autotune
    (and cached), else the cached or shipped entry for `key`, else defaults.
    Returns (config, source)."""
    from voxelmapping_b200 import autotune as AT
    if args.autotune and tune is not None:
        cfg, table = tune()
        AT.store(key, cfg, {"medians_ms": {f: {str(c): v for c, v in t.items()} for f, t in table.items()}})
        target.set_launch_config(**cfg)
        return cfg, "tuned"
    cfg, src = AT.lookup(key)
    if cfg:
        target.set_launch_config(**cfg)
        return cfg, src
    return target.get_launch_config(), "default"


def percentile(xs, q):
    return float(np.percentile(np.asarray(xs, np.float64), q)) if xs else 0.0


def workload_config(wl, args, extra=None):
    cfg = {"workload": "%s: %dx%d depth (uint16 mm) + rgb, %g mm voxels, 2^%d entries, 2^%d-block pool, "
                       "%s TSDF + weight + uint8x3 colour, figure-8 trajectory; step = fuse one frame + raycast "
                       "vertex/normal maps at its pose" % (wl.name, wl.width, wl.height, wl.voxel_size * 1e3,
                                                           int(np.log2(wl.num_entries)), int(np.log2(wl.num_blocks)),
                                                           wl.voxel_format.upper()),
           "path": "plain single map per GPU", "frames": "%d..%d" % (args.warmup, args.warmup + args.steps - 1),
           "warmup_frames": "0..%d" % (args.warmup - 1), "l2": "flushed between steps (256 MiB write)",
           "parallelism": "independent maps per rank" if args.gpus > 1 else "single GPU"}
    if extra:
        cfg.update(extra)
    return cfg


# ------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap", "utilization.gpu"]

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None

    def __enter__(self):
        try:
            cmd = ["nvidia-smi", "--query-gpu=" + ",".join(self.FIELDS), "--format=csv,noheader,nounits", "-lms",
                   "50"]
            if self.gpu_id is not None:
                cmd += ["-i", str(self.gpu_id)]
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        """Median SM clock and throttle reasons over the samples taken while
        the GPU was busy (utilisation >= 50 %; all samples if none was)."""
        rows = [r.split(", ") for r in getattr(self, "out", "").strip().splitlines() if r.count(",") >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        num = lambda x: float(x) if x.strip().replace(".", "").isdigit() else None
        busy = [r for r in rows if (num(r[9]) or 0.0) >= 50.0] or rows
        sm = [num(r[1]) for r in busy if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in busy for i in range(4) if r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "busy_samples": len(busy) if busy is not rows else 0}


def gpu_index(local_rank):
    """nvidia-smi id of this rank's GPU: its UUID (robust to device remapping)."""
    try:
        import torch
        u = str(torch.cuda.get_device_properties(local_rank).uuid)
        if u:
            return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        pass
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local_rank < len(ids):
            return ids[local_rank]
    return local_rank


# -------------------------------------------------------------- CPU baseline
def cpu_oracle_run(wl, frames, n_threads, seconds=None, steps=None, om=None):
    """Reference algorithm (FP32 restatement, same voxel format) on the host:
    fuse, then raycast + normal map, per frame, like one GPU step. Returns the
    oracle map and per-frame seconds of the two stages."""
    from oracle import oracle as O
    from voxelmapping_b200 import synth
    O.set_threads(n_threads)
    if om is None:
        om = O.OracleMap(wl.width, wl.height, wl.K, wl.num_blocks, wl.voxel_size, storage=wl.voxel_format,
                         max_weight=wl.max_weight, with_color=wl.with_color)
    st = {"fuse": [], "raycast": []}
    t_start = time.perf_counter()
    for d, rgb, pose in frames:
        t0 = time.perf_counter()
        om.fuse(synth.depth_to_metres(d, wl.depth_scale), rgb if wl.with_color else None, pose)
        t1 = time.perf_counter()
        O.compute_normal(om.raycast(pose))
        st["fuse"].append(t1 - t0)
        st["raycast"].append(time.perf_counter() - t1)
        if seconds is not None and time.perf_counter() - t_start > seconds:
            break
        if steps is not None and len(st["fuse"]) >= steps:
            break
    return om, st


def cpu_baseline(wl, scene, frames, threads, seconds=None, skip=0, one_thread_frames=2):
    """The oracle on the host cores: frames/s over `frames` (after `skip`
    untimed ones) with `threads` threads, per-stage p50 / p99, one mesh
    extraction of the resulting map, and the next `one_thread_frames` frames
    on one thread."""
    from oracle import oracle as O
    om, st = cpu_oracle_run(wl, frames, threads, seconds=seconds)
    used = len(st["fuse"])
    fr = [f + r for f, r in zip(st["fuse"], st["raycast"])][skip:]
    ms = lambda xs: {"p50": 1e3 * percentile(xs, 50), "p99": 1e3 * percentile(xs, 99)}
    out = {"value": len(fr) / sum(fr), "unit": "frames/s", "cores": threads, "kind": "port",
           "frames_timed": len(fr), "frame_ms": ms(fr), "fuse_ms": ms(st["fuse"][skip:]),
           "raycast_normals_ms": ms(st["raycast"][skip:])}
    t0 = time.perf_counter()
    n, _, _ = om.polygonize()
    out["mesh"] = {"ms": 1e3 * (time.perf_counter() - t0), "triangles": int(n), "threads": threads,
                   "map_frames": used}
    if one_thread_frames > 0:
        nxt = [frames[i] if i < len(frames) else scene.render(i) for i in range(used, used + one_thread_frames)]
        _, st1 = cpu_oracle_run(wl, nxt, 1, om=om)
        fr1 = [f + r for f, r in zip(st1["fuse"], st1["raycast"])]
        out["one_thread"] = {"frames/s": len(fr1) / sum(fr1), "frame_ms": ms(fr1), "fuse_ms": ms(st1["fuse"]),
                             "raycast_normals_ms": ms(st1["raycast"]),
                             "sample": "frames %d..%d on the same map" % (used, used + len(fr1) - 1)}
        O.set_threads(threads)
    return out


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from voxelmapping_b200 import synth
    wl = synth.WORKLOADS[WORKLOAD]
    scene = synth.Scene(wl)
    frames = [scene.render(i) for i in range(args.warmup + args.steps)]
    threads = os.cpu_count() or 1
    cb = cpu_baseline(wl, scene, frames, threads, skip=args.warmup)
    value = cb["value"]
    cb["sample"] = ("frames %d..%d of %s, fuse + raycast + normals each (every step a full frame)"
                    % (args.warmup, args.warmup + args.steps - 1, WORKLOAD))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value,
            "p50_ms": cb["frame_ms"]["p50"], "p99_ms": cb["frame_ms"]["p99"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": wl.voxel_format,
            "data": "synthetic",
            "config": workload_config(wl, args, {"path": "reference algorithm, CPU restatement (oracle port)"}),
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# -------------------------------------------------------------- batched arm
def run_batched(args, wls, dev, flush, world, distinct_frames=None):
    """One map per workload in `wls` (one voxel format for all), each fed its
    own seeded scene; one vmap_batch_step per step (one launch per stage over
    all maps, graph-replayed on a side stream). With `distinct_frames` F, each
    map renders F frames and the steps cycle through them.

    The same maps' frames are then run through the plain path: FP32 TSDF +
    float weight + colour maps, one map per call (vmap_fuse_depth_rgb +
    vmap_render_scene, six launches per map), same steps, same L2 flush;
    `ratio_vs_plain` compares the two on identical work."""
    import dataclasses

    import torch
    import torch.distributed as dist
    from voxelmapping_b200 import MapBatch, VoxelMapping
    from voxelmapping_b200 import _lib as L
    from voxelmapping_b200 import synth

    B = len(wls)
    K = args.batch_steps or max(4, args.steps // 4)
    W = min(args.warmup, 5)
    nfr = W + K
    F = min(nfr, distinct_frames or nfr)
    depth, rgb, poses, vmaps, nmaps = [], [], [], [], []
    for b, w in enumerate(wls):
        sc = synth.Scene(w)
        d_b = torch.empty((F, w.height, w.width), dtype=torch.int16, device=dev)
        c_b = torch.empty((F, w.height, w.width * 3), dtype=torch.uint8, device=dev) if w.with_color else None
        p_b = np.zeros((F, 16))
        stride = max(1, w.n_poses // max(F, 1)) if F < nfr else 1
        for i in range(F):
            d, c, p = sc.render(i * stride)
            d_b[i].copy_(torch.from_numpy(d.view(np.int16)))
            if c_b is not None:
                c_b[i].copy_(torch.from_numpy(c).reshape(w.height, -1))
            p_b[i] = p.reshape(16)
        del sc
        depth.append(d_b), rgb.append(c_b), poses.append(p_b)
        vmaps.append(torch.empty((w.height, w.width, 4), dtype=torch.float32, device=dev))
        nmaps.append(torch.empty((w.height, w.width, 4), dtype=torch.float32, device=dev))

    def make_maps(fmt_wls):
        maps = []
        for w in fmt_wls:
            vm = VoxelMapping(w.width, w.height, w.K, voxel_format=w.voxel_format, with_color=w.with_color,
                              max_weight=w.max_weight)
            vm.CreateMap(w.num_entries, w.num_blocks, w.voxel_size)
            maps.append(vm)
        return maps

    lib = L.lib()
    side = torch.cuda.Stream(device=dev)
    sp = C.c_void_p(side.cuda_stream)

    def timed(run_step):
        """W untimed + K timed steps on the side stream; per-step ms (max over ranks of the sum)."""
        torch.cuda.synchronize()
        with torch.cuda.stream(side):
            for i in range(W):
                run_step(i)
            side.synchronize()
            if world > 1:
                dist.barrier()
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
            for k in range(K):
                flush.fill_(k & 255)
                ev[k][0].record(side)
                run_step(W + k)
                ev[k][1].record(side)
            side.synchronize()
        step_ms = [a.elapsed_time(b) for a, b in ev]
        return step_ms, max_over_ranks(sum(step_ms), dev, world)

    # --- batched: one vmap_batch_step over all maps per step
    maps = make_maps(wls)
    batch = MapBatch(maps)
    frames = []
    for i in range(nfr):
        fr = (L.BatchFrame * B)()
        for b, w in enumerate(wls):
            f, j = fr[b], i % F
            f.depth_dev, f.depth_type, f.depth_pitch, f.depth_scale = depth[b][j].data_ptr(), L.DEPTH_U16, \
                w.width * 2, w.depth_scale
            if rgb[b] is not None:
                f.rgb_dev, f.rgb_pitch = rgb[b][j].data_ptr(), w.width * 3
            for k in range(16):
                f.pose[k] = poses[b][j, k]
            f.vmap_dev, f.vmap_pitch = vmaps[b].data_ptr(), w.width * 16
            f.nmap_dev, f.nmap_pitch = nmaps[b].data_ptr(), w.width * 16
        frames.append(fr)
    def batch_step(i):
        L.check(lib.vmap_batch_step(batch._h, frames[i % nfr], sp))
    batch_step.stream = side

    def tune():
        from voxelmapping_b200 import autotune as AT
        torch.cuda.synchronize()
        res = AT.tune_batch(batch, batch_step)
        torch.cuda.synchronize()
        for m in maps:  # the timed steps start from empty maps
            m.reset()
        torch.cuda.synchronize()
        return res
    from voxelmapping_b200 import autotune as AT
    key = AT.key_for("batch", wls[0].voxel_format, wls[0].width, wls[0].height, B) if len(
        {(w.width, w.height) for w in wls}) == 1 else AT.key_for("batch", wls[0].voxel_format, 0, 0, B)
    launch_cfg, tune_src = apply_tuning(batch, key, args, tune)
    step_ms, tot = timed(batch_step)
    value = job_throughput(B * K, tot, world)
    pixels = sum(w.width * w.height for w in wls)
    hits = float(sum(torch.isfinite(v[..., 0]).sum().item() for v in vmaps)) / pixels
    stats = [m.stats() for m in maps]
    batch.release()
    for m in maps:
        m.release()

    # --- plain: the same frames, FP32 maps, one map per call
    pwls = [dataclasses.replace(w, voxel_format="f32", max_weight=255) for w in wls]
    pmaps = make_maps(pwls)
    from voxelmapping_b200 import autotune as AT
    for w, m in zip(pwls, pmaps):  # the plain path with its own tuned shapes, where a table has them
        cfg, _ = AT.lookup(AT.key_for("map", w.voxel_format, w.width, w.height))
        if cfg:
            m.set_launch_config(**cfg)
    pargs = [[L.pose_arg(poses[b][j].reshape(4, 4)) for j in range(F)] for b in range(B)]

    def plain_step(i):
        j = i % F
        for b, (w, vm) in enumerate(zip(pwls, pmaps)):
            L.check(lib.vmap_fuse_depth_rgb(vm._map, depth[b][j].data_ptr(), L.DEPTH_U16, w.width * 2, w.depth_scale,
                                            rgb[b][j].data_ptr() if rgb[b] is not None else None, w.width * 3,
                                            pargs[b][j], sp))
            L.check(lib.vmap_render_scene(vm._map, pargs[b][j], vmaps[b].data_ptr(), w.width * 16,
                                          nmaps[b].data_ptr(), w.width * 16, sp))

    p_ms, p_tot = timed(plain_step)
    p_value = job_throughput(B * K, p_tot, world)
    for m in pmaps:
        m.release()
    return {"value": value, "unit": "frames/s", "maps": B, "steps": K, "warmup": W,
            "ms_per_step": tot / K, "p50_ms_per_step": percentile(step_ms, 50),
            "p99_ms_per_step": percentile(step_ms, 99),
            "plain_same_frames": {"value": p_value, "unit": "frames/s", "ms_per_step": p_tot / K,
                                  "p50_ms_per_step": percentile(p_ms, 50), "p99_ms_per_step": percentile(p_ms, 99),
                                  "dtype": "f32",
                                  "path": "FP32 maps, one map per call (vmap_fuse_depth_rgb + vmap_render_scene)"},
            "ratio_vs_plain": value / p_value, "megapixels_per_step": pixels / 1e6, "dtype": wls[0].voxel_format,
            "launch_config": launch_cfg, "tuning": tune_src,
            "hit_fraction_last_step": hits, "error_flags": int(np.bitwise_or.reduce([s["error_flags"] for s in stats])),
            "maps_pool_full": int(sum(1 for s in stats if s["error_flags"] & L.FLAG_POOL_FULL)),
            "allocated_blocks_total": int(sum(s["allocated_blocks"] for s in stats))}


def batched_same_size(args, wl, rank):
    """args.batch maps of the 640x480 / 5 mm workload, FP16 TSDF + uint16
    weight (cap 128) + colour, each its own seeded room and figure-8."""
    import dataclasses
    wlb = dataclasses.replace(wl, voxel_format="f16", max_weight=128, num_blocks=args.batch_blocks)
    wls = [dataclasses.replace(wlb, seed=1000 * (rank + 1) + b) for b in range(args.batch)]
    desc = ("%d maps x 640x480 depth + rgb, 5 mm voxels, FP16 TSDF + uint16 weight (cap 128) + uint8x3 colour, "
            "2^%d-block pool each, each map its own seeded room scene and figure-8; one step = one frame per map "
            "fused + raycast (vmap_batch_step: one launch per stage over all maps, CUDA-graph replay); L2 flushed "
            "between steps" % (args.batch, int(np.log2(wlb.num_blocks))))
    return wls, desc


def batched_uneven(args, rank):
    """args.uneven maps of uneven extent U(1,8) m, voxel size {4,8,12,16} mm,
    resolution {320x240, 640x480, 1280x720}, pools 2^14..2^19, FP16 + colour."""
    from voxelmapping_b200 import synth
    wls = synth.uneven_workloads(args.uneven, seed=rank + 1)
    desc = ("%d maps of uneven extent U(1,8) m, voxel size {4,8,12,16} mm, depth resolution {320x240, 640x480, "
            "1280x720}, pools 2^14..2^19 blocks, FP16 TSDF + uint16 weight (cap 128) + uint8x3 colour, each its own "
            "seeded scene; one step = one frame per map fused + raycast in one vmap_batch_step; each map cycles "
            "through 8 rendered frames; L2 flushed between steps" % args.uneven)
    return wls, desc


# --------------------------------------------------------------- product arm
def run_product(args):
    import torch
    import torch.distributed as dist
    from voxelmapping_b200 import VoxelMapping
    from voxelmapping_b200 import _lib as L
    from voxelmapping_b200 import synth

    rank, world, local = dist_env()
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    wl = synth.WORKLOADS[WORKLOAD]
    import dataclasses
    if args.num_blocks:
        wl = dataclasses.replace(wl, num_blocks=args.num_blocks)
    wl_r = dataclasses.replace(wl, seed=wl.seed + rank)
    scene = synth.Scene(wl_r)
    nfr = args.warmup + args.steps
    frames = [scene.render(i) for i in range(nfr)]
    depth_d = torch.from_numpy(np.stack([f[0] for f in frames]).view(np.int16)).to(dev)
    rgb_d = torch.from_numpy(np.stack([f[1] for f in frames])).to(dev).reshape(nfr, wl.height, wl.width * 3)
    poses = [L.pose_arg(f[2]) for f in frames]
    vm = VoxelMapping(wl.width, wl.height, wl.K, voxel_format=wl.voxel_format, with_color=wl.with_color,
                      max_weight=wl.max_weight)
    vm.CreateMap(wl.num_entries, wl.num_blocks, wl.voxel_size)
    lib = L.lib()
    vmap = torch.empty((wl.height, wl.width, 4), dtype=torch.float32, device=dev)
    nmap = torch.empty_like(vmap)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    counters = torch.zeros((args.steps, 16), dtype=torch.int32, device=dev)
    h = vm._map
    vpitch = wl.width * 16

    def step(i):
        L.check(lib.vmap_fuse_depth_rgb(h, depth_d[i].data_ptr(), L.DEPTH_U16, wl.width * 2, wl.depth_scale,
                                        rgb_d[i].data_ptr(), wl.width * 3, poses[i], sp))
        L.check(lib.vmap_render_scene(h, poses[i], vmap.data_ptr(), vpitch, nmap.data_ptr(), vpitch, sp))

    def tune():
        # on a scratch map of the same configuration, so the timed map's
        # frames and state stay those of the measured workload
        from voxelmapping_b200 import autotune as AT
        tmp = VoxelMapping(wl.width, wl.height, wl.K, voxel_format=wl.voxel_format, with_color=wl.with_color,
                           max_weight=wl.max_weight)
        tmp.CreateMap(wl.num_entries, wl.num_blocks, wl.voxel_size)

        def tstep(i):
            j = i % nfr
            L.check(lib.vmap_fuse_depth_rgb(tmp._map, depth_d[j].data_ptr(), L.DEPTH_U16, wl.width * 2,
                                            wl.depth_scale, rgb_d[j].data_ptr(), wl.width * 3, poses[j], sp))
            L.check(lib.vmap_render_scene(tmp._map, poses[j], vmap.data_ptr(), vpitch, nmap.data_ptr(), vpitch, sp))
        best, table = AT.tune_map(tmp, tstep, n_steps=8)
        best["mesh_ctas_per_sm"], table["mesh_ctas_per_sm"] = AT.tune_mesh(tmp)
        tmp.release()
        return best, table
    from voxelmapping_b200 import autotune as AT
    launch_cfg, tune_src = apply_tuning(vm, AT.key_for("map", wl.voxel_format, wl.width, wl.height), args, tune)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    L.check(lib.vmap_timing_enable(h, args.steps * 8))
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    # clocks are sampled from here through the e2e and batched arms' timed work
    # (the plain loop alone lasts only tens of milliseconds)
    clk = ClockSampler(gpu_index(local)).__enter__()
    for k in range(args.steps):
        flush.fill_(k & 255)
        ev[k][0].record()
        step(args.warmup + k)
        ev[k][1].record()
        L.check(lib.vmap_copy_counters(h, counters[k].data_ptr(), sp))
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    stage_ms = (C.c_double * 7)()
    stage_n = (C.c_uint32 * 7)()
    L.check(lib.vmap_timing_read(h, stage_ms, stage_n))
    L.check(lib.vmap_timing_enable(h, 0))
    total_ms = sum(step_ms)
    max_total_ms = max_over_ranks(total_ms, dev, world)
    if world > 1:
        dist.barrier()
    value = job_throughput(args.steps, max_total_ms, world)
    st = vm.stats()
    cnt = counters.cpu().numpy()
    vis = cnt[:, 1].astype(np.float64)
    alloc = np.minimum(cnt[:, 0], wl.num_blocks).astype(np.float64)

    # --- roofline: algorithmic bytes per launch of each stage (bench model) --
    P = wl.width * wl.height
    s_vox = L.lib().vmap_block_bytes(L.FORMAT_NAMES[wl.voxel_format], int(wl.with_color)) / 512.0
    s_tsdf = {"ref": 3, "f32": 8, "f16": 4, "i16": 4}[wl.voxel_format]
    stage_bytes = {
        "alloc": P * 2 + vis.mean() * 32,                         # depth read + one probe sector per block
        "visibility": alloc.mean() * 8 + vis.mean() * 4,          # block keys + visible list
        "fuse": vis.mean() * (512 * s_vox * 2 + 12) + P * 5,      # block RMW + depth/colour images
        "zrange": alloc.mean() * 8,
        "raycast": vis.mean() * 512 * s_tsdf + P * 16,            # touched blocks' tsdf+weight + vertex map
        "normals": P * 32,
    }
    stages = {}
    for i, name in enumerate(L.STAGES):
        if stage_n[i]:
            per = stage_ms[i] / stage_n[i]
            b = stage_bytes.get(name)
            stages[name] = {"launches": int(stage_n[i]), "ms_per_launch": per,
                            "share": stage_ms[i] / max(sum(stage_ms), 1e-9),
                            "alg_bytes": b, "gbs": (b / (per * 1e-3) / 1e9) if b else None}
    dom = max(stages, key=lambda k: stages[k]["ms_per_launch"] * stages[k]["launches"])
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    traffic, l2_pct, traffic_capture, scale = None, None, None, None
    tf = ROOT / "profiles" / "ncu_traffic.json"
    if tf.exists():
        entry = json.loads(tf.read_text()).get(dom, {})
        traffic_capture, l2_pct = entry.get("dram_bytes_per_launch"), entry.get("l2_throughput_pct")
        # the capture is a smaller frame: scale its DRAM bytes to this run's
        # launches by the units the kernel processes (visible blocks)
        units = entry.get("visible_blocks_at_capture")
        if traffic_capture is not None and units:
            scale = float(vis.mean()) / units
            traffic = traffic_capture * scale
    roof = {"kernel": dom, "bound": "hbm", "achieved": stages[dom]["gbs"], "peak": peak, "peak_source": peak_src,
            "unit": "GB/s", "frac": stages[dom]["gbs"] / peak, "traffic": traffic,
            "alg_bytes_per_launch": stages[dom]["alg_bytes"],
            "traffic_at_capture": traffic_capture, "traffic_scale": scale,
            # a latency-bound kernel: its L2 throughput (% of peak, one ncu capture) beside the HBM fraction
            "l2_throughput_pct_ncu": l2_pct}

    line = {"metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_total_ms / args.steps,
            "p50_ms": percentile(step_ms, 50), "p99_ms": percentile(step_ms, 99), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": wl.voxel_format, "data": "synthetic",
            "config": workload_config(wl, args), "roofline": roof, "stages": stages,
            "gpu_launches": int(sum(stage_n)),
            "launch_config": launch_cfg, "tuning": tune_src,
            "map": {"allocated_blocks": int(st["allocated_blocks"]), "visible_blocks_mean": float(vis.mean()),
                    "error_flags": int(st["error_flags"])}}

    # --- mesh: marching cubes over every allocated block of the map -------
    # (Polygonize, marching_cubes.cu:251-305): a counting pass, then the emit
    # pass into buffers of that size; each timed alone after an L2 flush.
    cnt_d = torch.zeros(1, dtype=torch.int32, device=dev)
    mev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    L.check(lib.vmap_polygonize(h, None, None, 0, cnt_d.data_ptr(), sp))  # untimed: loads the kernels
    flush.fill_(1)
    mev[0].record()
    L.check(lib.vmap_polygonize(h, None, None, 0, cnt_d.data_ptr(), sp))
    mev[1].record()
    torch.cuda.synchronize()
    ntri = int(cnt_d.item())
    mverts = torch.empty((max(ntri, 1), 9), dtype=torch.float32, device=dev)
    mnorms = torch.empty_like(mverts)
    flush.fill_(2)
    mev[2].record()
    L.check(lib.vmap_polygonize(h, mverts.data_ptr(), mnorms.data_ptr(), ntri, None, sp))
    mev[3].record()
    torch.cuda.synchronize()
    count_ms, emit_ms = mev[0].elapsed_time(mev[1]), mev[2].elapsed_time(mev[3])
    nblk = float(st["allocated_blocks"])
    halo = (9.0 / 8.0) ** 3  # a block's 8^3 cubes read a 9^3 voxel neighbourhood
    mesh_bytes = nblk * 512 * s_tsdf * halo + ntri * 72
    line["mesh"] = {"triangles": ntri, "blocks": int(nblk), "count_pass_ms": count_ms, "emit_pass_ms": emit_ms,
                    "alg_bytes_emit": mesh_bytes, "emit_gbs": mesh_bytes / (emit_ms * 1e-3) / 1e9,
                    "emit_frac_of_peak": mesh_bytes / (emit_ms * 1e-3) / 1e9 / peak}
    del mverts, mnorms

    # --- e2e: same steps through the host-buffer C ABI calls --------------
    if not args.no_e2e:
        depth_h = torch.from_numpy(np.stack([f[0] for f in frames]).view(np.int16)).pin_memory()
        rgb_h = torch.from_numpy(np.stack([f[1] for f in frames])).pin_memory()
        vmap_h = torch.empty((wl.height, wl.width, 4), dtype=torch.float32).pin_memory()
        nmap_h = torch.empty_like(vmap_h).pin_memory()
        vm.reset()

        def step_host(i):
            L.check(lib.vmap_fuse_host(h, depth_h[i].data_ptr(), L.DEPTH_U16, wl.depth_scale, rgb_h[i].data_ptr(),
                                       poses[i], sp))
            L.check(lib.vmap_render_scene_host(h, poses[i], vmap_h.data_ptr(), nmap_h.data_ptr(), sp))

        for i in range(args.warmup):
            step_host(i)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        for k in range(args.steps):
            flush.fill_(k & 255)
            ev2[k][0].record()
            step_host(args.warmup + k)
            ev2[k][1].record()
        torch.cuda.synchronize()
        e_ms = [a.elapsed_time(b) for a, b in ev2]
        e_tot = max_over_ranks(sum(e_ms), dev, world)
        sync_path = {"value": job_throughput(args.steps, e_tot, world), "unit": "frames/s",
                     "p50_ms": percentile(e_ms, 50), "p99_ms": percentile(e_ms, 99),
                     "path": "vmap_fuse_host + vmap_render_scene_host per frame (copy in, kernels, copy out, "
                             "one after another), L2 flushed between frames outside each frame's events"}

        # the pipelined host path: copies of neighbouring frames overlap each
        # other's kernels; the whole run is timed, L2 flush included
        vm.reset()
        outs = [(torch.empty((wl.height, wl.width, 4), dtype=torch.float32).pin_memory(),
                 torch.empty((wl.height, wl.width, 4), dtype=torch.float32).pin_memory()) for _ in range(2)]
        hframes = []
        for i in range(nfr):
            f = L.HostFrame()
            f.depth_host, f.depth_type, f.depth_scale = depth_h[i].data_ptr(), L.DEPTH_U16, wl.depth_scale
            f.rgb_host = rgb_h[i].data_ptr()
            f.pose[:] = list(poses[i])
            f.vmap_host, f.nmap_host = outs[i & 1][0].data_ptr(), outs[i & 1][1].data_ptr()
            hframes.append(f)
        for i in range(args.warmup):
            L.check(lib.vmap_frame_host_async(h, C.byref(hframes[i]), sp))
        L.check(lib.vmap_host_wait(h, sp))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        fl0, fl1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fl0.record()
        for k in range(args.steps):
            flush.fill_(k & 255)
        fl1.record()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        for k in range(args.steps):
            flush.fill_(k & 255)
            L.check(lib.vmap_frame_host_async(h, C.byref(hframes[args.warmup + k]), sp))
        L.check(lib.vmap_host_wait(h, sp))
        t1.record()
        torch.cuda.synchronize()
        p_tot = max_over_ranks(t0.elapsed_time(t1), dev, world)
        line["e2e"] = {"value": job_throughput(args.steps, p_tot, world), "unit": "frames/s",
                       "h2d_bytes_per_step": P * 2 + P * 3, "d2h_bytes_per_step": 2 * P * 16,
                       "ms_per_step": p_tot / args.steps, "flush_ms_per_step": fl0.elapsed_time(fl1) / args.steps,
                       "path": "vmap_frame_host_async per frame + vmap_host_wait: pinned host buffers, depth + "
                               "colour in and vertex + normal maps out on two copy streams, overlapping the "
                               "neighbouring frames' kernels; the 256 MiB L2 flush between frames is inside the "
                               "timed region",
                       "sync_path": sync_path}

    # --- batched arm: many maps per step ------------------------------------
    if args.batch > 0 or args.uneven > 0:
        vm.release()
    if args.batch > 0:
        wls, desc = batched_same_size(args, wl, rank)
        line["batched"] = run_batched(args, wls, dev, flush, world)
        line["batched"]["config"] = desc
    if args.uneven > 0:
        wls, desc = batched_uneven(args, rank)
        line["batched_uneven"] = run_batched(args, wls, dev, flush, world, distinct_frames=8)
        line["batched_uneven"]["config"] = desc

    clk.__exit__(None, None, None)
    line["clocks"] = clk.summary()
    line["clocks"]["window"] = "plain, e2e and batched timed work"

    # --- CPU baseline: oracle on the host cores (rank 0, N = 1 only) -------
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cb = cpu_baseline(wl, scene, frames, threads, seconds=args.cpu_seconds)
        cb["sample"] = ("frames 0..%d of %s (fuse + raycast + normals each, FP32 reference-algorithm "
                        "restatement, %d threads)" % (cb["frames_timed"] - 1, WORKLOAD, threads))
        line["cpu_baseline"] = cb
    if args.serving:
        from voxelmapping_b200 import serving as S
        rates = [float(r) for r in args.serving_rates.split(",")]
        line["serving"] = {"config": "256 sessions per GPU of uneven extent / voxel size / resolution (FP16 + "
                                     "colour; with N GPUs the job's N x 256 sessions are partitioned over them by free "
                                     "device memory), 4 pre-rendered frames each in pinned host memory; Poisson "
                                     "arrivals at each offered rate per GPU, %d requests per GPU, 70/25/5 "
                                     "fuse/raycast/mesh; raycasts return vertex + normal maps to pinned host memory, "
                                     "meshes their triangles; latency = completion - arrival, wall clock; summaries "
                                     "merged over the ranks" % args.serving_requests, "runs": []}
        gather = lambda x: all_gather_objects(x, world)  # noqa: E731
        for frac in [float(b) for b in args.serving_budgets.split(",")]:
            res, ex = S.run_serving(n_sessions=256, rates=rates, count=args.serving_requests, budget_frac=frac,
                                    warmup=500, seed=0, rank=rank, world=world, all_gather=gather)
            ex.release()
            parts = gather(res)
            for k in range(len(res)):
                r = S.merge_summaries([p[k] for p in parts])
                r["budget_frac"] = frac
                line["serving"]["runs"].append({key: v for key, v in r.items() if not key.startswith("_")})
    if rank == 0:
        print(json.dumps(line), flush=True)
    vm.release()
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_product(args)


if __name__ == "__main__":
    main()
