#!/usr/bin/env python
"""Fused+raycast frames/s at 640x480, 5 mm voxels (plain FP32 single map).

One step = fuse one synthetic RGB-D frame (uint16 mm depth + uint8x3 colour)
into the map and raycast the vertex + normal maps at that frame's pose,
through the library's C ABI (libvmap_b200.so).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 is launched with torch.distributed.run: every rank maps its own seeded
scene (independent maps, no collective on the data path: weak scaling) and
the timed region is the max over ranks of the summed per-step device times.
Before the warm-up, --prefix frames (default 100) are fused untimed, so the
timed frames see a steady-state map rather than a young one.

--impl reference times the reference algorithm's CPU restatement (the oracle
port: the reference has no CPU implementation) on the host cores, rank 0
only, on the same frames; beside it (extra key) the reference's own CUDA
build, compiled from its sources against project-written Eigen/OpenCV
subsets (oracle/_ref), timed on the GPU as the plain drop-in comparison.
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


def l2_flush_buffer(dev):
    """The L2 flush buffer: FLUSH_BYTES of float32, so that fill_ writes it
    with 16-byte vector stores (a uint8 buffer is filled 4 bytes per store,
    at about half the speed, which the pipelined e2e run counts in full)."""
    import torch
    return torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="product", choices=["product", "reference"])
    p.add_argument("--prefix", type=int, default=100,
                   help="frames fused untimed before the warm-up (steady-state map)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--num-blocks", type=int, default=0, help="override the block pool (small profiling runs)")
    p.add_argument("--batch", type=int, default=32, help="maps per batched step (0 skips the batched arm)")
    p.add_argument("--batch-steps", type=int, default=0, help="timed batched steps (default: --steps // 4)")
    p.add_argument("--batch-blocks", type=int, default=1 << 17, help="block pool per batched map")
    p.add_argument("--uneven", type=int, default=64, help="maps of the uneven batch (0 skips it)")
    p.add_argument("--no-serving", action="store_true",
                   help="skip the serving sweep (256 sessions, Poisson arrivals, 70/25/5 fuse/raycast/mesh)")
    p.add_argument("--serving-rates", default="600,200",
                   help="offered requests/s per GPU, one per budget (or one for all), comma-separated")
    p.add_argument("--serving-budgets", default="1.0,0.5", help="device memory budgets, fractions of all sessions' bytes")
    p.add_argument("--serving-requests", type=int, default=600)
    p.add_argument("--serving-warmup", type=int, default=200)
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
           "path": "plain single map per GPU",
           "frames": "%d..%d" % (args.prefix + args.warmup, args.prefix + args.warmup + args.steps - 1),
           "prefix_frames": "0..%d fused untimed (steady-state map)" % (args.prefix - 1) if args.prefix else "none",
           "warmup_frames": "%d..%d" % (args.prefix, args.prefix + args.warmup - 1),
           "l2": "flushed between steps (256 MiB write)",
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


def bind_to_gpu_cpus(local_rank):
    """Restricts this process to the CPUs NVML reports as local to the rank's
    GPU (its NUMA node), so pinned host buffers and the threads that drive the
    copies sit next to the GPU's PCIe link, as a deployment would place them.
    Returns the previous CPU set (to restore for host-only work), or None when
    NVML gives no affinity."""
    try:
        import pynvml
        pynvml.nvmlInit()
        try:
            h = pynvml.nvmlDeviceGetHandleByUUID(str(gpu_index(local_rank)))
            words = pynvml.nvmlDeviceGetCpuAffinity(h, (os.cpu_count() + 63) // 64)
        finally:
            pynvml.nvmlShutdown()
        cpus = {64 * i + b for i, w in enumerate(words) for b in range(64) if (int(w) >> b) & 1}
        before = os.sched_getaffinity(0)
        cpus &= before
        if not cpus or cpus == before:
            return None
        os.sched_setaffinity(0, cpus)
        return before
    except Exception:
        return None


# -------------------------------------------------------------- CPU baseline
def cpu_oracle_run(wl, frames, n_threads, seconds=None, steps=None, om=None, precision=0, counts=None):
    """Reference algorithm (the oracle in FP32 reference arithmetic, or FP64,
    same voxel format) on the host: fuse, then raycast + normal map, per
    frame, like one GPU step. Returns the oracle map and per-frame seconds of
    the two stages; with `counts` (a dict of lists) also the frame's visible
    blocks, the unique blocks its allocation touched (A) and the unique
    blocks its rays read (U)."""
    from oracle import oracle as O
    from voxelmapping_b200 import synth
    O.set_threads(n_threads)
    if om is None:
        om = O.OracleMap(wl.width, wl.height, wl.K, wl.num_blocks, wl.voxel_size, storage=wl.voxel_format,
                         max_weight=wl.max_weight, with_color=wl.with_color, precision=precision)
    st = {"fuse": [], "raycast": []}
    t_start = time.perf_counter()
    for d, rgb, pose in frames:
        t0 = time.perf_counter()
        r = om.fuse(synth.depth_to_metres(d, wl.depth_scale), rgb if wl.with_color else None, pose)
        t1 = time.perf_counter()
        O.compute_normal(om.raycast(pose))
        st["fuse"].append(t1 - t0)
        st["raycast"].append(time.perf_counter() - t1)
        if counts is not None:
            counts["visible"].append(r["visible"])
            counts["alloc_touched"].append(om.last_alloc_blocks())
            counts["ray_blocks"].append(om.last_raycast_blocks())
        if seconds is not None and time.perf_counter() - t_start > seconds:
            break
        if steps is not None and len(st["fuse"]) >= steps:
            break
    return om, st


def oracle_prefix(wl, frames, n_threads, precision=0):
    """An oracle map with `frames` fused (untimed, fusion only): the same
    steady-state map the GPU arm's prefix builds."""
    from oracle import oracle as O
    from voxelmapping_b200 import synth
    O.set_threads(n_threads)
    om = O.OracleMap(wl.width, wl.height, wl.K, wl.num_blocks, wl.voxel_size, storage=wl.voxel_format,
                     max_weight=wl.max_weight, with_color=wl.with_color, precision=precision)
    for d, rgb, pose in frames:
        om.fuse(synth.depth_to_metres(d, wl.depth_scale), rgb if wl.with_color else None, pose)
    return om


def cpu_baseline(wl, scene, frames, threads, seconds=None, skip=0, one_thread_frames=2, prefix=0):
    """The oracle on the host cores, after fusing the first `prefix` frames
    untimed: frames/s over the next frames (after `skip` untimed ones,
    bounded by `seconds`) with `threads` threads in the reference's FP32
    arithmetic, per-stage p50 / p99, the unique blocks allocation touched
    (A) and rays read (U) per frame, one mesh extraction of the resulting map,
    the next `one_thread_frames` frames on one thread, and the FP64 accuracy
    oracle timed the same way on a third of the time."""
    from oracle import oracle as O
    ms = lambda xs: {"p50": 1e3 * percentile(xs, 50), "p99": 1e3 * percentile(xs, 99)}  # noqa: E731
    t0 = time.perf_counter()
    om = oracle_prefix(wl, frames[:prefix], threads)
    prefix_s = time.perf_counter() - t0
    counts = {"visible": [], "alloc_touched": [], "ray_blocks": []}
    om, st = cpu_oracle_run(wl, frames[prefix:], threads, seconds=seconds, om=om, counts=counts)
    used = prefix + len(st["fuse"])
    fr = [f + r for f, r in zip(st["fuse"], st["raycast"])][skip:]
    out = {"value": len(fr) / sum(fr), "unit": "frames/s", "cores": threads, "kind": "port",
           "precision": "fp32 (the reference's own arithmetic)", "frames_timed": len(fr), "frame_ms": ms(fr),
           "fuse_ms": ms(st["fuse"][skip:]), "raycast_normals_ms": ms(st["raycast"][skip:]),
           "prefix_frames_untimed": prefix, "prefix_fuse_s": prefix_s,
           "oracle_counts_mean": {k: float(np.mean(v[skip:] or v)) for k, v in counts.items()}}
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
    del om
    # the FP64 accuracy oracle (the double-precision transcription) on the same frames
    o64 = oracle_prefix(wl, frames[:prefix], threads, precision=1)
    _, s64 = cpu_oracle_run(wl, frames[prefix:], threads, seconds=(seconds or 15.0) / 3, om=o64)
    f64 = [f + r for f, r in zip(s64["fuse"], s64["raycast"])]
    f64 = f64[skip:] or f64
    out["fp64"] = {"value": len(f64) / sum(f64), "unit": "frames/s", "cores": threads, "frames_timed": len(f64),
                   "frame_ms": ms(f64), "fuse_ms": ms(s64["fuse"]), "raycast_normals_ms": ms(s64["raycast"])}
    return out


def reference_cuda_build(args, wl, frames):
    """The reference's own CUDA build (oracle/_ref: src/*.cu compiled against
    project-written Eigen/OpenCV subsets) timed on the GPU: the class's path,
    FuseDepthAndImage (depth in metres + colour) then RenderScene and
    computeNormal per step, after the same prefix; device time per step with
    CUDA events on the default stream (the reference synchronises the device
    between its kernels, which the events include), L2 flushed between
    steps; and end to end from pinned host buffers (depth + colour in, vertex
    + normal maps out) with the copies inside the timed region."""
    try:
        import torch
        from oracle import refbuild as RB
    except Exception as e:  # pragma: no cover - import failure is reported
        return {"unavailable": "import failed: %s" % e}
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    if not RB.available():
        return {"unavailable": "reference build missing (make -C oracle ref with the reference sources)"}
    dev = torch.device("cuda", 0)
    H, W = wl.height, wl.width
    nfr = len(frames)
    depth_m = [torch.from_numpy(f[0].astype(np.float32) * np.float32(wl.depth_scale)).to(dev) for f in frames]
    rgb_d = [torch.from_numpy(np.ascontiguousarray(f[1])).to(dev) for f in frames]
    poses = [np.asarray(f[2], np.float32) for f in frames]
    rm = RB.RefMap(W, H, wl.K, wl.num_entries, wl.num_blocks, wl.voxel_size, with_color=True)
    lib = RB.lib()
    vmap = torch.empty((H, W, 4), dtype=torch.float32, device=dev)
    nmap = torch.empty_like(vmap)
    flush = l2_flush_buffer(dev)
    pp = [np.ascontiguousarray(p.reshape(16)) for p in poses]
    pc = [p.ctypes.data_as(C.POINTER(C.c_float)) for p in pp]

    def step(i, d, c):
        RB._check(lib.ref_fuse(rm._h, d.data_ptr(), W * 4, c.data_ptr(), W * 3, pc[i], 0, None), "ref_fuse")
        RB._check(lib.ref_render(rm._h, vmap.data_ptr(), W * 16, pc[i]), "ref_render")
        RB._check(lib.ref_compute_normal(vmap.data_ptr(), W * 16, nmap.data_ptr(), W * 16, W, H), "ref_compute_normal")

    P, K, Wm = args.prefix, args.steps, args.warmup
    for i in range(P):
        RB._check(lib.ref_fuse(rm._h, depth_m[i].data_ptr(), W * 4, rgb_d[i].data_ptr(), W * 3, pc[i], 0, None),
                  "ref_fuse")
    for i in range(P, P + Wm):
        step(i, depth_m[i], rgb_d[i])
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    for k in range(K):
        i = P + Wm + k
        flush.fill_(k & 255)
        ev[k][0].record()
        step(i, depth_m[i], rgb_d[i])
        ev[k][1].record()
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in ev]
    out = {"value": K / (sum(ms) / 1e3), "unit": "frames/s", "ms_per_step": sum(ms) / K,
           "p50_ms": percentile(ms, 50), "p99_ms": percentile(ms, 99), "kind": "reference",
           "path": "reference CUDA sources (src/*.cu) built for sm_100a against Eigen/OpenCV subsets; "
                   "FuseDepthAndImage + RenderScene (CheckVisibleBlocks, ProjectRenderingBlocks, ray march) + "
                   "computeNormal per step, VoxelRGB storage (int16 TSDF + uint8 weight + colour)"}
    # end to end: pinned host depth (float metres, as the reference's API
    # takes it) + colour in, vertex + normal maps out
    rm.reset()
    dh = [t.cpu().pin_memory() for t in depth_m]
    ch = [t.cpu().pin_memory() for t in rgb_d]
    vh = torch.empty((H, W, 4), dtype=torch.float32).pin_memory()
    nh = torch.empty_like(vh).pin_memory()
    dd, cd = torch.empty_like(depth_m[0]), torch.empty_like(rgb_d[0])
    for i in range(P):
        RB._check(lib.ref_fuse(rm._h, depth_m[i].data_ptr(), W * 4, rgb_d[i].data_ptr(), W * 3, pc[i], 0, None),
                  "ref_fuse")

    def step_host(i):
        dd.copy_(dh[i], non_blocking=True)
        cd.copy_(ch[i], non_blocking=True)
        step(i, dd, cd)
        vh.copy_(vmap, non_blocking=True)
        nh.copy_(nmap, non_blocking=True)

    for i in range(P, P + Wm):
        step_host(i)
    torch.cuda.synchronize()
    e2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    for k in range(K):
        flush.fill_(k & 255)
        e2[k][0].record()
        step_host(P + Wm + k)
        e2[k][1].record()
    torch.cuda.synchronize()
    ems = [a.elapsed_time(b) for a, b in e2]
    out["e2e"] = {"value": K / (sum(ems) / 1e3), "unit": "frames/s", "p50_ms": percentile(ems, 50),
                  "p99_ms": percentile(ems, 99), "h2d_bytes_per_step": W * H * (4 + 3),
                  "d2h_bytes_per_step": 2 * W * H * 16}
    rm.close()
    return out


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from voxelmapping_b200 import synth
    wl = synth.WORKLOADS[WORKLOAD]
    scene = synth.Scene(wl)
    frames = [scene.render(i) for i in range(args.prefix + args.warmup + args.steps)]
    threads = os.cpu_count() or 1
    cb = cpu_baseline(wl, scene, frames, threads, skip=args.warmup, prefix=args.prefix)
    value = cb["value"]
    cb["sample"] = ("frames %d..%d of %s after %d untimed prefix frames, fuse + raycast + normals each (every "
                    "step a full frame), FP32 reference arithmetic" % (args.prefix + args.warmup,
                                                                       args.prefix + args.warmup + args.steps - 1,
                                                                       WORKLOAD, args.prefix))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value,
            "p50_ms": cb["frame_ms"]["p50"], "p99_ms": cb["frame_ms"]["p99"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": wl.voxel_format,
            "data": "synthetic",
            "config": workload_config(wl, args, {"path": "reference algorithm, CPU restatement (oracle port)"}),
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    try:
        bind_to_gpu_cpus(0)  # as the product arm: host threads and pinned buffers next to the GPU
        line["reference_cuda_build"] = reference_cuda_build(args, wl, frames)
    except Exception as e:  # reported, not fatal: the CPU port is the arm's value
        line["reference_cuda_build"] = {"unavailable": "failed: %s" % e}
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
    from voxelmapping_b200 import autotune as AT
    key = AT.key_for("batch", wls[0].voxel_format, wls[0].width, wls[0].height, B) if len(
        {(w.width, w.height) for w in wls}) == 1 else AT.key_for("batch", wls[0].voxel_format, 0, 0, B)

    def batched(schedule=None):
        """Fresh maps, the same frames: the tuned launch shapes (schedule None)
        or those shapes with batch_schedule = schedule."""
        maps = make_maps(wls)
        batch = MapBatch(maps)

        def batch_step(i):
            L.check(lib.vmap_batch_step(batch._h, frames[i % nfr], sp))
        batch_step.stream = side

        def tune():
            torch.cuda.synchronize()
            res = AT.tune_batch(batch, batch_step)
            torch.cuda.synchronize()
            for m in maps:  # the timed steps start from empty maps
                m.reset()
            torch.cuda.synchronize()
            return res
        if schedule is None:
            launch_cfg, tune_src = apply_tuning(batch, key, args, tune)
        else:
            batch.set_launch_config(batch_schedule=schedule)
            launch_cfg, tune_src = None, None
        step_ms, tot = timed(batch_step)
        hits = float(sum(torch.isfinite(v[..., 0]).sum().item() for v in vmaps)) / pixels
        stats = [m.stats() for m in maps]
        cfg = batch.get_launch_config()
        batch.release()
        for m in maps:
            m.release()
        return step_ms, tot, hits, stats, launch_cfg or cfg, tune_src, cfg["batch_schedule"]

    pixels = sum(w.width * w.height for w in wls)
    step_ms, tot, hits, stats, launch_cfg, tune_src, sched = batched()
    value = job_throughput(B * K, tot, world)
    # the other schedule on the same frames (1: one launch per stage, 2: one persistent launch)
    o_ms, o_tot, _, o_stats, _, _, o_sched = batched(3 - sched)
    other = {"batch_schedule": o_sched, "value": job_throughput(B * K, o_tot, world), "unit": "frames/s",
             "ms_per_step": o_tot / K, "p50_ms_per_step": percentile(o_ms, 50),
             "error_flags": int(np.bitwise_or.reduce([s["error_flags"] for s in o_stats]))}

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
            "launch_config": launch_cfg, "tuning": tune_src, "batch_schedule": sched, "other_schedule": other,
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
    resolution {320x240, 640x480, 1280x720}, pools 2^14..2^19, FP16 + colour.
    Each pool is twice the generator's surface-area estimate (capped at 2^19
    blocks), so that no map runs out of blocks over the timed frames."""
    import dataclasses
    from voxelmapping_b200 import synth
    wls = [dataclasses.replace(w, num_blocks=min(2 * w.num_blocks, 1 << 19), num_entries=min(2 * w.num_entries, 1 << 21))
           for w in synth.uneven_workloads(args.uneven, seed=rank + 1)]
    desc = ("%d maps of uneven extent U(1,8) m, voxel size {4,8,12,16} mm, depth resolution {320x240, 640x480, "
            "1280x720}, pools 2^14..2^19 blocks (twice the surface-area estimate), FP16 TSDF + uint16 weight (cap 128) "
            "+ uint8x3 colour, each its own seeded scene; one step = one new frame per map (consecutive poses) fused + "
            "raycast in one vmap_batch_step; L2 flushed between steps" % args.uneven)
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
    host_cpus = bind_to_gpu_cpus(local)  # the full CPU set, restored for the CPU baseline
    dev = torch.device("cuda", local)
    wl = synth.WORKLOADS[WORKLOAD]
    import dataclasses
    if args.num_blocks:
        wl = dataclasses.replace(wl, num_blocks=args.num_blocks)
    wl_r = dataclasses.replace(wl, seed=wl.seed + rank)
    scene = synth.Scene(wl_r)
    P0 = args.prefix
    nfr = P0 + args.warmup + args.steps
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
    flush = l2_flush_buffer(dev)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    counters = torch.zeros((2, args.steps, 16), dtype=torch.int32, device=dev)  # timed loop, stage-timing pass
    h = vm._map
    vpitch = wl.width * 16

    def fuse_only(i):
        L.check(lib.vmap_fuse_depth_rgb(h, depth_d[i].data_ptr(), L.DEPTH_U16, wl.width * 2, wl.depth_scale,
                                        rgb_d[i].data_ptr(), wl.width * 3, poses[i], sp))

    def step(i):
        fuse_only(i)
        L.check(lib.vmap_render_scene(h, poses[i], vmap.data_ptr(), vpitch, nmap.data_ptr(), vpitch, sp))

    def prefix():
        """Frames 0 .. prefix-1 fused untimed: a steady-state map."""
        for i in range(P0):
            fuse_only(i)
        torch.cuda.synchronize()

    def tune():
        # on a scratch map of the same configuration, so the timed map's
        # frames and state stay those of the measured workload
        from voxelmapping_b200 import autotune as AT
        tmp = VoxelMapping(wl.width, wl.height, wl.K, voxel_format=wl.voxel_format, with_color=wl.with_color,
                           max_weight=wl.max_weight)
        tmp.CreateMap(wl.num_entries, wl.num_blocks, wl.voxel_size)
        # every trial fuses and renders the same frame after the same prefix,
        # so the candidates are compared on one workload (the blocks a frame
        # sees and its rays do not change when it is fused again)
        for j in range(P0):
            L.check(lib.vmap_fuse_depth_rgb(tmp._map, depth_d[j].data_ptr(), L.DEPTH_U16, wl.width * 2,
                                            wl.depth_scale, rgb_d[j].data_ptr(), wl.width * 3, poses[j], sp))
        j0 = P0

        def tstep(i):
            L.check(lib.vmap_fuse_depth_rgb(tmp._map, depth_d[j0].data_ptr(), L.DEPTH_U16, wl.width * 2,
                                            wl.depth_scale, rgb_d[j0].data_ptr(), wl.width * 3, poses[j0], sp))
            L.check(lib.vmap_render_scene(tmp._map, poses[j0], vmap.data_ptr(), vpitch, nmap.data_ptr(), vpitch,
                                          sp))
        best, table = AT.tune_map(tmp, tstep, n_steps=8)
        best["mesh_ctas_per_sm"], table["mesh_ctas_per_sm"] = AT.tune_mesh(tmp)
        tmp.release()
        return best, table
    from voxelmapping_b200 import autotune as AT
    launch_cfg, tune_src = apply_tuning(vm, AT.key_for("map", wl.voxel_format, wl.width, wl.height), args, tune)

    prefix()
    for i in range(args.warmup):
        step(P0 + i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    # clocks are sampled from here through the e2e and batched arms' timed work
    # (the plain loop alone lasts only tens of milliseconds)
    clk = ClockSampler(gpu_index(local)).__enter__()
    for k in range(args.steps):
        flush.fill_(k & 255)
        ev[k][0].record()
        step(P0 + args.warmup + k)
        ev[k][1].record()
        L.check(lib.vmap_copy_counters(h, counters[0, k].data_ptr(), sp))
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    max_total_ms = max_over_ranks(total_ms, dev, world)
    if world > 1:
        dist.barrier()
    value = job_throughput(args.steps, max_total_ms, world)
    # per-stage device times in a second pass over the same frames from the
    # same prefix: the events that bracket every launch cost about 15 % of a
    # step and keep the stages' launches from overlapping, so the timed loop
    # above runs without them; the stage bytes below use this pass's counters
    vm.reset()
    prefix()
    for i in range(args.warmup):
        step(P0 + i)
    L.check(lib.vmap_timing_enable(h, args.steps * 8))
    for k in range(args.steps):
        flush.fill_(k & 255)
        step(P0 + args.warmup + k)
        L.check(lib.vmap_copy_counters(h, counters[1, k].data_ptr(), sp))
    torch.cuda.synchronize()
    stage_ms = (C.c_double * 7)()
    stage_n = (C.c_uint32 * 7)()
    L.check(lib.vmap_timing_read(h, stage_ms, stage_n))
    L.check(lib.vmap_timing_enable(h, 0))
    st = vm.stats()
    cnt_all = counters.cpu().numpy()
    cnt = cnt_all[1]
    vis = cnt[:, 1].astype(np.float64)
    alloc = np.minimum(cnt[:, 0], wl.num_blocks).astype(np.float64)
    vis_timed = cnt_all[0][:, 1].astype(np.float64)

    # stage timings now; their algorithmic bytes (and the roofline) once the
    # CPU leg has counted the oracle's U and A on the same frames
    P = wl.width * wl.height
    s_vox = L.lib().vmap_block_bytes(L.FORMAT_NAMES[wl.voxel_format], int(wl.with_color)) / 512.0
    s_tsdf = {"ref": 4, "f32": 8, "f16": 4, "i16": 4}[wl.voxel_format]  # the voxel word rays read
    stage_time = {name: (int(stage_n[i]), stage_ms[i] / stage_n[i]) for i, name in enumerate(L.STAGES) if stage_n[i]}
    total_stage_ms = max(sum(stage_ms), 1e-9)
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0

    line = {"metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_total_ms / args.steps,
            "p50_ms": percentile(step_ms, 50), "p99_ms": percentile(step_ms, 99), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": wl.voxel_format, "data": "synthetic",
            "config": workload_config(wl, args), "roofline": None, "stages": None,
            # the timed loop launches per step the kernels the stage-timing pass counts per step
            "gpu_launches": int(sum(stage_n)),
            "launch_config": launch_cfg, "tuning": tune_src,
            "map": {"allocated_blocks": int(st["allocated_blocks"]), "visible_blocks_mean": float(vis_timed.mean()),
                    "visible_blocks_mean_stage_pass": float(vis.mean()), "error_flags": int(st["error_flags"])}}
    line["config"]["host_cpus"] = (
        "the %d CPUs local to the GPU (NVML affinity) for the GPU arms, all %d for the CPU baseline"
        % (len(os.sched_getaffinity(0)), len(host_cpus)) if host_cpus else
        "all host CPUs (NVML reports no narrower affinity for the GPU)")

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
        prefix()

        def step_host(i):
            L.check(lib.vmap_fuse_host(h, depth_h[i].data_ptr(), L.DEPTH_U16, wl.depth_scale, rgb_h[i].data_ptr(),
                                       poses[i], sp))
            L.check(lib.vmap_render_scene_host(h, poses[i], vmap_h.data_ptr(), nmap_h.data_ptr(), sp))

        for i in range(args.warmup):
            step_host(P0 + i)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        for k in range(args.steps):
            flush.fill_(k & 255)
            ev2[k][0].record()
            step_host(P0 + args.warmup + k)
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
        prefix()
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
            L.check(lib.vmap_frame_host_async(h, C.byref(hframes[P0 + i]), sp))
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
            L.check(lib.vmap_frame_host_async(h, C.byref(hframes[P0 + args.warmup + k]), sp))
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
        line["batched_uneven"] = run_batched(args, wls, dev, flush, world)
        line["batched_uneven"]["config"] = desc

    clk.__exit__(None, None, None)
    line["clocks"] = clk.summary()
    line["clocks"]["window"] = "plain, e2e and batched timed work"

    # --- CPU baseline: oracle on the host cores (rank 0, N = 1 only) -------
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        if host_cpus:  # the CPU leg gets every host core
            os.sched_setaffinity(0, host_cpus)
        threads = os.cpu_count() or 1
        cb = cpu_baseline(wl, scene, frames, threads, seconds=args.cpu_seconds, prefix=args.prefix)
        if host_cpus:
            bind_to_gpu_cpus(local)
        cb["sample"] = ("frames %d..%d of %s after %d untimed prefix frames (fuse + raycast + normals each, FP32 "
                        "reference-algorithm restatement, %d threads; FP64 beside)"
                        % (args.prefix, args.prefix + cb["frames_timed"] - 1, WORKLOAD, args.prefix, threads))
        line["cpu_baseline"] = cb
    # --- roofline: algorithmic bytes per launch of each stage ---------------
    # P pixels, V visible blocks and B allocated blocks (device counters of the
    # timed steps), A blocks the allocation touched and U blocks rays read
    # (the oracle's counts on the same frames, when the CPU leg ran; else the
    # visible blocks stand in, an upper bound), S bytes per voxel (word +
    # colour), S_w the word rays read; hash bucket 64 B, block key 8 B, list
    # entry 4 B.
    oc = (line.get("cpu_baseline") or {}).get("oracle_counts_mean")
    V, B = float(vis.mean()), float(alloc.mean())
    A = oc["alloc_touched"] if oc else V
    U = oc["ray_blocks"] if oc else V
    src = "oracle counts on the same frames" if oc else "visible blocks (no oracle count: upper bound)"
    stage_bytes = {
        "alloc": P * 2 + A * 64,                          # depth + one bucket probe per touched block
        "visibility": B * 8 + V * 4,                      # block keys + visible list
        "fuse": V * (512 * s_vox * 2 + 4 + 8) + P * 5,    # block RMW + list + key + depth/colour
        "zrange": B * 8,
        "raycast": U * 512 * s_tsdf + P * 16,             # blocks rays read + vertex map
        "normals": P * 32,
    }
    stages = {}
    for name, (n_l, per) in stage_time.items():
        bts = stage_bytes.get(name)
        g = bts / (per * 1e-3) / 1e9 if bts else None
        stages[name] = {"launches": n_l, "ms_per_launch": per, "share": n_l * per / total_stage_ms,
                        "alg_bytes": bts, "gbs": g, "frac": g / peak if g else None}
    # whole-frame aggregates: the fused frame
    # P(2+3) + A E_alloc + B E_list + 2 V 512 S + 4 V, the rendered frame
    # U 512 S_w + P 32 (vertex + normal maps)
    agg = {"fused_frame": (("alloc", "visibility", "fuse"),
                           P * 5 + A * 64 + B * 8 + V * 512 * s_vox * 2 + V * 4),
           "rendered_frame": (("zrange", "raycast", "normals"), U * 512 * s_tsdf + P * 32)}
    for name, (parts, bts) in agg.items():
        t = sum(stages[p_]["ms_per_launch"] for p_ in parts if p_ in stages)
        g = bts / (t * 1e-3) / 1e9
        stages[name] = {"stages": list(parts), "ms": t, "alg_bytes": bts, "gbs": g, "frac": g / peak}
    dom = max(stage_time, key=lambda k: stage_time[k][0] * stage_time[k][1])
    traffic, l2_pct, traffic_capture, scale = None, None, None, None
    tf = ROOT / "profiles" / "ncu_traffic.json"
    if tf.exists():
        entry = json.loads(tf.read_text()).get(dom, {})
        traffic_capture, l2_pct = entry.get("dram_bytes_per_launch"), entry.get("l2_throughput_pct")
        # the capture is a smaller frame: scale its DRAM bytes to this run's
        # launches by the units the kernel processes
        units = entry.get("units_at_capture") or entry.get("visible_blocks_at_capture")
        unit_now = U if entry.get("units_at_capture") else V
        if traffic_capture is not None and units:
            scale = float(unit_now) / units
            traffic = traffic_capture * scale
    line["roofline"] = {"kernel": dom, "bound": "hbm", "achieved": stages[dom]["gbs"], "peak": peak,
                        "peak_source": peak_src, "unit": "GB/s", "frac": stages[dom]["frac"], "traffic": traffic,
                        "alg_bytes_per_launch": stages[dom]["alg_bytes"], "units": {"P": P, "V": V, "B": B,
                                                                                   "A": A, "U": U, "source": src},
                        "traffic_at_capture": traffic_capture, "traffic_scale": scale,
                        # a latency-bound kernel: its L2 throughput (% of peak, one ncu capture) beside
                        "l2_throughput_pct_ncu": l2_pct}
    line["stages"] = stages
    line["mesh"]["emit_frac_of_peak"] = line["mesh"]["emit_gbs"] / peak

    if not args.no_serving:
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
        budgets = [float(b) for b in args.serving_budgets.split(",")]
        for bi, frac in enumerate(budgets):
            # one rate per budget when as many are given, else every rate at every budget
            rts = [rates[bi]] if len(rates) == len(budgets) else rates
            res, ex = S.run_serving(n_sessions=256, rates=rts, count=args.serving_requests, budget_frac=frac,
                                    warmup=args.serving_warmup, seed=0, rank=rank, world=world, all_gather=gather)
            ex.release()
            parts = gather(res)
            for k in range(len(res)):
                r = S.merge_summaries([p[k] for p in parts])
                r["budget_frac"] = frac
                line["serving"]["runs"].append({key: v for key, v in r.items() if not key.startswith("_")})
    line["headline"] = headline(line)
    if rank == 0:
        print(json.dumps(line), flush=True)
    vm.release()
    if world > 1:
        dist.destroy_process_group()


def headline(line):
    """The numbers a reader looks for first, compact, as the line's last key."""
    r = lambda x, n=3: None if x is None else round(float(x), n)  # noqa: E731
    h = {"plain_fps": r(line["value"], 1), "plain_p50_ms": r(line["p50_ms"]), "plain_p99_ms": r(line["p99_ms"]),
         "e2e_fps": r((line.get("e2e") or {}).get("value"), 1),
         "raycast_roofline_frac": r((line.get("roofline") or {}).get("frac"), 4)}
    for arm in ("batched", "batched_uneven"):
        b = line.get(arm)
        if b:
            h[arm] = {"fps": r(b["value"], 1), "plain_same_frames_fps": r(b["plain_same_frames"]["value"], 1),
                      "ratio_vs_plain": r(b["ratio_vs_plain"]), "p50_ms_per_step": r(b["p50_ms_per_step"]),
                      "p99_ms_per_step": r(b["p99_ms_per_step"]), "maps_pool_full": b["maps_pool_full"],
                      "batch_schedule": b.get("batch_schedule"),
                      "other_schedule_fps": r((b.get("other_schedule") or {}).get("value"), 1)}
    sv = line.get("serving")
    if sv:
        h["serving"] = [{"budget": x.get("budget_frac"), "offered_rps": r(x.get("offered_rps"), 1),
                         "served_rps": r(x.get("throughput_rps"), 1),
                         "p50_ms": {k: r(x[k]["p50_ms"], 2) for k in ("fuse", "raycast", "mesh") if k in x},
                         "p99_ms": {k: r(x[k]["p99_ms"], 2) for k in ("fuse", "raycast", "mesh") if k in x}}
                        for x in sv["runs"]]
    cb = line.get("cpu_baseline")
    if cb:
        h["cpu_fp32_fps"] = r(cb["value"], 2)
        h["cpu_fp64_fps"] = r((cb.get("fp64") or {}).get("value"), 2)
    return h


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_product(args)


if __name__ == "__main__":
    main()
