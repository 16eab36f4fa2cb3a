"""Launch-shape autotuner for the fuse / raycast / mesh stages.

The library's kernels stride over their work items, so a stage's grid (CTAs
per SM, vmap_launch_config) changes only its time. The tuner measures the
candidates on the caller's own data and keeps the fastest:

* a single map (`tune_map`): coordinate descent on whole-step time, every
  stage's grid and then the ray marcher's tile shape (width 8, 16 or 4 of a
  32-ray tile), threads per CTA (256 or 128) and tile order, one field at a
  time with the rest fixed at their best; a field's candidates are visited
  round-robin several times and each keeps its median. Per-stage events would
  serialise the stage launches that programmatic dependent launch overlaps,
  so only whole steps are timed;
* a batch (`tune_batch`): the stages run inside one recorded CUDA graph, so
  the whole step is timed, one stage at a time (coordinate descent);
* the mesh grid (`tune_mesh`): the counting pass of vmap_polygonize.

Results are cached as JSON keyed by device name, path (map or batch), voxel
format and image size: in $VMAP_TUNING_CACHE, else
~/.cache/voxelmapping_b200/tuning.json. `tuning_b200.json` beside this file
holds a table measured on a B200, used when the cache has no entry.
"""
import ctypes as C
import json
import os
import statistics
from pathlib import Path

from . import _lib as L

FIELDS = ["alloc_ctas_per_sm", "visibility_ctas_per_sm", "fuse_ctas_per_sm", "zrange_ctas_per_sm",
          "raycast_ctas_per_sm", "normals_ctas_per_sm", "mesh_ctas_per_sm", "raycast_tile_order",
          "raycast_tile_width", "raycast_threads_per_cta", "batch_schedule"]
# the ray marcher's parameters besides its grid, swept one at a time
RAYCAST_PARAMS = ["raycast_tile_width", "raycast_threads_per_cta", "raycast_tile_order"]
STAGE = {"alloc_ctas_per_sm": "alloc", "visibility_ctas_per_sm": "visibility", "fuse_ctas_per_sm": "fuse",
         "zrange_ctas_per_sm": "zrange", "raycast_ctas_per_sm": "raycast", "normals_ctas_per_sm": "normals"}
CANDIDATES = {
    "alloc_ctas_per_sm": [2, 4, 8, 16],
    "visibility_ctas_per_sm": [1, 2, 4, 8],
    "fuse_ctas_per_sm": [4, 8, 16, 32],
    "zrange_ctas_per_sm": [1, 2, 4, 8],
    "raycast_ctas_per_sm": [2, 3, 4, 0],
    "normals_ctas_per_sm": [2, 4, 8, 16],
    "mesh_ctas_per_sm": [4, 8, 16, 32],
    "raycast_tile_order": [0, 1, 2],  # bottom rows first, top rows first, alternating ends
    "raycast_tile_width": [8, 16, 4],  # 8x4, 16x2 or 4x8 rays per warp
    "raycast_threads_per_cta": [256, 128],
    "batch_schedule": [2, 1],  # one persistent launch per batch step, or one launch per stage
}
SHIPPED = Path(__file__).resolve().parent / "tuning_b200.json"


def cache_path():
    p = os.environ.get("VMAP_TUNING_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "voxelmapping_b200" / "tuning.json"


def device_name():
    import torch
    if not torch.cuda.is_available():
        return "no-cuda-device"
    return torch.cuda.get_device_name(torch.cuda.current_device())


def key_for(kind, voxel_format, width, height, n_maps=1):
    """kind: "map" or "batch" (batches are keyed by their map count too; a
    batch of maps of different sizes uses width = height = 0)."""
    k = "%s|%s|%s|%dx%d" % (device_name(), kind, voxel_format, width, height)
    if kind == "batch":
        k += "|maps=%d" % n_maps
    return k


def _read(path):
    try:
        return json.loads(Path(path).read_text())
    except (OSError, ValueError):
        return {}


def lookup(key):
    """(launch config dict, source) of the cached or shipped entry, or (None, None)."""
    for src, path in (("cache", cache_path()), ("shipped", SHIPPED)):
        entry = _read(path).get(key)
        if entry:
            return {f: int(entry["config"].get(f, 0)) for f in FIELDS}, src
    return None, None


def store(key, config, meta=None):
    path = cache_path()
    path.parent.mkdir(parents=True, exist_ok=True)
    table = _read(path)
    table[key] = {"config": config, "meta": meta or {}}
    tmp = path.with_suffix(".tmp")
    tmp.write_text(json.dumps(table, indent=1, sort_keys=True))
    tmp.replace(path)


def tune_map(vm, step, n_steps, rounds=3, warmup=3):
    """Tunes a single map's launch shapes by coordinate descent on whole-step
    time (CUDA events around n_steps steps, no per-stage events: those
    serialise the stage launches that programmatic dependent launch lets
    overlap). step(i) runs step i (fuse + render) on the current stream; every
    field's candidates are measured in interleaved rounds, so they see the same
    stretch of frames. Returns (best config, {field: {candidate: median ms per
    step}})."""
    import torch
    best = vm.get_launch_config()
    for i in range(warmup):
        step(i)
    torch.cuda.synchronize()
    it = warmup
    table = {}
    for f in list(STAGE) + RAYCAST_PARAMS:
        samples = {c: [] for c in CANDIDATES[f]}
        for _ in range(rounds):
            for c in samples:
                vm.set_launch_config(**dict(best, **{f: c}))
                step(it)  # the first step after a change of shape is not timed
                it += 1
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                for _ in range(n_steps):
                    step(it)
                    it += 1
                b.record()
                torch.cuda.synchronize()
                samples[c].append(a.elapsed_time(b) / n_steps)
        med = {c: statistics.median(v) for c, v in samples.items()}
        table[f] = med
        best[f] = min(med, key=med.get)
    vm.set_launch_config(**best)
    return best, table


def tune_mesh(vm, rounds=3):
    """Tunes the marching-cubes grid on the counting pass. Returns (best, {candidate: median ms})."""
    import torch
    lib = L.lib()
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    L.check(lib.vmap_polygonize(vm._map, None, None, 0, C.c_void_p(cnt.data_ptr()), s))  # loads the kernels
    samples = {c: [] for c in CANDIDATES["mesh_ctas_per_sm"]}
    for _ in range(rounds):
        for c in samples:
            vm.set_launch_config(mesh_ctas_per_sm=c)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            L.check(lib.vmap_polygonize(vm._map, None, None, 0, C.c_void_p(cnt.data_ptr()), s))
            b.record()
            torch.cuda.synchronize()
            samples[c].append(a.elapsed_time(b))
    med = {c: statistics.median(v) for c, v in samples.items()}
    best = min(med, key=med.get)
    vm.set_launch_config(mesh_ctas_per_sm=best)
    return best, med


def tune_batch(batch, step, n_steps=4, rounds=2, fields=None):
    """Coordinate descent over the batch's stage grids on whole-step time.
    step(i) runs batch step i on a non-default stream `step.stream`. Returns
    (best config, {field: {candidate: median ms per step}})."""
    import torch
    stream = step.stream
    best = batch.get_launch_config()
    table = {}
    it = 0
    # the schedule first: the persistent launch has one grid (raycast_ctas_per_sm)
    for f in fields or ["batch_schedule"] + [f for f in FIELDS if f not in ("mesh_ctas_per_sm", "batch_schedule")]:
        samples = {c: [] for c in CANDIDATES[f]}
        for _ in range(rounds):
            for c in samples:
                cfg = dict(best)
                cfg[f] = c
                batch.set_launch_config(**cfg)
                with torch.cuda.stream(stream):
                    for _ in range(2):  # the first two steps record the graphs
                        step(it)
                        it += 1
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    for _ in range(n_steps):
                        step(it)
                        it += 1
                    b.record(stream)
                stream.synchronize()
                samples[c].append(a.elapsed_time(b) / n_steps)
        med = {c: statistics.median(v) for c, v in samples.items()}
        table[f] = med
        best[f] = min(med, key=med.get)
    batch.set_launch_config(**best)
    return best, table
