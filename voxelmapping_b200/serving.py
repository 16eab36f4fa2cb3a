"""Serving many mapping sessions from one GPU or several.

A session is one map (its own scene, camera, voxel size and pool). Requests
arrive over time: "fuse" (a depth + colour frame to integrate), "raycast"
(render the vertex + normal maps at a pose and return them to the host) and
"mesh" (extract the full triangle mesh to the host). The reference serves a
single map per process and has no counterpart; this module adds the server
around the library's batch step (vmap_batch_step) and map snapshots
(vmap_snapshot_save / vmap_snapshot_load).

Scheduling works in ticks. A tick takes, for every session with waiting
requests, the oldest one (a fuse directly followed by a raycast of the same
session goes into the same tick: one batch frame fuses, then renders), runs
all of them as ONE batch step over the resident maps (maps without work are
idle in that step), copies raycast results to pinned host memory, then runs
at most `max_mesh_per_tick` mesh requests. Requests of one session complete
in arrival order.

Admission is by device memory: a session's map (voxel-block pool, hash table,
frame buffers) must be resident to serve it. A non-resident session is
admitted if its bytes fit the budget, evicting least-recently-used idle
sessions (snapshot to pinned host memory, map released) as needed; if they
still do not fit, its requests wait. At most VMAP_MAX_BATCH (256) maps are
resident, the batch step's limit.

On several GPUs (one process per GPU) sessions stay independent: they are
partitioned over the ranks by free device memory (partition_sessions), every
rank serves the requests of its own sessions (local_requests) with its own
scheduler and executor, and only control data crosses ranks: the free-memory
figures before and the summaries after (merge_summaries).

`Scheduler` is pure host logic (tested on the CPU with a fake executor);
`GpuExecutor` drives the library.
"""
import collections
import ctypes as C
import dataclasses
import math
import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L

KINDS = ("fuse", "raycast", "mesh")
MAX_RESIDENT = 256


@dataclass
class Request:
    kind: str
    session: int
    arrival: float            # seconds after the start of the run
    index: int = 0            # position in the arrival order
    done: float = math.nan    # completion time, seconds after the start
    tick: int = -1
    result: object = None

    @property
    def latency(self):
        return self.done - self.arrival


def poisson_requests(n_sessions, rate, count, mix=(0.70, 0.25, 0.05), seed=0):
    """`count` requests with exponential inter-arrival times at `rate` per
    second, sessions uniform at random, kinds drawn with probabilities `mix`
    (fuse, raycast, mesh)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, count))
    sess = rng.integers(0, n_sessions, count)
    kinds = rng.choice(len(KINDS), count, p=np.asarray(mix, np.float64) / np.sum(mix))
    return [Request(KINDS[k], int(s), float(a), i) for i, (k, s, a) in enumerate(zip(kinds, sess, t))]


@dataclass
class TickPlan:
    batch: list = field(default_factory=list)    # (session, fuse request or None, raycast request or None)
    mesh: list = field(default_factory=list)     # mesh requests
    evict: list = field(default_factory=list)    # sessions to evict before the tick
    restore: list = field(default_factory=list)  # sessions to make resident before the tick

    def requests(self):
        out = [r for _, f, q in self.batch for r in (f, q) if r is not None]
        return out + list(self.mesh)


class Scheduler:
    """Admission, eviction and tick formation (no GPU work).

    session_bytes[s] is the device memory session s holds while resident;
    budget the bytes all resident sessions may hold together."""

    def __init__(self, session_bytes, budget, max_mesh_per_tick=2, max_resident=MAX_RESIDENT):
        """max_mesh_per_tick: meshes started per tick, or in flight at once
        when a mesh worker runs them beside the ticks."""
        self.bytes = list(session_bytes)
        if max(self.bytes) > budget:
            raise ValueError("a session needs more device memory than the whole budget")
        self.budget = budget
        self.max_mesh = max_mesh_per_tick
        self.max_resident = max_resident
        self.resident = collections.OrderedDict()  # session -> None, least recently used first
        self.used = 0
        self.queues = collections.defaultdict(collections.deque)  # session -> waiting requests
        self.waiting = 0
        self.evictions = 0
        self.restores = 0

    def submit(self, req):
        self.queues[req.session].append(req)
        self.waiting += 1

    def free(self):
        return self.budget - self.used

    def plan(self, blocked=()):
        """Take the next tick's work off the queues. `blocked`: sessions with
        work still in flight from earlier ticks (meshes on the mesh worker):
        they get no new work and are not evicted; they count against the
        mesh limit."""
        p = TickPlan()
        heads = sorted((q[0].arrival, s) for s, q in self.queues.items() if q)
        busy = set(blocked)
        for _, s in heads:
            q = self.queues[s]
            if s in busy:
                continue
            if q[0].kind == "mesh" and len(p.mesh) + len(blocked) >= self.max_mesh:
                continue
            if s not in self.resident and (s in p.evict or not self._admit(s, busy, p)):
                continue
            busy.add(s)
            self.resident.move_to_end(s)
            head = q.popleft()
            self.waiting -= 1
            if head.kind == "mesh":
                p.mesh.append(head)
            elif head.kind == "raycast":
                p.batch.append((s, None, head))
            else:
                ray = None
                if q and q[0].kind == "raycast":
                    ray = q.popleft()
                    self.waiting -= 1
                p.batch.append((s, head, ray))
        return p

    def _admit(self, s, busy, p):
        need = self.bytes[s]
        # idle sessions, least recently used first; those without waiting work before the rest
        idle = [v for v in self.resident if v not in busy]
        victims = [v for v in idle if not self.queues[v]] + [v for v in idle if self.queues[v]]
        freed, take = 0, []
        for v in victims:
            if self.free() + freed >= need and len(self.resident) - len(take) < self.max_resident:
                break
            take.append(v)
            freed += self.bytes[v]
        if self.free() + freed < need or len(self.resident) - len(take) >= self.max_resident:
            return False
        for v in take:
            del self.resident[v]
            self.used -= self.bytes[v]
            p.evict.append(v)
            self.evictions += 1
        self.resident[s] = None
        self.used += need
        p.restore.append(s)
        self.restores += 1
        return True


class GpuExecutor:
    """Runs tick plans on the GPU.

    All resident maps sit in the slots of ONE long-lived slot batch
    (vmap_batch_create_slots), so its recorded CUDA graphs are reused whatever
    sessions come and go. A resident session owns a device block from torch's
    caching allocator holding its map (vmap_create_in: creating and
    destroying maps allocates and frees no device memory) plus buffers for one
    frame and one vertex + normal map; an evicted session owns a snapshot in
    pinned host memory. Frames are pre-rendered into pinned host memory
    (frames[s] = list of (depth int16 (h, w), rgb uint8 (h, 3w), pose (4, 4)))
    and copied in per fuse request. Meshes are extracted on the device into
    shared buffers and copied to one pinned host buffer."""

    def __init__(self, workloads, frames, device="cuda", copy_results=True, keep_results=False,
                 n_slots=MAX_RESIDENT, mesh_worker=True):
        import torch
        self.torch = torch
        self.wls = list(workloads)
        self.frames = frames
        self.dev = torch.device(device)
        self.dev_index = self.dev.index if self.dev.index is not None else torch.cuda.current_device()
        self.stream = torch.cuda.Stream(device=self.dev)
        self.sp = C.c_void_p(self.stream.cuda_stream)
        self.copy_results = copy_results
        self.keep_results = keep_results  # fresh host buffers per raycast (tests), else one pair per session
        self.lib = L.lib()
        fmts = {w.voxel_format for w in self.wls}
        if len(fmts) != 1:
            raise ValueError("all sessions need one voxel format")
        self.n_slots = min(n_slots, MAX_RESIDENT)
        h = C.c_void_p()
        L.check(self.lib.vmap_batch_create_slots(self.n_slots, L.FORMAT_NAMES[fmts.pop()], C.byref(h)),
                "vmap_batch_create_slots")
        self.batch = h
        self.frames_arr = (L.BatchFrame * self.n_slots)()
        self.free_slots = list(range(self.n_slots - 1, -1, -1))
        self.slot = {}       # session -> batch slot (resident)
        self.maps = {}       # session -> VoxelMapping (resident)
        self.bufs = {}       # session -> (depth, rgb, vmap, nmap) device tensors
        self.snaps = {}      # session -> pinned uint8 snapshot
        self.outs = {}       # session -> (vmap, nmap) pinned host results
        self.next_frame = collections.Counter()
        self.dirty = []      # slots whose frame pointers the last tick set
        self.mesh_dev = None  # (verts, norms) device buffers, grown on demand
        self.mesh_host = None
        self.mesh_count = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.mesh_count_host = torch.zeros(1, dtype=torch.int32, pin_memory=True)
        self.phase = collections.Counter()  # seconds per phase
        # meshes run on their own stream in a worker thread, beside the ticks
        # (the scheduler keeps their sessions out of the ticks meanwhile)
        self.mesh_stream = torch.cuda.Stream(device=self.dev)
        self.mesh_sp = C.c_void_p(self.mesh_stream.cuda_stream)
        self._inflight = set()
        self._worker_error = None
        self._lock = threading.Lock()
        self._mesh_q = queue.Queue() if mesh_worker else None
        self._worker = None
        if mesh_worker:
            self._worker = threading.Thread(target=self._mesh_loop, name="vmap-mesh", daemon=True)
            self._worker.start()

    def inflight(self):
        """Sessions whose mesh is still running on the mesh worker."""
        with self._lock:
            running = frozenset(self._inflight)
        if running and self._worker is not None and not self._worker.is_alive():
            raise RuntimeError("the mesh worker stopped with meshes in flight") from self._worker_error
        return running

    def _mesh_loop(self):
        torch = self.torch
        item = None
        try:
            torch.cuda.set_device(self.dev_index)
            while True:
                item = self._mesh_q.get()
                if item is None:
                    return
                r, clock = item
                try:
                    t0 = clock()
                    with torch.cuda.stream(self.mesh_stream):
                        r.result = self._mesh(r.session, self.mesh_stream, self.mesh_sp)
                    r.done = clock()
                    self.phase["mesh"] += r.done - t0
                except BaseException as e:  # surfaced by serve() through the request
                    r.result = e
                    r.done = clock()
                finally:
                    with self._lock:
                        self._inflight.discard(r.session)
                item = None
        except BaseException as e:  # the worker itself failed: fail what it holds and stop
            self._worker_error = e
            pending = [item] if item is not None else []
            while True:
                try:
                    nxt = self._mesh_q.get_nowait()
                except queue.Empty:
                    break
                if nxt is not None:
                    pending.append(nxt)
            for r, clock in pending:
                r.result, r.done = e, clock()
            with self._lock:
                self._inflight.clear()

    # -- memory ----------------------------------------------------------------
    def _new_map(self, s):
        from .vmapping import VoxelMapping
        w = self.wls[s]
        return VoxelMapping(w.width, w.height, w.K, voxel_format=w.voxel_format, with_color=w.with_color,
                            max_weight=w.max_weight)

    def map_bytes(self, s):
        w = self.wls[s]
        return self._new_map(s).required_bytes(w.num_entries, w.num_blocks, w.voxel_size)

    def session_bytes(self, s):
        """Device bytes of session s while resident (session_bytes)."""
        return session_bytes(self.wls[s])

    def restore(self, s):
        torch = self.torch
        w = self.wls[s]
        with torch.cuda.stream(self.stream):
            mem = torch.empty(self.map_bytes(s), dtype=torch.uint8, device=self.dev)
            vm = self._new_map(s)
            vm.CreateMapIn(w.num_entries, w.num_blocks, w.voxel_size, mem)
            if s in self.snaps:
                vm.load_snapshot(self.snaps[s])
            self.bufs[s] = (torch.empty((w.height, w.width), dtype=torch.int16, device=self.dev),
                            torch.empty((w.height, w.width * 3), dtype=torch.uint8, device=self.dev),
                            torch.empty((w.height, w.width, 4), dtype=torch.float32, device=self.dev),
                            torch.empty((w.height, w.width, 4), dtype=torch.float32, device=self.dev))
        slot = self.free_slots.pop()
        L.check(self.lib.vmap_batch_set_map(self.batch, slot, vm._map), "vmap_batch_set_map")
        self.maps[s], self.slot[s] = vm, slot
        f = self.frames_arr[slot]
        f.depth_type, f.depth_pitch, f.depth_scale = L.DEPTH_U16, w.width * 2, w.depth_scale
        f.rgb_pitch, f.vmap_pitch, f.nmap_pitch = w.width * 3, w.width * 16, w.width * 16

    def evict(self, s):
        torch = self.torch
        vm = self.maps.pop(s)
        slot = self.slot.pop(s)
        with torch.cuda.stream(self.stream):
            n = vm.snapshot_bytes()
            buf = self.snaps.get(s)
            if buf is None or buf.numel() < n:  # room to grow: pinning host memory is slow
                buf = torch.empty(max(2 * n, 16 << 20), dtype=torch.uint8, pin_memory=True)
            self.snaps[s] = buf[:vm.save_snapshot(buf).shape[0]]  # synchronous
        L.check(self.lib.vmap_batch_set_map(self.batch, slot, None), "vmap_batch_set_map")
        vm.release()  # the map's memory returns to torch's cache; nothing of it is in flight
        self.bufs.pop(s)
        self.free_slots.append(slot)
        f = self.frames_arr[slot]
        f.depth_dev = f.rgb_dev = f.vmap_dev = f.nmap_dev = None

    # -- one tick ----------------------------------------------------------------
    def _mesh(self, s, stream, sp):
        """Full mesh of session s to pinned host memory on `stream`; returns the triangle count."""
        torch = self.torch
        vm = self.maps[s]
        lib = self.lib
        L.check(lib.vmap_polygonize(vm._map, None, None, 0, C.c_void_p(self.mesh_count.data_ptr()), sp),
                "vmap_polygonize")
        self.mesh_count_host.copy_(self.mesh_count, non_blocking=True)
        stream.synchronize()
        n = int(self.mesh_count_host.item())
        if n == 0:
            return 0
        if self.mesh_dev is None or self.mesh_dev[0].shape[0] < n:
            cap = max(n * 5 // 4, 1 << 16)
            self.mesh_dev = (torch.empty((cap, 9), dtype=torch.float32, device=self.dev),
                             torch.empty((cap, 9), dtype=torch.float32, device=self.dev))
            self.mesh_host = (torch.empty((cap, 9), dtype=torch.float32, pin_memory=True),
                              torch.empty((cap, 9), dtype=torch.float32, pin_memory=True))
        v, nr = self.mesh_dev
        L.check(lib.vmap_polygonize(vm._map, C.c_void_p(v.data_ptr()), C.c_void_p(nr.data_ptr()), v.shape[0],
                                    None, sp), "vmap_polygonize")
        self.mesh_host[0][:n].copy_(v[:n], non_blocking=True)
        self.mesh_host[1][:n].copy_(nr[:n], non_blocking=True)
        stream.synchronize()
        return n

    def run_tick(self, plan, clock):
        """Executes `plan`; sets each request's completion time from `clock()`."""
        torch = self.torch
        t0 = clock()
        for s in plan.evict:
            self.evict(s)
        t1 = clock()
        for s in plan.restore:
            self.restore(s)
        t2 = clock()
        self.phase["evict"] += t1 - t0
        self.phase["restore"] += t2 - t1
        with torch.cuda.stream(self.stream):
            if plan.batch:
                for i in self.dirty:
                    f = self.frames_arr[i]
                    f.depth_dev = f.rgb_dev = f.vmap_dev = f.nmap_dev = None
                self.dirty = []
                for s, fuse, ray in plan.batch:
                    slot = self.slot[s]
                    f = self.frames_arr[slot]
                    self.dirty.append(slot)
                    d_dev, c_dev, v_dev, n_dev = self.bufs[s]
                    if fuse is not None:
                        k = self.next_frame[s] % len(self.frames[s])
                        self.next_frame[s] += 1
                        d, c, pose = self.frames[s][k]
                        d_dev.copy_(d, non_blocking=True)
                        c_dev.copy_(c, non_blocking=True)
                        f.depth_dev, f.rgb_dev = d_dev.data_ptr(), c_dev.data_ptr()
                    else:
                        k = max(self.next_frame[s] - 1, 0) % len(self.frames[s])
                        pose = self.frames[s][k][2]
                    f.pose[:] = [float(x) for x in np.asarray(pose, np.float64).reshape(16)]
                    if ray is not None:
                        f.vmap_dev, f.nmap_dev = v_dev.data_ptr(), n_dev.data_ptr()
                L.check(self.lib.vmap_batch_step(self.batch, self.frames_arr, self.sp), "vmap_batch_step")
                for s, fuse, ray in plan.batch:
                    if ray is not None and self.copy_results:
                        out = None if self.keep_results else self.outs.get(s)
                        _, _, v_dev, n_dev = self.bufs[s]
                        if out is None:
                            out = (torch.empty(v_dev.shape, dtype=torch.float32, pin_memory=True),
                                   torch.empty(n_dev.shape, dtype=torch.float32, pin_memory=True))
                            if not self.keep_results:
                                self.outs[s] = out
                        out[0].copy_(v_dev, non_blocking=True)
                        out[1].copy_(n_dev, non_blocking=True)
                        ray.result = (out[0], out[1], self.next_frame[s])  # maps + frames fused so far
                self.stream.synchronize()
                t = clock()
                for r in plan.requests():
                    if r.kind != "mesh":
                        r.done = t
            t3 = clock()
            self.phase["batch"] += t3 - t2
            for r in plan.mesh:
                if self._mesh_q is not None:
                    with self._lock:
                        self._inflight.add(r.session)
                    self._mesh_q.put((r, clock))
                else:
                    r.result = self._mesh(r.session, self.stream, self.sp)
                    r.done = clock()
                    self.phase["mesh"] += r.done - t3

    def release(self):
        if self._worker is not None:
            self._mesh_q.put(None)
            self._worker.join()
            self._worker = None
        self.torch.cuda.synchronize()
        for s in list(self.maps):
            L.check(self.lib.vmap_batch_set_map(self.batch, self.slot[s], None), "vmap_batch_set_map")
            self.maps.pop(s).release()
        self.slot.clear()
        if self.batch is not None:
            L.check(self.lib.vmap_batch_destroy(self.batch), "vmap_batch_destroy")
            self.batch = None


def serve(requests, scheduler, executor, clock=None, wait_until=None, stall_s=120.0):
    """Replays `requests` (sorted by arrival) against wall-clock time: a
    request becomes visible to the scheduler at its arrival time; ticks run
    back to back while work is waiting. `clock` / `wait_until` replace the
    wall clock and the idle wait (for simulated time). Raises when work is
    waiting or in flight and nothing completes for `stall_s` seconds. Returns
    (requests, stats)."""
    start = time.perf_counter()
    clock = clock or (lambda: time.perf_counter() - start)

    def sleep_until(t):
        while True:
            wait = t - clock()
            if wait <= 0:
                return
            # sleeping (or yielding) releases the GIL to the mesh worker
            time.sleep(wait - 1e-4 if wait > 2e-4 else 0)

    wait_until = wait_until or sleep_until
    inflight = getattr(executor, "inflight", lambda: frozenset())  # sessions with a mesh still running
    pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
    ticks, batch_sizes, busy = 0, [], 0.0
    last_progress, last_state = clock(), None
    while pending or scheduler.waiting or inflight():
        now = clock()
        state = (ticks, inflight(), scheduler.waiting, len(pending))
        if state != last_state:
            last_state, last_progress = state, now
        elif (scheduler.waiting or state[1]) and now - last_progress > stall_s:
            raise RuntimeError("serving made no progress for %.0f s (%d waiting, meshes in flight for sessions %s)"
                               % (now - last_progress, scheduler.waiting, sorted(state[1])))
        while pending and pending[0].arrival <= now:
            scheduler.submit(pending.popleft())
        if not scheduler.waiting:
            if inflight():
                wait_until(min(pending[0].arrival, now + 1e-4) if pending else now + 1e-4)
            else:
                wait_until(pending[0].arrival)
            continue
        blocked = inflight()
        plan = scheduler.plan(blocked)
        if not plan.batch and not plan.mesh:
            if blocked:  # the waiting work belongs to sessions whose meshes are running
                wait_until(now + 1e-4)
                continue
            raise RuntimeError("no admissible work: the budget cannot hold any waiting session")
        t0 = clock()
        executor.run_tick(plan, clock)
        busy += clock() - t0
        for r in plan.requests():
            r.tick = ticks
        ticks += 1
        batch_sizes.append(len(plan.batch))
    makespan = clock()
    for r in requests:
        if isinstance(r.result, BaseException):
            raise RuntimeError("request %d (%s) failed" % (r.index, r.kind)) from r.result
    stats = {"ticks": ticks, "mean_batch": float(np.mean(batch_sizes)) if batch_sizes else 0.0,
             "max_batch": int(max(batch_sizes)) if batch_sizes else 0, "busy_s": busy, "makespan_s": makespan,
             "evictions": scheduler.evictions, "restores": scheduler.restores}
    return requests, stats


def _latency_stats(lat):
    return {"n": len(lat), "p50_ms": 1e3 * float(np.percentile(lat, 50)),
            "p99_ms": 1e3 * float(np.percentile(lat, 99)), "mean_ms": 1e3 * float(np.mean(lat))}


def summarize(requests, stats):
    """Throughput and latency percentiles (ms) per request kind; the raw
    latencies (seconds) per kind stay under "_latencies" for merge_summaries."""
    out = {"requests": len(requests), "throughput_rps": len(requests) / stats["makespan_s"], "_latencies": {}}
    for kind in KINDS + ("all",):
        lat = [r.latency for r in requests if kind in ("all", r.kind)]
        if lat:
            out[kind] = _latency_stats(lat)
            out["_latencies"][kind] = lat
    out.update(stats)
    return out


# -- several GPUs: sessions are independent, so they are partitioned ----------
def session_bytes(w):
    """Device bytes of a session with workload w while resident: its map
    (vmap_required_bytes, computed on the host) plus its frame and vertex /
    normal map buffers."""
    from .vmapping import VoxelMapping
    vm = VoxelMapping(w.width, w.height, w.K, voxel_format=w.voxel_format, with_color=w.with_color,
                      max_weight=w.max_weight)
    return vm.required_bytes(w.num_entries, w.num_blocks, w.voxel_size) + w.width * w.height * (2 + 3 + 16 + 16)


def partition_sessions(sizes, capacities):
    """Session -> rank. Sessions in decreasing size (ties by index), each to
    the rank whose fill (bytes held / capacity, e.g. its free device memory)
    is lowest once it takes the session (ties to the lower rank). Each rank's
    share of the bytes then follows its capacity, however small the sessions
    are against it: fills differ by at most one session's size over the
    smallest capacity. Capacities may be exceeded; the ranks then evict."""
    if not capacities or min(capacities) <= 0:
        raise ValueError("every rank needs a positive capacity")
    held = [0.0] * len(capacities)
    owner = [0] * len(sizes)
    for s in sorted(range(len(sizes)), key=lambda s: (-sizes[s], s)):
        r = min(range(len(held)), key=lambda r: ((held[r] + sizes[s]) / capacities[r], r))
        owner[s] = r
        held[r] += sizes[s]
    return owner


def local_requests(requests, owner, rank):
    """The requests addressed to the sessions that `owner` gives `rank`, with
    sessions renumbered to that rank's list (global order) and indices to the
    order of arrival. Returns (requests, global session ids of the rank)."""
    mine = [s for s, r in enumerate(owner) if r == rank]
    local = {s: i for i, s in enumerate(mine)}
    out = []
    for q in requests:
        if q.session in local:
            out.append(Request(q.kind, local[q.session], q.arrival, len(out)))
    return out, mine


def merge_summaries(parts):
    """One job-level summary from the per-rank summaries of the same run:
    requests, offered rates, sessions, budgets and eviction counters add up;
    throughput is all requests over the slowest rank's makespan; percentiles
    are over every rank's latencies ("_latencies"). Per-rank tick statistics
    stay under "per_rank". A single part comes back as it is, with ranks = 1."""
    if len(parts) == 1:
        return dict(parts[0], ranks=1)
    out = {"ranks": len(parts), "requests": sum(p["requests"] for p in parts),
           "makespan_s": max(p["makespan_s"] for p in parts)}
    out["throughput_rps"] = out["requests"] / out["makespan_s"]
    for kind in KINDS + ("all",):
        lat = [x for p in parts for x in p.get("_latencies", {}).get(kind, [])]
        if lat:
            out[kind] = _latency_stats(lat)
    for k in ("offered_rps", "sessions", "budget_gb", "all_sessions_gb", "evictions", "restores"):
        if all(k in p for p in parts):
            out[k] = sum(p[k] for p in parts)
    out["per_rank"] = [{k: p[k] for k in ("requests", "makespan_s", "ticks", "mean_batch", "busy_s", "sessions")
                        if k in p} for p in parts]
    return out


def render_frames(workloads, n_frames, pin=True):
    """n_frames frames per workload, spread over its trajectory, as pinned
    host tensors: [(depth int16 (h, w), rgb uint8 (h, 3w), pose (4, 4)), ...]."""
    import torch
    from . import synth
    out = []
    for w in workloads:
        sc = synth.Scene(w)
        stride = max(1, w.n_poses // n_frames)
        fr = []
        for i in range(n_frames):
            d, c, p = sc.render(i * stride)
            dt = torch.from_numpy(d.view(np.int16))
            ct = torch.from_numpy(c).reshape(w.height, -1)
            fr.append((dt.pin_memory() if pin else dt, ct.pin_memory() if pin else ct, p))
        out.append(fr)
    return out


def run_serving(n_sessions=256, rates=(2000.0,), count=4000, budget_bytes=None, budget_frac=0.5, n_frames=4,
                seed=0, warmup=500, max_mesh_per_tick=2, keep_results=False, pool_scale=1, log=None,
                rank=0, world=1, all_gather=None):
    """Builds n_sessions uneven sessions (FP16 + colour), then for each rate
    replays `count` Poisson requests (70/25/5 fuse/raycast/mesh) after a
    warm-up that touches every session and `warmup` more requests. The
    budget is `budget_bytes`, or
    `budget_frac` of all sessions' bytes, capped at 85 % of the free device
    memory. `pool_scale` multiplies every pool.

    With world > 1 ranks (one process per GPU) the job holds n_sessions x
    world sessions, partitioned over the ranks by free device memory
    (partition_sessions; `all_gather(x)` returns every rank's x in rank
    order); rate and request count scale by world and every rank serves the
    requests of its own sessions, so the work per GPU stays that of one rank
    alone. merge_summaries combines the ranks' summaries. Returns (list of
    this rank's per-rate summaries, executor)."""
    import torch
    from . import synth
    total = n_sessions * world
    all_wls = [dataclasses.replace(w, num_blocks=w.num_blocks * pool_scale)
               for w in synth.uneven_workloads(total, seed=seed)]
    owner = [0] * total
    if world > 1:
        free, _ = torch.cuda.mem_get_info()
        owner = partition_sessions([session_bytes(w) for w in all_wls], all_gather(free))
    # the partition is the same on every rank: every rank refuses it together
    empty = sorted(set(range(world)) - set(owner))
    if empty:
        raise ValueError("rank(s) %s hold no session (%d sessions over %d ranks)" % (empty, total, world))
    wls = [all_wls[s] for s in range(total) if owner[s] == rank]
    n_local = len(wls)
    frames = render_frames(wls, n_frames)
    ex = GpuExecutor(wls, frames, keep_results=keep_results)
    sizes = [ex.session_bytes(s) for s in range(n_local)]
    free, _ = torch.cuda.mem_get_info()
    budget = int(budget_bytes or budget_frac * sum(sizes))
    budget = max(max(sizes), min(budget, int(0.85 * free)))
    results = []
    try:
        sched = Scheduler(sizes, budget, max_mesh_per_tick=max_mesh_per_tick)
        if warmup:
            # every session once per distinct frame, in order (restores, frame
            # uploads, renders, result buffers; every map fuses all its frames
            # and reaches its steady size, and under a tight budget every
            # session is evicted at that size, so its snapshot buffer is
            # allocated), meshes of the 16 largest pools (mesh buffers at full
            # size), then `warmup` requests at the highest rate: first-touch
            # costs stay out of the measured runs
            for _ in range(max(2, n_frames)):
                serve([Request(k, s, 0.0, 0) for s in range(n_local) for k in ("fuse", "raycast")], sched, ex)
            big = sorted(range(n_local), key=lambda s: -wls[s].num_blocks)[:16]
            serve([Request("mesh", s, 0.0, 0) for s in big], sched, ex)
            serve(poisson_requests(n_local, max(rates), warmup, seed=seed + 7), sched, ex)
        for k, rate in enumerate(rates):
            sched.evictions = sched.restores = 0
            reqs = poisson_requests(total, rate * world, count * world, seed=seed + 100 + k)
            if world > 1:
                reqs, _ = local_requests(reqs, owner, rank)
            ex.phase.clear()
            reqs, stats = serve(reqs, sched, ex)
            summ = summarize(reqs, stats)
            summ["phase_s"] = {k: round(v, 4) for k, v in ex.phase.items()}
            # offered_rps: this rank's share of the job's Poisson rate by
            # session count (requests pick sessions uniformly, so it is the
            # expected rate; summed over ranks it is the job's rate);
            # offered_rps_measured: its requests over the span of their
            # arrival times, the rate this rank actually drew
            span = (max(r.arrival for r in reqs) - min(r.arrival for r in reqs)) if len(reqs) > 1 else 0.0
            summ.update({"offered_rps": rate * world * n_local / total,
                         "offered_rps_measured": (len(reqs) - 1) / span if span > 0 else None,
                         "sessions": n_local, "budget_gb": budget / 1e9,
                         "all_sessions_gb": sum(sizes) / 1e9})
            results.append(summ)
            if log:
                log(summ)
            if keep_results:
                summ["_requests"] = reqs
    except BaseException:
        ex.release()
        raise
    return results, ex
