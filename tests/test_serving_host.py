"""Serving scheduler (voxelmapping_b200.serving.Scheduler) on the host with a
fake executor: every request completes, requests of a session complete in
arrival order, a session is only served while resident, resident bytes never
exceed the budget, eviction picks idle sessions, and oversize sessions are
refused up front."""
import numpy as np
import pytest

from voxelmapping_b200 import serving as S


class FakeExecutor:
    def __init__(self, sched):
        self.sched = sched
        self.resident = set()
        self.log = []
        self.t = 0.0

    def run_tick(self, plan, clock):
        for s in plan.evict:
            assert s in self.resident
            self.resident.remove(s)
        for s in plan.restore:
            assert s not in self.resident
            self.resident.add(s)
        assert sum(self.sched.bytes[s] for s in self.resident) <= self.sched.budget
        assert len(self.resident) <= self.sched.max_resident
        touched = [s for s, _, _ in plan.batch] + [r.session for r in plan.mesh]
        assert len(touched) == len(set(touched)), "one request group per session per tick"
        assert len(plan.mesh) <= self.sched.max_mesh
        for s in touched:
            assert s in self.resident
        assert not (set(plan.evict) & set(touched))
        for s, f, r in plan.batch:
            assert f is not None or r is not None
            if f is not None:
                assert f.kind == "fuse" and f.session == s
            if r is not None:
                assert r.kind == "raycast" and r.session == s
        self.t += 1e-4
        for r in plan.requests():
            r.done = clock()
            self.log.append(r)


def run(n_sessions, rate, count, budget_frac, seed=0, max_resident=S.MAX_RESIDENT):
    rng = np.random.default_rng(seed)
    sizes = [int(x) for x in rng.integers(1, 20, n_sessions) * 1000]
    budget = max(max(sizes), int(sum(sizes) * budget_frac))
    sched = S.Scheduler(sizes, budget, max_mesh_per_tick=2, max_resident=max_resident)
    ex = FakeExecutor(sched)
    reqs = S.poisson_requests(n_sessions, rate, count, seed=seed)
    out, stats = S.serve(reqs, sched, ex, clock=lambda: ex.t, wait_until=lambda t: setattr(ex, "t", max(ex.t, t)))
    return out, stats, ex


@pytest.mark.parametrize("budget_frac,max_resident", [(1.0, 256), (0.3, 256), (0.05, 256), (1.0, 4)])
def test_every_request_completes_in_session_order(budget_frac, max_resident):
    out, stats, ex = run(40, 1e9, 3000, budget_frac, max_resident=max_resident)
    assert all(np.isfinite(r.done) for r in out)
    assert len(ex.log) == len(out) == 3000
    by_session = {}
    for r in sorted(out, key=lambda r: (r.tick, r.index)):
        by_session.setdefault(r.session, []).append(r.index)
    for s, idx in by_session.items():
        assert idx == sorted(idx), s
    if budget_frac < 1.0 or max_resident < 40:
        assert stats["evictions"] > 0
    else:
        assert stats["evictions"] == 0 and stats["restores"] == 40


def test_fuse_then_raycast_share_a_batch_frame():
    sched = S.Scheduler([10, 10], 100)
    reqs = [S.Request("fuse", 0, 0.0, 0), S.Request("raycast", 0, 0.1, 1), S.Request("raycast", 1, 0.2, 2),
            S.Request("fuse", 1, 0.3, 3), S.Request("mesh", 0, 0.4, 4)]
    for r in reqs:
        sched.submit(r)
    p = sched.plan()
    assert [(s, f and f.index, r and r.index) for s, f, r in p.batch] == [(0, 0, 1), (1, None, 2)]
    assert p.restore == [0, 1] and not p.mesh
    p = sched.plan()
    assert [(s, f and f.index, r and r.index) for s, f, r in p.batch] == [(1, 3, None)]
    assert [r.index for r in p.mesh] == [4]
    assert sched.waiting == 0 and not sched.plan().requests()


def test_eviction_takes_least_recently_used_idle_sessions():
    sched = S.Scheduler([10, 10, 10, 10], 30)
    for i, s in enumerate([0, 1, 2]):
        sched.submit(S.Request("fuse", s, float(i), i))
    p = sched.plan()
    assert p.restore == [0, 1, 2] and not p.evict
    sched.submit(S.Request("fuse", 1, 5.0, 10))
    sched.plan()  # session 1 becomes most recently used
    sched.submit(S.Request("fuse", 3, 6.0, 11))
    p = sched.plan()
    assert p.evict == [0] and p.restore == [3]
    # a session that cannot fit while all others are busy waits
    sched2 = S.Scheduler([20, 20], 30)
    sched2.submit(S.Request("fuse", 0, 0.0, 0))
    sched2.submit(S.Request("fuse", 1, 0.0, 1))
    p = sched2.plan()
    assert p.restore == [0] and sched2.waiting == 1
    p = sched2.plan()
    assert p.evict == [0] and p.restore == [1]


def test_oversize_session_is_refused():
    with pytest.raises(ValueError):
        S.Scheduler([10, 50], 40)


def test_poisson_mix_and_rate():
    reqs = S.poisson_requests(256, 1000.0, 20000, seed=3)
    kinds = np.array([S.KINDS.index(r.kind) for r in reqs])
    frac = np.bincount(kinds, minlength=3) / len(reqs)
    assert np.allclose(frac, [0.70, 0.25, 0.05], atol=0.015)
    gaps = np.diff([r.arrival for r in reqs])
    assert abs(gaps.mean() - 1e-3) < 5e-5 and gaps.min() >= 0
    assert len({r.session for r in reqs}) == 256


class FakeAsyncMeshExecutor(FakeExecutor):
    """Meshes finish 2.5e-4 s (simulated) after they start, like a mesh worker beside the ticks."""

    def __init__(self, sched):
        super().__init__(sched)
        self.running = {}  # session -> (request, completion time)

    def inflight(self):
        for s in [s for s, (_, t) in self.running.items() if t <= self.t]:
            r, t = self.running.pop(s)
            r.done = t
            self.log.append(r)
        return frozenset(self.running)

    def run_tick(self, plan, clock):
        running = self.inflight()
        touched = [s for s, _, _ in plan.batch] + [r.session for r in plan.mesh]
        assert not set(touched) & running, "a session with a mesh in flight got new work"
        assert not set(plan.evict) & running, "a session with a mesh in flight was evicted"
        assert len(running) + len(plan.mesh) <= self.sched.max_mesh
        mesh, plan.mesh = plan.mesh, []
        super().run_tick(plan, clock)
        for r in mesh:
            self.running[r.session] = (r, self.t + 2.5e-4)


@pytest.mark.parametrize("budget_frac", [1.0, 0.2])
def test_meshes_in_flight_block_their_sessions(budget_frac):
    rng = np.random.default_rng(4)
    sizes = [int(x) for x in rng.integers(1, 20, 30) * 1000]
    sched = S.Scheduler(sizes, max(max(sizes), int(sum(sizes) * budget_frac)), max_mesh_per_tick=2)
    ex = FakeAsyncMeshExecutor(sched)
    reqs = S.poisson_requests(30, 1e9, 2000, mix=(0.5, 0.2, 0.3), seed=5)
    out, stats = S.serve(reqs, sched, ex, clock=lambda: ex.t, wait_until=lambda t: setattr(ex, "t", max(ex.t, t)))
    assert all(np.isfinite(r.done) for r in out) and len(ex.log) == 2000
    by_session = {}
    for r in sorted(out, key=lambda r: (r.done, r.index)):
        by_session.setdefault(r.session, []).append(r.index)
    for s, idx in by_session.items():
        assert idx == sorted(idx), s


class StuckMeshExecutor(FakeAsyncMeshExecutor):
    """A mesh that never finishes (a stopped worker): serve() must raise, not spin."""

    def inflight(self):
        return frozenset(self.running)


def test_serve_raises_instead_of_spinning_on_a_stuck_mesh():
    sched = S.Scheduler([10, 10], 100)
    ex = StuckMeshExecutor(sched)
    reqs = [S.Request("mesh", 0, 0.0, 0), S.Request("fuse", 0, 0.0, 1), S.Request("fuse", 1, 0.0, 2)]
    with pytest.raises(RuntimeError, match="no progress"):
        S.serve(reqs, sched, ex, clock=lambda: ex.t, wait_until=lambda t: setattr(ex, "t", max(ex.t, t)), stall_s=1.0)


def _bare_executor(set_device, mesh_fn):
    """GpuExecutor's mesh-worker machinery without a GPU: fake torch shim, fake mesh."""
    import collections
    import contextlib
    import queue
    import threading
    import types
    ex = S.GpuExecutor.__new__(S.GpuExecutor)
    ex.torch = types.SimpleNamespace(cuda=types.SimpleNamespace(set_device=set_device,
                                                                stream=lambda s: contextlib.nullcontext()))
    ex.dev_index, ex.mesh_stream, ex.mesh_sp = 0, None, None
    ex._mesh_q, ex._inflight, ex._lock, ex._worker_error = queue.Queue(), set(), threading.Lock(), None
    ex.phase = collections.Counter()
    ex._mesh = mesh_fn
    ex._worker = threading.Thread(target=ex._mesh_loop, daemon=True)
    ex._worker.start()
    return ex


def _submit(ex, reqs, clock):
    for r in reqs:
        with ex._lock:
            ex._inflight.add(r.session)
        ex._mesh_q.put((r, clock))


def test_mesh_worker_completes_fails_and_stops_cleanly():
    import time as T
    clock = T.perf_counter

    def mesh(s, stream, sp):
        if s == 3:
            raise ValueError("mesh failed")
        return 100 + s
    ex = _bare_executor(lambda i: None, mesh)
    reqs = [S.Request("mesh", s, 0.0, s) for s in range(5)]
    _submit(ex, reqs, clock)
    t0 = T.perf_counter()
    while ex.inflight() and T.perf_counter() - t0 < 10:
        T.sleep(0.001)
    assert not ex.inflight()
    assert [r.result for r in reqs if r.session != 3] == [100, 101, 102, 104]
    assert isinstance(reqs[3].result, ValueError) and all(np.isfinite(r.done) for r in reqs)
    ex._mesh_q.put(None)
    ex._worker.join(5)
    assert not ex._worker.is_alive()


def test_mesh_worker_that_cannot_start_fails_its_requests():
    import time as T

    def bad_set_device(i):
        raise ValueError("no such device")
    ex = _bare_executor(bad_set_device, lambda s, st, sp: 0)
    ex._worker.join(5)
    assert not ex._worker.is_alive() and isinstance(ex._worker_error, ValueError)
    # requests handed to a dead worker are never served: inflight() reports it instead of hiding it
    reqs = [S.Request("mesh", 0, 0.0, 0)]
    _submit(ex, reqs, T.perf_counter)
    with pytest.raises(RuntimeError, match="mesh worker stopped"):
        ex.inflight()


# -- several GPUs: partition, routing and merging ------------------------------
def test_partition_follows_capacity_and_balances_bytes():
    rng = np.random.default_rng(3)
    sizes = [int(x) for x in rng.integers(1, 50, 512) * 1000]
    # capacities far above, near and below the sessions' total (12.8 MB)
    for caps in ([1e6] * 4, [4e6, 2e6, 1e6, 1e6], [80e9, 40e9], [8e9] * 8, [3e5, 1e5]):
        owner = S.partition_sessions(sizes, caps)
        assert len(owner) == len(sizes) and set(owner) == set(range(len(caps)))
        held = [sum(b for b, r in zip(sizes, owner) if r == k) for k in range(len(caps))]
        fill = [h / c for h, c in zip(held, caps)]
        assert max(fill) - min(fill) <= max(sizes) / min(caps), caps
        assert owner == S.partition_sessions(sizes, caps)  # deterministic
    owner = S.partition_sessions(sizes, [80e9, 40e9])
    held = [sum(b for b, r in zip(sizes, owner) if r == k) for k in range(2)]
    assert abs(held[0] / held[1] - 2.0) < 0.05  # shares follow free memory
    assert S.partition_sessions(sizes, [1.0]) == [0] * len(sizes)
    for bad in ([], [1e6, 0]):
        with pytest.raises(ValueError):
            S.partition_sessions(sizes, bad)


def test_local_requests_split_the_stream_by_owner():
    reqs = S.poisson_requests(10, 1000.0, 500, seed=4)
    owner = [s % 3 for s in range(10)]
    seen = []
    for rank in range(3):
        loc, mine = S.local_requests(reqs, owner, rank)
        assert mine == [s for s in range(10) if s % 3 == rank]
        assert [r.index for r in loc] == list(range(len(loc)))
        assert all(a.arrival <= b.arrival for a, b in zip(loc, loc[1:]))
        seen += [(mine[r.session], r.kind, r.arrival) for r in loc]
    assert sorted(seen) == sorted((r.session, r.kind, r.arrival) for r in reqs)


def _summary(n_sessions, seed, makespan_scale=1.0):
    out, stats, _ = run(n_sessions, 1e9, 400, 1.0, seed=seed)
    stats["makespan_s"] *= makespan_scale
    return S.summarize(out, stats)


def test_merge_summaries():
    one = _summary(8, 0)
    m = S.merge_summaries([one])
    assert m["ranks"] == 1 and all(m[k] == one[k] for k in one)
    a, b = _summary(8, 1), _summary(8, 2, makespan_scale=2.0)
    for p in (a, b):
        p.update(offered_rps=100.0, sessions=8, budget_gb=1.0, all_sessions_gb=1.0)
    m = S.merge_summaries([a, b])
    assert m["ranks"] == 2 and m["requests"] == 800 and m["sessions"] == 16 and m["offered_rps"] == 200.0
    assert m["makespan_s"] == max(a["makespan_s"], b["makespan_s"])
    assert m["throughput_rps"] == pytest.approx(800 / m["makespan_s"])
    lat = a["_latencies"]["all"] + b["_latencies"]["all"]
    assert m["all"]["n"] == 800 and m["all"]["p99_ms"] == pytest.approx(1e3 * np.percentile(lat, 99))
    assert m["evictions"] == a["evictions"] + b["evictions"] and len(m["per_rank"]) == 2


def test_session_bytes_is_the_map_plus_its_image_buffers():
    from voxelmapping_b200 import synth
    from voxelmapping_b200.vmapping import VoxelMapping
    for w in synth.uneven_workloads(6, seed=5):
        vm = VoxelMapping(w.width, w.height, w.K, voxel_format=w.voxel_format, with_color=w.with_color,
                          max_weight=w.max_weight)
        assert S.session_bytes(w) == vm.required_bytes(w.num_entries, w.num_blocks, w.voxel_size) + \
            w.width * w.height * 37


class FakeGpuExecutor:
    """Stands in for GpuExecutor inside run_serving: completes every request
    at once on the wall clock (no device)."""

    def __init__(self, wls, frames, keep_results=False):
        import collections
        self.wls, self.frames = wls, frames
        self.phase = collections.Counter()
        self.ticks = 0

    def session_bytes(self, s):
        return S.session_bytes(self.wls[s])

    def run_tick(self, plan, clock):
        self.ticks += 1
        for r in plan.requests():
            r.done = clock()

    def inflight(self):
        return frozenset()

    def release(self):
        pass


@pytest.mark.parametrize("world", [1, 2])
def test_run_serving_drives_its_executor_for_each_rank(monkeypatch, world):
    import torch
    monkeypatch.setattr(S, "GpuExecutor", FakeGpuExecutor)
    monkeypatch.setattr(S, "render_frames", lambda wls, n: [[None] * n for _ in wls])
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda *a: (80 << 30, 180 << 30))
    caps = [80 << 30, 40 << 30][:world]
    per_rank = []
    for rank in range(world):
        res, ex = S.run_serving(n_sessions=6, rates=(2000.0,), count=60, budget_frac=1.0, n_frames=2, warmup=10,
                                seed=3, rank=rank, world=world, all_gather=lambda x: caps)
        assert len(res) == 1 and ex.ticks > 0
        per_rank.append(res[0])
    m = S.merge_summaries(per_rank)
    assert m["requests"] == 60 * world and m["sessions"] == 6 * world
    assert m["offered_rps"] == pytest.approx(2000.0 * world)
    if world == 1:
        assert per_rank[0]["offered_rps"] == 2000.0 and per_rank[0]["sessions"] == 6
    else:
        assert per_rank[0]["sessions"] > per_rank[1]["sessions"]  # twice the free memory
