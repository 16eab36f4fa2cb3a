"""The N > 1 host path of bench.py on CPU: two gloo ranks (127.0.0.1).
Every rank reports its own device time; the job's time is the maximum over
ranks and its throughput counts every rank's units. Ranks map their own
seeded scenes (independent maps, no collective on the data path), and the
reference arm runs on rank 0 only."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = [120.0, 150.0][rank]
        mx = bench.max_over_ranks(local_ms, "cpu", world)
        thr = bench.job_throughput(100, mx, world)
        from voxelmapping_b200 import synth
        wl = synth.WORKLOADS["room_full"]

        class A:
            uneven, batch, batch_blocks = 3, 2, 1 << 14
        un, _ = bench.batched_uneven(A, rank)
        same, _ = bench.batched_same_size(A, wl, rank)
        out.put((rank, mx, thr, tuple(w.seed for w in un), tuple(w.seed for w in same)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_max_time_and_map_distinct_scenes():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, mx0, thr0, un0, sm0), (_, mx1, thr1, un1, sm1) = res
    assert mx0 == mx1 == 150.0
    assert thr0 == thr1 == pytest.approx(2 * 100 / 0.150)
    assert not set(un0) & set(un1) and not set(sm0) & set(sm1)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        warmup, steps, gpus = 1, 1, 2
    assert bench.run_reference(A) is None  # returns at once, prints nothing


def _serve_rank(rank, world, port, out):
    """One rank of a served job: capacities shared with bench.all_gather_objects,
    sessions partitioned, this rank's requests served (fake executor, simulated
    clock), summaries gathered and merged."""
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta

    import numpy as np
    import torch.distributed as dist
    import bench
    from test_serving_host import FakeExecutor
    from voxelmapping_b200 import serving as S
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        sizes = [int(x) for x in np.random.default_rng(0).integers(1, 20, 64) * 1000]  # the job's sessions
        caps = bench.all_gather_objects([3e5, 1e5][rank], world)  # each rank's free memory
        owner = S.partition_sessions(sizes, caps)
        reqs = S.poisson_requests(64, 1e9, 2000, seed=1)
        loc, mine = S.local_requests(reqs, owner, rank)
        lsizes = [sizes[s] for s in mine]
        sched = S.Scheduler(lsizes, sum(lsizes), max_mesh_per_tick=2)
        ex = FakeExecutor(sched)
        done, stats = S.serve(loc, sched, ex, clock=lambda: ex.t,
                              wait_until=lambda t: setattr(ex, "t", max(ex.t, t)))
        merged = S.merge_summaries(bench.all_gather_objects(S.summarize(done, stats), world))
        out.put((rank, caps, owner, mine, sum(lsizes), merged["requests"], merged["ranks"], merged["all"]["n"]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_partition_sessions_by_free_memory_and_merge_serving_summaries():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_serve_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, caps0, own0, mine0, held0, n0, k0, a0), (_, caps1, own1, mine1, held1, n1, k1, a1) = res
    assert caps0 == caps1 == [3e5, 1e5] and own0 == own1
    assert not set(mine0) & set(mine1) and sorted(mine0 + mine1) == list(range(64))
    assert held0 > held1  # the rank with more free memory holds more of the sessions' bytes
    assert n0 == n1 == 2000 and k0 == k1 == 2 and a0 == a1 == 2000
