"""`bench.py --impl reference` on CPU: the oracle port on the host cores prints
one JSON line with the bench contract's keys, the per-stage CPU times (fuse,
raycast + normals, mesh), a one-thread sample, the FP64 oracle beside, the
oracle's block counts, and the reference CUDA build's entry (unavailable
without a GPU)."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_prints_one_contract_line():
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1",
                          "--prefix", "3"],
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["unit"] == "frames/s" and line["higher_is_better"] is True
    assert line["steps"] == 2 and line["warmup"] == 1 and line["value"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert cb["frames_timed"] == 2 and "frames 4..5" in cb["sample"] and cb["prefix_frames_untimed"] == 3
    assert cb["fp64"]["value"] > 0 and set(cb["oracle_counts_mean"]) == {"visible", "alloc_touched", "ray_blocks"}
    assert 0 < cb["oracle_counts_mean"]["ray_blocks"] <= cb["oracle_counts_mean"]["visible"]
    assert "unavailable" in line["reference_cuda_build"] or line["reference_cuda_build"]["value"] > 0
    assert line["config"]["frames"] == "4..5"
    for k in ("frame_ms", "fuse_ms", "raycast_normals_ms"):
        assert 0 < cb[k]["p50"] <= cb[k]["p99"]
    assert cb["mesh"]["triangles"] > 0 and cb["mesh"]["ms"] > 0
    assert cb["one_thread"]["frames/s"] > 0
    assert line["e2e"] == {"value": line["value"], "unit": "frames/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_cpu_baseline_renders_frames_past_the_sample_for_the_one_thread_run():
    sys.path.insert(0, str(ROOT))
    import bench
    from voxelmapping_b200 import synth
    wl = synth.WORKLOADS["room_small"]
    scene = synth.Scene(wl)
    frames = [scene.render(i) for i in range(2)]
    cb = bench.cpu_baseline(wl, scene, frames, 2, seconds=30.0)
    assert cb["frames_timed"] == 2 and cb["cores"] == 2
    assert cb["one_thread"]["sample"] == "frames 2..3 on the same map"
    assert cb["mesh"]["map_frames"] == 2 and cb["mesh"]["triangles"] > 0
