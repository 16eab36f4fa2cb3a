"""The ctypes mirror of include/vmap_c.h matches the C declarations (no GPU):
every struct's size and field offsets, as a C compiler lays them out, and every
function's parameter count and return type."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest
import torch

from voxelmapping_b200 import _lib as L
from voxelmapping_b200 import snapshot_header

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "vmap_c.h"

STRUCTS = {"vmap_config": L.Config, "vmap_stats": L.Stats, "vmap_host_frame": L.HostFrame,
           "vmap_launch_config": L.LaunchConfig, "vmap_batch_frame": L.BatchFrame,
           "vmap_snapshot_header": L.SnapshotHeader}


def c_layout(tmp_path):
    src = ["#include <stdio.h>", "#include <stddef.h>", '#include "vmap_c.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        src.append('printf("%s . %%zu %%zu\\n", (size_t)0, sizeof(%s));' % (cname, cname))
        for f, _ in py._fields_:
            src.append('printf("%s %s %%zu %%zu\\n", offsetof(%s, %s), sizeof(((%s*)0)->%s));'
                       % (cname, f, cname, f, cname, f))
    src += ["return 0;", "}"]
    (tmp_path / "layout.c").write_text("\n".join(src) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(tmp_path / "layout.c"),
                    "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {(a, b): (int(c), int(d)) for a, b, c, d in (l.split() for l in out.splitlines())}


def test_ctypes_structs_match_the_c_layout(tmp_path):
    lay = c_layout(tmp_path)
    for cname, py in STRUCTS.items():
        assert lay[(cname, ".")][1] == C.sizeof(py), cname
        for f, _ in py._fields_:
            d = getattr(py, f)
            assert lay[(cname, f)] == (d.offset, d.size), (cname, f)
    assert C.sizeof(L.SnapshotHeader) == 64


def declarations():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    decl = re.findall(r"^(vmap_status|void|int|size_t|const char\s*\*)\s*(vmap_\w+)\s*\(([^;]*?)\)\s*;", text,
                      flags=re.M | re.S)
    return {name: (ret.replace(" ", ""), 0 if args.strip() in ("", "void") else args.count(",") + 1)
            for ret, name, args in decl}


def test_ctypes_signatures_match_the_declarations():
    decl = declarations()
    assert len(decl) >= 40
    assert set(decl) == set(L.SIGNATURES), set(decl) ^ set(L.SIGNATURES)
    want_res = {"vmap_status": C.c_int, "int": C.c_int, "void": None, "size_t": C.c_size_t,
                "constchar*": C.c_char_p}
    for name, (ret, nargs) in decl.items():
        res, args = L.SIGNATURES[name]
        assert res is want_res[ret], name
        assert len(args) == nargs, (name, len(args), nargs)


def test_snapshot_header_reader():
    h = L.SnapshotHeader(magic=b"VMAPSNAP", version=1, header_bytes=64, voxel_format=L.VOXEL_F16, with_color=1,
                         block_bytes=512 * 7, n_blocks=3, voxel_size=0.005, truncation=0.02, max_weight=0,
                         error_flags=0, keys_offset=64, pool_offset=256)
    img = np.zeros(256 + 3 * 512 * 7, np.uint8)
    img[:64] = np.frombuffer(bytes(h), np.uint8)
    for form in (img, bytes(img), torch.from_numpy(img)):
        f = snapshot_header(form)
        assert f["n_blocks"] == 3 and f["block_bytes"] == 512 * 7 and f["pool_offset"] == 256
        assert f["voxel_format"] == L.VOXEL_F16 and f["with_color"] == 1
        assert f["voxel_size"] == pytest.approx(0.005)
    with pytest.raises(ValueError):
        snapshot_header(img[:32])
    bad = img.copy()
    bad[0] = ord("X")
    with pytest.raises(ValueError):
        snapshot_header(bad)


def expected_map_bytes(w, h, num_entries, num_blocks, fmt, color):
    """Device bytes of one map as documented: hash slots (4 x 16 B per bucket;
    buckets = int(0.9 numVoxels), raised to cover numEntries), block keys,
    voxel pool, 16 counters, visible list, near and far z-range tiles (8x8
    pixels), a triangle counter, 7 forward neighbour links per block; each
    buffer starts on a 256-byte boundary."""
    nb = max(int(num_blocks * 0.9), 1)
    nb = max(nb, -(-num_entries // 4))
    tiles = -(-w // 8) * -(-h // 8)
    bb = L.lib().vmap_block_bytes(fmt, color)
    sizes = [nb * 4 * 16, num_blocks * 8, num_blocks * bb, 16 * 4, num_blocks * 4, tiles * 8, tiles * 8, 4,
             num_blocks * 7 * 4]
    return sum(-(-s // 256) * 256 for s in sizes)


@pytest.mark.parametrize("case", [(640, 480, 1 << 21, 1 << 20, L.VOXEL_F32, 1), (320, 240, 0, 1 << 18, L.VOXEL_REF, 0),
                                  (1280, 720, 1 << 20, 1 << 16, L.VOXEL_F16, 1), (64, 48, 0, 1000, L.VOXEL_I16, 0)])
def test_required_bytes_matches_the_documented_layout(case):
    w, h, ne, nb, fmt, color = case
    cfg = L.Config(width=w, height=h, fx=500.0, fy=500.0, cx=w / 2, cy=h / 2, num_entries=ne, num_blocks=nb,
                   voxel_size=0.005, num_buckets=0, truncation=0.0, voxel_format=fmt, max_weight=0, with_color=color,
                   raycast_mode=0)
    got = C.c_uint64()
    assert L.lib().vmap_required_bytes(C.byref(cfg), C.byref(got)) == L.VMAP_OK
    assert got.value == expected_map_bytes(w, h, ne, nb, fmt, color)
    bad = L.Config(**{k: getattr(cfg, k) for k, _ in L.Config._fields_})
    bad.voxel_size = 0.0
    assert L.lib().vmap_required_bytes(C.byref(bad), C.byref(got)) == 1  # VMAP_ERR_INVALID_ARG


def test_every_entry_point_refuses_null_and_bad_sizes_without_a_device():
    """Misuse is refused on the host with VMAP_ERR_INVALID_ARG (1) before any
    device call: NULL handles and pointers, batch sizes outside 1..256,
    unknown formats, misaligned or too small caller memory."""
    lib = L.lib()
    out, u64 = C.c_void_p(), C.c_uint64()
    cfg = L.Config(64, 48, 50.0, 50.0, 32.0, 24.0, 0, 1024, 0.01, 0, 0.0, 1, 0, 0, 0)
    pose = (C.c_double * 16)(1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1)
    calls = {
        "vmap_create": lambda: lib.vmap_create(None, C.byref(out)),
        "vmap_destroy": lambda: lib.vmap_destroy(None),
        "vmap_reset": lambda: lib.vmap_reset(None, None),
        "vmap_get_config": lambda: lib.vmap_get_config(None, None),
        "vmap_required_bytes": lambda: lib.vmap_required_bytes(None, C.byref(u64)),
        "vmap_create_in": lambda: (lib.vmap_create_in(C.byref(cfg), C.c_void_p(0x1001), 1 << 30, None, C.byref(out)),
                                   lib.vmap_create_in(C.byref(cfg), None, 1 << 30, None, C.byref(out)),
                                   lib.vmap_create_in(C.byref(cfg), C.c_void_p(1 << 20), 1024, None, C.byref(out))),
        "vmap_fuse_depth": lambda: lib.vmap_fuse_depth(None, None, 0, 0, 1.0, pose, None),
        "vmap_fuse_depth_rgb": lambda: lib.vmap_fuse_depth_rgb(None, None, 0, 0, 1.0, None, 0, pose, None),
        "vmap_fuse_host": lambda: lib.vmap_fuse_host(None, None, 0, 1.0, None, pose, None),
        "vmap_check_visible_blocks": lambda: lib.vmap_check_visible_blocks(None, pose, None),
        "vmap_render_scene": lambda: lib.vmap_render_scene(None, pose, None, 0, None, 0, None),
        "vmap_render_scene_host": lambda: lib.vmap_render_scene_host(None, pose, None, None, None),
        "vmap_compute_normal": lambda: lib.vmap_compute_normal(None, 0, None, 0, 64, 48, None),
        "vmap_render_phong": lambda: lib.vmap_render_phong(None, 0, None, 0, None, 0, 64, 48, None),
        "vmap_frame_host_async": lambda: lib.vmap_frame_host_async(None, None, None),
        "vmap_host_wait": lambda: lib.vmap_host_wait(None, None),
        "vmap_polygonize": lambda: lib.vmap_polygonize(None, None, None, 0, None, None),
        "vmap_polygonize_host": lambda: lib.vmap_polygonize_host(None, None, None, None, None),
        "vmap_surface_points": lambda: lib.vmap_surface_points(None, 4, None, None),
        "vmap_batch_create": lambda: (lib.vmap_batch_create(None, 0, C.byref(out)),
                                      lib.vmap_batch_create((C.c_void_p * 257)(), 257, C.byref(out))),
        "vmap_batch_create_slots": lambda: (lib.vmap_batch_create_slots(0, 1, C.byref(out)),
                                            lib.vmap_batch_create_slots(257, 1, C.byref(out)),
                                            lib.vmap_batch_create_slots(4, 9, C.byref(out))),
        "vmap_batch_set_map": lambda: lib.vmap_batch_set_map(None, 0, None),
        "vmap_batch_destroy": lambda: lib.vmap_batch_destroy(None),
        "vmap_batch_step": lambda: lib.vmap_batch_step(None, None, None),
        # (a non-NULL batch with a stall limit out of range is refused before it is read)
        "vmap_batch_stall_probe": lambda: (lib.vmap_batch_stall_probe(None, None, 100, None),
                                           lib.vmap_batch_stall_probe(C.c_void_p(1), (L.BatchFrame * 1)(), 0, None),
                                           lib.vmap_batch_stall_probe(C.c_void_p(1), (L.BatchFrame * 1)(), 10001,
                                                                      None)),
        "vmap_get_launch_config": lambda: lib.vmap_get_launch_config(None, None),
        "vmap_set_launch_config": lambda: lib.vmap_set_launch_config(None, None),
        "vmap_batch_get_launch_config": lambda: lib.vmap_batch_get_launch_config(None, None),
        "vmap_batch_set_launch_config": lambda: lib.vmap_batch_set_launch_config(None, None),
        "vmap_get_stats": lambda: lib.vmap_get_stats(None, None, None),
        "vmap_clear_errors": lambda: lib.vmap_clear_errors(None, None),
        "vmap_copy_counters": lambda: lib.vmap_copy_counters(None, None, None),
        "vmap_export_blocks": lambda: lib.vmap_export_blocks(None, None, None, None, None, 0, None, None),
        "vmap_export_blocks_static": lambda: lib.vmap_export_blocks_static(None, 0, 1, None, None, None, None, None,
                                                                           None),
        "vmap_snapshot_save": lambda: lib.vmap_snapshot_save(None, None, 0, C.byref(u64), None),
        "vmap_snapshot_load": lambda: lib.vmap_snapshot_load(None, None, 0, None),
        "vmap_timing_enable": lambda: lib.vmap_timing_enable(None, 4),
        "vmap_timing_read": lambda: lib.vmap_timing_read(None, None, None),
        "vmap_block_hash_device": lambda: lib.vmap_block_hash_device(None, 4, 100, None, None),
    }
    for name, call in calls.items():
        got = call()
        for st in (got if isinstance(got, tuple) else (got,)):
            assert st == 1, (name, st)
    # every entry point that takes a handle or a buffer is covered; the rest are pure helpers
    helpers = {"vmap_pose_inverse", "vmap_block_hash", "vmap_block_bytes", "vmap_status_string", "vmap_last_error",
               "vmap_abi_version"}
    assert set(calls) | helpers == set(declarations()), set(declarations()) - set(calls) - helpers
