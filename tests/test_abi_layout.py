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
