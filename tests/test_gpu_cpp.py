"""The C++ drop-in class (include/vmapping.h) against the Python/ctypes path:
tests/cpp/test_vmapping.cpp is compiled against libvmap_b200.so, drives the
reference-style class (host and device fuse, RenderScene into an empty image,
computeNormal, Polygonize, GetSurfacePoints) and must produce bit-identical
vertex maps, normals and meshes."""
import shutil
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest
import torch

from tests.common import sorted_rows
from voxelmapping_b200 import VoxelMapping, synth

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


def build_cpp(tmp):
    exe = tmp / "test_vmapping"
    cuda = Path("/usr/local/cuda")
    cxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else shutil.which("g++")
    cmd = [cxx, "-std=c++17", "-O2", str(ROOT / "tests" / "cpp" / "test_vmapping.cpp"), "-o", str(exe),
           "-I" + str(ROOT / "include"), "-I" + str(cuda / "include"), "-L" + str(ROOT / "voxelmapping_b200"),
           "-lvmap_b200", "-L" + str(cuda / "lib64"), "-lcudart", "-Wl,-rpath," + str(ROOT / "voxelmapping_b200"),
           "-Wl,-rpath," + str(cuda / "lib64")]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_class_matches_python_path(tmp_path):
    exe = build_cpp(tmp_path)
    wl = synth.WORKLOADS["room_small"]
    sc = synth.Scene(wl)
    frames = [sc.render(i) for i in (0, 4, 8)]
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        f.write(struct.pack("<5i5f", wl.width, wl.height, len(frames), wl.num_entries, 1 << 16, wl.fx, wl.fy, wl.cx,
                            wl.cy, wl.voxel_size))
        for d, c, p in frames:
            f.write(p.astype(np.float32).tobytes())
            f.write(synth.depth_to_metres(d).tobytes())
            f.write(c.tobytes())
    out = tmp_path / "out.bin"
    r = subprocess.run([str(exe), str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stderr
    raw = out.read_bytes()
    n = wl.width * wl.height * 4
    off = 0
    v_cpp = np.frombuffer(raw, np.float32, n, off).reshape(wl.height, wl.width, 4); off += 4 * n
    n_cpp = np.frombuffer(raw, np.float32, n, off).reshape(wl.height, wl.width, 4); off += 4 * n
    ntri = struct.unpack_from("<i", raw, off)[0]; off += 4
    verts_cpp = np.frombuffer(raw, np.float32, ntri * 9, off).reshape(-1, 9); off += 36 * ntri
    norms_cpp = np.frombuffer(raw, np.float32, ntri * 9, off).reshape(-1, 9); off += 36 * ntri
    npts = struct.unpack_from("<i", raw, off)[0]; off += 4
    pts_cpp = np.frombuffer(raw, np.float32, npts * 3, off).reshape(-1, 3)

    # the same calls through the Python mirror (poses rounded to float like the C++ Mat4f)
    vm = VoxelMapping(wl.width, wl.height, wl.K, voxel_format="ref", with_color=True)
    vm.CreateMap(wl.num_entries, 1 << 16, wl.voxel_size)
    for i, (d, c, p) in enumerate(frames):
        pf = p.astype(np.float32).astype(np.float64)
        dm = synth.depth_to_metres(d)
        if i + 1 < len(frames):
            vm.FuseDepthAndImage(c, dm, pf)
        else:
            vm.FuseDepth(torch.from_numpy(dm).cuda(), pf)
    nm = torch.empty((wl.height, wl.width, 4), dtype=torch.float32, device="cuda")
    v_py = vm.RenderScene(None, pf, nmap=nm).cpu().numpy()
    n_py = nm.cpu().numpy()
    k, verts, norms = vm.Polygonize()
    assert np.array_equal(np.nan_to_num(v_cpp, nan=-9), np.nan_to_num(v_py, nan=-9))
    assert np.array_equal(np.nan_to_num(n_cpp, nan=-9), np.nan_to_num(n_py, nan=-9))
    assert ntri == k > 1000 and npts == ntri
    assert np.array_equal(sorted_rows(np.concatenate([verts_cpp, norms_cpp], 1)),
                          sorted_rows(np.concatenate([verts, norms], 1)))
    assert np.array_equal(sorted_rows(pts_cpp), sorted_rows(vm.GetSurfacePoints()))
