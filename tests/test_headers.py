"""The public headers stand alone: include/vmap_c.h compiles as C99 and C++,
include/vmapping.h as C++17, and the C++ drop-in test program compiles and
links against libvmap_b200.so (it runs in tests/test_gpu_cpp.py)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
CUDA = Path("/usr/local/cuda")


def compiler(name):
    p = Path("/usr/bin") / name
    return str(p) if p.exists() else shutil.which(name)


@pytest.mark.parametrize("lang,flags", [("c", ["-std=c99"]), ("c++", ["-std=c++17"])])
def test_c_header_compiles_alone(tmp_path, lang, flags):
    src = tmp_path / ("t." + ("c" if lang == "c" else "cpp"))
    src.write_text('#include "vmap_c.h"\nint main(void) { vmap_config c; (void)c; return (int)sizeof(vmap_launch_config) == 0; }\n')
    cc = compiler("gcc" if lang == "c" else "g++")
    r = subprocess.run([cc, *flags, "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I" + str(ROOT / "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cpp_class_header_compiles_alone(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text('#include "vmapping.h"\nint main() { return 0; }\n')
    r = subprocess.run([compiler("g++"), "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                        "-I" + str(ROOT / "include"), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cpp_drop_in_program_links(tmp_path):
    lib = ROOT / "voxelmapping_b200" / "libvmap_b200.so"
    if not lib.exists():
        pytest.skip("library not built")
    exe = tmp_path / "t"
    r = subprocess.run([compiler("g++"), "-std=c++17", "-O1", str(ROOT / "tests" / "cpp" / "test_vmapping.cpp"), "-o",
                        str(exe), "-I" + str(ROOT / "include"), "-I" + str(CUDA / "include"),
                        "-L" + str(lib.parent), "-lvmap_b200", "-L" + str(CUDA / "lib64"), "-lcudart"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_drop_in_example_compiles():
    """tests/cpp/drop_in_example.cpp, the drop-in use of the class (construct,
    CreateMap, fuse from device and host buffers, render, mesh), compiles
    against include/vmapping.h as declared."""
    r = subprocess.run([compiler("g++"), "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I" + str(ROOT / "include"),
                        str(ROOT / "tests" / "cpp" / "drop_in_example.cpp")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
