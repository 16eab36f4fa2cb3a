"""In-tree build of the native libraries.

* ``libvmap_b200.so``  - the CUDA library behind include/vmap_c.h (sm_100a only)
* ``libvmap_synth.so`` - the synthetic RGB-D scene generator (host C++)

Run ``python -m voxelmapping_b200.build`` (or ``__graft_entry__.build()``).
Objects are rebuilt only when a source or header is newer than the output.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libvmap_b200.so"
SYNTH = PKG / "libvmap_synth.so"

CUDA_SOURCES = ["fusion.cu", "raycast.cu", "raymarch.cu", "step.cu", "mesh.cu", "map.cu", "batch.cu", "export_static.cu",
                "snapshot.cu", "vmapping.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-Wall",
                     "--expt-relaxed-constexpr", "-I" + str(ROOT / "include")]
# host compiler: the system g++ (the one nvcc uses); $CXX may point elsewhere
HOST_CXX = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"


def nvcc():
    cand = os.environ.get("CUDA_HOME", "/usr/local/cuda") + "/bin/nvcc"
    return cand if Path(cand).exists() else (shutil.which("nvcc") or "nvcc")


def _headers():
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(CSRC.glob("*.inc")) + \
        list((ROOT / "include").glob("*.h"))


def _stale(out, deps):
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(map(str, cmd)), r.stdout, r.stderr))
    if verbose and (r.stdout.strip() or r.stderr.strip()):
        print(r.stdout + r.stderr, flush=True)
    return r


def build(verbose=False):
    OBJ.mkdir(exist_ok=True)
    hdrs = _headers()
    jobs = []
    objs = []
    for src in CUDA_SOURCES:
        s = CSRC / src
        o = OBJ / (src + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs):
            jobs.append([nvcc()] + NVCC_FLAGS + ["-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=len(CUDA_SOURCES)) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    if _stale(LIB, objs):
        _run([nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"],
             verbose)
    synth_src = CSRC / "synth.cpp"
    if _stale(SYNTH, [synth_src, CSRC / "vmap_synth.h"]):
        _run([HOST_CXX, "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-shared", "-Wall", "-o", SYNTH, synth_src],
             verbose)
    return LIB


def ptxas_report(sources=("raymarch.cu", "step.cu", "fusion.cu", "mesh.cu", "raycast.cu", "batch.cu",
                           "export_static.cu", "snapshot.cu", "map.cu")):
    """Per-kernel resources as ptxas reports them (-Xptxas -v) for the given
    CUDA sources, compiled with the library's flags into a temporary
    directory: {kernel (demangled): {"registers", "spill_stores",
    "spill_loads", "stack", "smem"}}."""
    import re
    import tempfile
    with tempfile.TemporaryDirectory() as tmp:
        cmds = [[nvcc()] + NVCC_FLAGS + ["-Xptxas", "-v", "-c", CSRC / src, "-o", Path(tmp) / (src + ".o")]
                for src in sources]
        with cf.ThreadPoolExecutor(max_workers=len(cmds)) as ex:
            text = "".join(r.stderr + r.stdout for r in ex.map(lambda c: _run(c, False), cmds))
    out, cur = {}, None
    for line in text.splitlines():
        m = re.search(r"Compiling entry function '([^']+)'", line)
        if m:
            cur = m.group(1)
            out[cur] = {"registers": 0, "spill_stores": 0, "spill_loads": 0, "stack": 0, "smem": 0}
            continue
        if cur is None:
            continue
        m = re.search(r"(\d+) bytes stack frame, (\d+) bytes spill stores, (\d+) bytes spill loads", line)
        if m:
            out[cur].update(stack=int(m.group(1)), spill_stores=int(m.group(2)), spill_loads=int(m.group(3)))
        m = re.search(r"Used (\d+) registers", line)
        if m:
            out[cur]["registers"] = int(m.group(1))
            sm = re.search(r"(\d+) bytes smem", line)
            out[cur]["smem"] = int(sm.group(1)) if sm else 0
    names = list(out)
    filt = shutil.which("c++filt")
    if filt and names:
        dem = subprocess.run([filt], input="\n".join(names), capture_output=True, text=True).stdout.splitlines()
        if len(dem) == len(names):
            return {d: out[n] for n, d in zip(names, dem)}
    return out


def build_oracle(verbose=False):
    """Compile the checkers (test infrastructure) with oracle/Makefile: the
    CPU oracle, and the reference's own CUDA build (oracle/_ref/) when the
    reference sources are present; where they are not, a prebuilt
    oracle/_ref/ is used as it is."""
    cc = "CC=" + ("/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc")
    _run(["make", "-s", "-C", ROOT / "oracle", cc], verbose)
    _run(["make", "-s", "-C", ROOT / "oracle", cc, "NVCC=" + nvcc(), "ref-if-present"], verbose)
    return ROOT / "oracle" / "libvmap_oracle.so"


if __name__ == "__main__":
    if "--ptxas" in sys.argv:  # resource table of every kernel, no build
        print("| kernel | registers | spill stores / loads (B) | stack (B) | static smem (B) |")
        print("|---|---:|---:|---:|---:|")
        for k, r in sorted(ptxas_report().items()):
            print("| `%s` | %d | %d / %d | %d | %d |" % (k.replace("vmapb::", ""), r["registers"], r["spill_stores"],
                                                     r["spill_loads"], r["stack"], r["smem"]))
    else:
        build(verbose=True)
        build_oracle(verbose=True)
