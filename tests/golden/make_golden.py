"""Generate the golden fixtures that pin the oracle to the reference.

The reference (xingruiyang/VoxelMapping) has no tests and ships no data, so
the only reference data are the constants and tables in its sources (its
CUDA build, oracle/ref_harness.cu, is the other anchor). This script parses
them into JSON:

  mc_tables.json  - edgeTable[256] and triTable[256][16] (src/triangle_table.h:7-278)
  constants.json  - BLOCK_SIZE, MIN_DEPTH, MAX_DEPTH (include/map_struct.h:6-10),
                    hash primes (map_struct.h:106), truncation factor and bucket
                    fraction (src/vmapping.cpp:59), weight cap and colour blend
                    (src/depth_fusion.cu:193,377), z-range subsample
                    (src/ray_tracing.cu:7), interpolation band (ray_tracing.cu:366),
                    mesh buffer size (src/vmapping.cpp:6)

Usage: python tests/golden/make_golden.py <reference-root>
"""
import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def braces(text, anchor):
    i = text.index(anchor)
    j = text.index("{", i)
    depth, k = 0, j
    while True:
        depth += {"{": 1, "}": -1}.get(text[k], 0)
        if depth == 0:
            return text[j:k + 1]
        k += 1


def ints(s):
    return [int(t, 0) for t in re.findall(r"-?0x[0-9a-fA-F]+|-?\d+", s)]


def main(ref):
    ref = Path(ref)
    tt = (ref / "src/triangle_table.h").read_text()
    edge = ints(braces(tt, "edgeTable[256]"))
    tri = ints(braces(tt, "triTable[256][16]"))
    assert len(edge) == 256 and len(tri) == 4096
    (HERE / "mc_tables.json").write_text(json.dumps(
        {"source": "src/triangle_table.h:7-278", "edgeTable": edge,
         "triTable": [tri[16 * c:16 * c + 16] for c in range(256)]}, separators=(",", ":")))

    ms = (ref / "include/map_struct.h").read_text()
    define = lambda name: re.search(r"#define\s+%s\s+([0-9.]+)f?" % name, ms).group(1)
    primes = [int(re.search(r"pos\[%d\]\s*\*\s*(\d+)" % i, ms).group(1)) for i in range(3)]
    vm = (ref / "src/vmapping.cpp").read_text()
    trunc = int(re.search(r"voxel_size\s*\*\s*(\d+)\)", vm).group(1))
    bucket = float(re.search(r"num_voxel\s*\*\s*([0-9.]+)\)", vm).group(1))
    maxverts = int(re.search(r"#define\s+MAX_VERTS_BUFFER\s+(\d+)", vm).group(1))
    df = (ref / "src/depth_fusion.cu").read_text()
    wcap = int(re.search(r"min\((\d+),\s*oldWT \+ 1\)", df).group(1))
    blend = [float(x) for x in re.search(r"\(([0-9.]+)f \* oldRGB.*?\+ ([0-9.]+)f \* RGB\)", df).groups()]
    rt = (ref / "src/ray_tracing.cu").read_text()
    sub = int(re.search(r"#define\s+RenderingBlockSubSample\s+(\d+)", rt).group(1))
    band = float(re.search(r"sdf <= ([0-9.]+)f && sdf >= -", rt).group(1))
    consts = {"BLOCK_SIZE": int(define("BLOCK_SIZE")), "MIN_DEPTH": float(define("MIN_DEPTH")),
              "MAX_DEPTH": float(define("MAX_DEPTH")), "hash_primes": primes, "truncation_voxels": trunc,
              "bucket_fraction": bucket, "weight_cap": wcap, "rgb_blend": blend, "zrange_subsample": sub,
              "interp_band": band, "max_mesh_triangles": maxverts}
    (HERE / "constants.json").write_text(json.dumps(consts, indent=1) + "\n")
    print(consts)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference source tree>")
    main(sys.argv[1])
