"""Generate ``mc_table.inc``: the marching-cubes triangulation in packed form.

Mesh parity with the reference requires the exact same triangulation table
(the classic 256-case Lorensen-Cline table, published by P. Bourke), so this
script reads the reference's ``src/triangle_table.h`` (``triTable[256][16]``,
lines 22-278) and re-encodes it for the GPU:

* one ``uint64`` per cube case: 15 edge-index nibbles (bits 0..59, triangle
  ``t`` uses nibbles ``3t..3t+2``) and the triangle count in bits 60..63.
  256 x 8 B = 2 KiB, small enough to stage in shared memory per CTA.

The edge table (``edgeTable[256]``, same file lines 7-20) is not stored: it is
derived from the cube topology and the script asserts that the derivation
equals the reference's table.

Run once when the table source changes (output is committed):
    python voxelmapping_b200/csrc/gen_mc_table.py <path-to-triangle_table.h>
"""
import re
import sys
from pathlib import Path

# Corner order used by the reference's marching cubes (marching_cubes.cu:75-99)
CORNERS = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0),
           (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
# Edge -> (corner a, corner b) (marching_cubes.cu:145-204)
EDGES = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4),
         (0, 4), (1, 5), (2, 6), (3, 7)]


def derived_edge_table():
    out = []
    for c in range(256):
        m = 0
        for e, (a, b) in enumerate(EDGES):
            if ((c >> a) & 1) != ((c >> b) & 1):
                m |= 1 << e
        out.append(m)
    return out


def parse_tables(text):
    def block(name):
        i = text.index(name)
        j = text.index("{", i)
        depth, k = 0, j
        while True:
            if text[k] == "{":
                depth += 1
            elif text[k] == "}":
                depth -= 1
                if depth == 0:
                    break
            k += 1
        return [int(tok, 0) for tok in re.findall(r"-?0x[0-9a-fA-F]+|-?\d+", text[j:k + 1])]

    edge = block("edgeTable[256]")
    tri = block("triTable[256][16]")
    assert len(edge) == 256 and len(tri) == 256 * 16
    return edge, [tri[16 * c:16 * c + 16] for c in range(256)]


def pack(tri_rows):
    packed = []
    for row in tri_rows:
        n = row.index(-1) if -1 in row else 16
        assert n % 3 == 0 and n <= 15
        word = (n // 3) << 60
        for i, e in enumerate(row[:n]):
            assert 0 <= e < 12
            word |= e << (4 * i)
        packed.append(word)
    return packed


def main(src):
    edge, tri = parse_tables(Path(src).read_text())
    assert edge == derived_edge_table(), "edge table differs from cube topology"
    words = pack(tri)
    lines = ["// Generated by gen_mc_table.py -- do not edit.",
             "// Packed marching-cubes triangulation: nibble i (bits 4i..4i+3) is the",
             "// edge of triangle vertex i, bits 60..63 the triangle count.",
             "#define VMAP_MC_TRI_PACKED_INIT { \\"]
    for r in range(0, 256, 4):
        lines.append("    " + ", ".join("0x%016xULL" % w for w in words[r:r + 4]) + ", \\")
    lines.append("}")
    out = Path(__file__).with_name("mc_table.inc")
    out.write_text("\n".join(lines) + "\n")
    print("wrote", out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: gen_mc_table.py <reference tree>/src/triangle_table.h")
    main(sys.argv[1])
