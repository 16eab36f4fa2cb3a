"""Pins: the reference's own tables and constants (the only reference data that
exists: it ships no tests) against the oracle and the product's packed table."""
import json
import os
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
# the reference tree, when present (fixtures regenerate from it)
REFERENCE = Path(os.environ["VMAP_REFERENCE_DIR"]) if os.environ.get("VMAP_REFERENCE_DIR") else None


def golden_tables():
    g = json.loads((GOLDEN / "mc_tables.json").read_text())
    return np.array(g["edgeTable"]), np.array(g["triTable"])


def product_packed_table():
    text = (ROOT / "voxelmapping_b200" / "csrc" / "mc_table.inc").read_text()
    return [int(t, 16) for t in re.findall(r"0x([0-9a-f]{16})ULL", text)]


CORNER_EDGES = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]


def test_packed_table_matches_reference_tritable():
    _, tri = golden_tables()
    packed = product_packed_table()
    assert len(packed) == 256
    for c in range(256):
        row = list(tri[c])
        n = row.index(-1) if -1 in row else 16
        assert packed[c] >> 60 == n // 3, c
        for i in range(n):
            assert (packed[c] >> (4 * i)) & 15 == row[i], (c, i)
        assert packed[c] & ((1 << (4 * n)) - 1) == packed[c] & ((1 << 60) - 1), c  # no stray nibbles


def test_edge_table_is_cube_topology():
    edge, tri = golden_tables()
    for c in range(256):
        m = 0
        for e, (a, b) in enumerate(CORNER_EDGES):
            if ((c >> a) & 1) != ((c >> b) & 1):
                m |= 1 << e
        assert m == edge[c], c
        used = {int(e) for e in tri[c] if e >= 0}
        assert all((edge[c] >> e) & 1 for e in used), c


def test_oracle_constants_match_reference():
    g = json.loads((GOLDEN / "constants.json").read_text())
    o = O.constants()
    assert o["block"] == g["BLOCK_SIZE"] == 8
    assert o["min_depth_mm"] == round(g["MIN_DEPTH"] * 1000)
    assert o["max_depth_mm"] == round(g["MAX_DEPTH"] * 1000)
    assert [o["p0"], o["p1"], o["p2"]] == g["hash_primes"]
    assert o["trunc_factor"] == g["truncation_voxels"]
    assert o["weight_cap"] == g["weight_cap"]
    assert o["subsample"] == g["zrange_subsample"]
    assert g["rgb_blend"] == [0.7, 0.3] and g["interp_band"] == 0.5 and g["bucket_fraction"] == 0.9


@pytest.mark.skipif(REFERENCE is None or not REFERENCE.exists(), reason="VMAP_REFERENCE_DIR not set")
def test_fixtures_reproduce_from_reference(tmp_path, monkeypatch):
    import importlib.util
    spec = importlib.util.spec_from_file_location("mg", GOLDEN / "make_golden.py")
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    monkeypatch.setattr(mg, "HERE", tmp_path)
    mg.main(REFERENCE)
    for f in ("mc_tables.json", "constants.json"):
        assert json.loads((tmp_path / f).read_text()) == json.loads((GOLDEN / f).read_text()), f
