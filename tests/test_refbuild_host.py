"""CPU checks of the reference-build harness (oracle/refbuild.py,
oracle/ref_harness.cu): it loads and binds every entry point, its bucket
function agrees with the oracle's, and the product never loads it."""
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from oracle import refbuild as R

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.skipif(not R.available(), reason="reference build missing (make -C oracle ref)")
def test_reference_build_loads_and_binds_every_entry_point():
    lib = R.lib()
    for name in R.SYMBOLS:
        assert hasattr(lib, name), name
    exported = set(re.findall(r"^\w[\w\s\*]*?\b(ref_\w+)\(", (ROOT / "oracle" / "ref_harness.cu").read_text(),
                              re.M))
    assert exported == set(R.SYMBOLS), exported ^ set(R.SYMBOLS)


def test_bucket_function_matches_the_oracle():
    rng = np.random.default_rng(3)
    coords = np.concatenate([rng.integers(-2000, 2000, (3000, 3)),
                             rng.integers(-(1 << 20), 1 << 20, (3000, 3)),
                             np.array([[0, 0, 0], [-1, -1, -1], [(1 << 20) - 1, -(1 << 20), 7]])])
    for nb in (1, 7, 235929, 943718, (1 << 31) - 1):
        got = R.hash_bucket(coords, nb)
        want = [O.block_hash(int(x), int(y), int(z), nb) for x, y, z in coords]
        assert np.array_equal(got, want), nb


def test_product_never_loads_the_checkers():
    # build.py compiles the checkers (the build step); nothing else names them
    for f in list((ROOT / "voxelmapping_b200").rglob("*.py")) + list((ROOT / "voxelmapping_b200" / "csrc").glob("*")):
        if f.is_file() and f.suffix in (".py", ".cu", ".cuh", ".h", ".cpp") and f.name != "build.py":
            text = f.read_text()
            assert not re.search(r"\bimport oracle\b|from oracle\b|refbuild|libvmap_ref|libvmap_oracle", text), f
