"""The hash the GPU table uses (remainder by multiplication) equals the
reference formula (map_struct.h:104-109) over the whole int32 range."""
import numpy as np
import pytest
import torch

from voxelmapping_b200 import _lib as L

pytestmark = pytest.mark.gpu


def test_device_hash_equals_reference_formula():
    rng = np.random.default_rng(7)
    n = 200000
    xyz = rng.integers(-(2 ** 31), 2 ** 31, size=(n, 3), dtype=np.int64).astype(np.int32)
    xyz[:1000] = rng.integers(-(2 ** 20), 2 ** 20, size=(1000, 3))
    xyz[1000] = (-(2 ** 31), -(2 ** 31), -(2 ** 31))
    xyz[1001] = (2 ** 31 - 1, 0, -1)
    lib = L.lib()
    d_xyz = torch.from_numpy(xyz).cuda()
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for nb in (1, 2, 7, 235929, 943718, 2 ** 20, 2 ** 31 - 1):
        L.check(lib.vmap_block_hash_device(d_xyz.data_ptr(), n, nb, out.data_ptr(), stream))
        got = out.cpu().numpy()
        want = np.array([lib.vmap_block_hash(int(a), int(b), int(c), nb) for a, b, c in xyz[:5000]])
        assert np.array_equal(got[:5000], want), nb
        # the rest against a vectorised restatement of the same formula
        h = (xyz[:, 0].astype(np.uint32) * np.uint32(73856093)) ^ (xyz[:, 1].astype(np.uint32) * np.uint32(19349669)) \
            ^ (xyz[:, 2].astype(np.uint32) * np.uint32(83492791))
        r = h.view(np.int32).astype(np.int64)
        m = np.fmod(r, nb)  # C remainder
        m = np.where(m < 0, m + nb, m)
        assert np.array_equal(got, m.astype(np.int32)), nb
