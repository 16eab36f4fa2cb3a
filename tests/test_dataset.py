"""TUM-format loader (voxelmapping_b200.dataset, after the reference's
example/dataset_loader.cpp) and the PLY mesh writer, on the CPU."""
import numpy as np

from voxelmapping_b200 import dataset as D
from voxelmapping_b200 import meshio, synth


def test_tum_round_trip(tmp_path):
    wl = synth.WORKLOADS["room_small"]
    sc = synth.Scene(wl)
    frames = []
    for i in (0, 5, 10, 15):
        d, c, p = sc.render(i)
        frames.append((synth.depth_to_metres(d), c, p))
    D.write_tum(tmp_path, frames, wl.K)
    lo = D.DatasetLoader(str(tmp_path))
    assert lo.loadImages(True) and lo.loadGroundTruth()
    K = lo.loadCalibration()
    assert K.dtype == np.float32 and np.allclose(K, wl.K, atol=1e-6)
    assert len(lo) == 4 and np.allclose(lo.getFirstFramePose(), frames[0][2], atol=1e-8)
    got = list(lo)
    assert len(got) == 4 and lo.GetNext() is None
    for (d, c, p), (du, col, t, pose) in zip(frames, got):
        assert du.dtype == np.uint16 and du.shape == d.shape
        assert np.array_equal(du, np.clip(np.round(d.astype(np.float64) * 5000), 0, 65535).astype(np.uint16))
        assert np.array_equal(col, c)
        assert np.allclose(pose, p, atol=1e-8)  # nearest ground truth, not the decoy
        assert np.allclose(du * D.DEPTH_SCALE, d, atol=1e-4)
    lo.reset()
    assert lo.GetNext()[2] == got[0][2]


def test_quaternion_pose_matches_reference_convention():
    # qw first in Eigen's constructor, (qx, qy, qz, qw) in the file; normalised
    T = D.quat_to_pose([1, 2, 3], [0, 0, 2 * np.sin(np.pi / 8), 2 * np.cos(np.pi / 8)])  # 45 deg about z, scaled
    c = np.cos(np.pi / 4)
    assert np.allclose(T[:3, :3], [[c, -c, 0], [c, c, 0], [0, 0, 1]]) and np.allclose(T[:3, 3], [1, 2, 3])
    rng = np.random.default_rng(0)
    for _ in range(50):
        q = rng.normal(size=4)
        R = D.quat_to_pose([0, 0, 0], q)[:3, :3]
        assert np.allclose(D.quat_to_pose([0, 0, 0], D._rot_to_quat(R))[:3, :3], R, atol=1e-12)


def test_ply_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    v = rng.normal(size=(100, 9)).astype(np.float32)
    n = rng.normal(size=(100, 9)).astype(np.float32)
    meshio.write_ply(tmp_path / "m.ply", v, n)
    v2, n2 = meshio.read_ply(tmp_path / "m.ply")
    assert np.array_equal(v, v2) and np.array_equal(n, n2)
    meshio.write_ply(tmp_path / "m2.ply", v)
    v3, n3 = meshio.read_ply(tmp_path / "m2.ply")
    assert np.array_equal(v, v3) and n3 is None
