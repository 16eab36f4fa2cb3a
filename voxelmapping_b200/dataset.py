"""TUM RGB-D format sequences (the reference example's DatasetLoader,
example/dataset_loader.cpp:28-166, example/dataset_loader.h:14-29).

A dataset directory holds
  associated.txt   - lines "t_rgb rgb/xxx.png t_depth depth/xxx.png" ('#' starts a comment)
  groundtruth.txt  - lines "t tx ty tz qx qy qz qw" (camera-to-world)
  calibration.txt  - first line "fx fy cx cy"
Depth PNGs are uint16 at 5000 units per metre (DEPTH_SCALE). Each frame gets
the ground-truth pose with the nearest timestamp (the first such line on a
tie), as in DatasetLoader::loadGroundTruth. Images are read as stored
(cv::imread(path, -1): colour in OpenCV's BGR order).

    loader = DatasetLoader(path)
    loader.loadImages(True); loader.loadGroundTruth()
    K = loader.loadCalibration()
    while (f := loader.GetNext()) is not None:
        depth_u16, color, t, cam_to_world = f
        vm.FuseDepth(torch.from_numpy(depth_u16.view(np.int16)).cuda(), cam_to_world, depth_scale=DEPTH_SCALE)
"""
from pathlib import Path

import numpy as np

DEPTH_SCALE = 1.0 / 5000.0  # TUM depth units per metre: depth.convertTo(..., 1 / 5000.0)


def quat_to_pose(t, q):
    """camToWorld from a translation and a quaternion (qx, qy, qz, qw),
    normalised first (Eigen::Quaterniond::normalize + toRotationMatrix)."""
    x, y, z, w = np.asarray(q, np.float64) / np.linalg.norm(q)
    T = np.eye(4)
    T[:3, :3] = [[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                 [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                 [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]]
    T[:3, 3] = t
    return T


def _lines(path):
    with open(path) as f:
        for line in f:
            line = line.rstrip("\n")
            if line and not line.startswith("#"):
                yield line.split()


class DatasetLoader:
    def __init__(self, filepath):
        self.root = Path(filepath)
        self.calib_path = self.root / "calibration.txt"
        self.gt_path = self.root / "groundtruth.txt"
        self.assoc_path = self.root / "associated.txt"
        self.color_paths, self.depth_paths, self.timestamps, self.ground_truth = [], [], [], []
        self.start = self.end = self.pos = 0

    def reset(self):
        self.pos = self.start

    def loadImages(self, pathOnly=True):
        """Reads associated.txt (the RGB timestamp is the frame's time)."""
        self.color_paths, self.depth_paths, self.timestamps = [], [], []
        for tok in _lines(self.assoc_path):
            self.timestamps.append(float(tok[0]))
            self.color_paths.append(self.root / tok[1])
            self.depth_paths.append(self.root / tok[3])
        self.start, self.end, self.pos = 0, len(self.timestamps), 0
        return True

    def loadGroundTruth(self):
        """Nearest-timestamp pose per frame; False when the file holds none."""
        times, poses = [], []
        for tok in _lines(self.gt_path):
            v = [float(x) for x in tok[:8]]
            times.append(v[0])
            poses.append(quat_to_pose(v[1:4], v[4:8]))
        if not times:
            return False
        times = np.asarray(times)
        self.ground_truth = []
        for t in self.timestamps:
            diff = np.abs(times - t)
            i = int(np.argmin(diff))  # the first minimum, like the reference's strict '<' scan
            if not diff[i] < 1000.0:  # the reference leaves no pose within 1000 s undefined
                raise ValueError("no ground-truth pose within 1000 s of frame time %.6f" % t)
            self.ground_truth.append(poses[i])
        return len(self.ground_truth) == len(self.timestamps)

    def loadCalibration(self):
        """K as float32 3x3 from the first line "fx fy cx cy"."""
        fx, fy, cx, cy = (float(x) for x in next(_lines(self.calib_path))[:4])
        K = np.eye(3, dtype=np.float32)
        K[0, 0], K[1, 1], K[0, 2], K[1, 2] = fx, fy, cx, cy
        return K

    def getFirstFramePose(self):
        return self.ground_truth[0]

    def GetNext(self):
        """(depth uint16 (h, w), colour as stored, time, camToWorld float64 4x4
        or None without ground truth), or None after the last frame."""
        import cv2
        if self.pos == self.end:
            return None
        i = self.pos
        depth = cv2.imread(str(self.depth_paths[i]), cv2.IMREAD_UNCHANGED)
        color = cv2.imread(str(self.color_paths[i]), cv2.IMREAD_UNCHANGED)
        if depth is None or color is None:
            raise FileNotFoundError("cannot read %s or %s" % (self.depth_paths[i], self.color_paths[i]))
        pose = self.ground_truth[i] if self.ground_truth else None
        self.pos += 1
        return depth, color, self.timestamps[i], pose

    def __len__(self):
        return self.end - self.start

    def __iter__(self):
        self.reset()
        while (f := self.GetNext()) is not None:
            yield f


def write_tum(path, frames, K, times=None, gt_offset=0.004):
    """Writes frames [(depth_m float32 (h, w), colour uint8 (h, w, 3), camToWorld 4x4), ...]
    as a TUM-format directory (depth at 5000 units per metre; ground truth at
    times offset by `gt_offset` s, with a decoy pose between frames). Used to
    check the loader and to feed the library recorded-style data."""
    import cv2
    root = Path(path)
    (root / "rgb").mkdir(parents=True, exist_ok=True)
    (root / "depth").mkdir(parents=True, exist_ok=True)
    times = times if times is not None else [1000.0 + 0.033 * i for i in range(len(frames))]
    with open(root / "associated.txt", "w") as fa, open(root / "groundtruth.txt", "w") as fg:
        fa.write("# rgb depth\n")
        fg.write("# timestamp tx ty tz qx qy qz qw\n")
        for i, ((d, c, T), t) in enumerate(zip(frames, times)):
            du = np.clip(np.round(np.nan_to_num(d, nan=0.0).astype(np.float64) * 5000.0), 0, 65535).astype(np.uint16)
            cv2.imwrite(str(root / "depth" / ("%06d.png" % i)), du)
            cv2.imwrite(str(root / "rgb" / ("%06d.png" % i)), c)
            fa.write("%.6f rgb/%06d.png %.6f depth/%06d.png\n" % (t, i, t + 0.001, i))
            q = _rot_to_quat(T[:3, :3])
            fg.write("%.6f %.9f %.9f %.9f %.12f %.12f %.12f %.12f\n" % ((t + gt_offset,) + tuple(T[:3, 3]) + tuple(q)))
            fg.write("%.6f 9 9 9 0 0 0 1\n" % (t + 0.0165))  # decoy: farther from every frame
    with open(root / "calibration.txt", "w") as f:
        f.write("%.6f %.6f %.6f %.6f\n" % (K[0, 0], K[1, 1], K[0, 2], K[1, 2]))


def _rot_to_quat(R):
    """(qx, qy, qz, qw) of a rotation matrix (Shepperd's method)."""
    R = np.asarray(R, np.float64)
    tr = np.trace(R)
    if tr > 0:
        s = 2.0 * np.sqrt(tr + 1.0)
        w, x, y, z = 0.25 * s, (R[2, 1] - R[1, 2]) / s, (R[0, 2] - R[2, 0]) / s, (R[1, 0] - R[0, 1]) / s
    else:
        i = int(np.argmax(np.diag(R)))
        j, k = (i + 1) % 3, (i + 2) % 3
        s = 2.0 * np.sqrt(1.0 + R[i, i] - R[j, j] - R[k, k])
        q = np.zeros(3)
        q[i] = 0.25 * s
        q[j] = (R[j, i] + R[i, j]) / s
        q[k] = (R[k, i] + R[i, k]) / s
        w = (R[k, j] - R[j, k]) / s
        x, y, z = q
    return (x, y, z, w)
