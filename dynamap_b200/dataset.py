"""RGB-D sequences in the TUM layout, read into the frames a session takes.

Mirrors DynaMap::utils::dataSet (include/utils/utils_Dataset.h:38-85,
utils_Dataset.cpp): a directory with rgb/ and depth/ images named by their
time stamps, an optional association file and an optional groundtruth.txt.
Frames come out as the session's inputs: the sensor's raw uint16 depth
(the session divides by depth_scaler, 5000 for TUM) and uint8 RGB.

Differences from the reference, each a fix:
* depth is read as 16-bit (the reference reads it with cv::IMREAD_COLOR,
  utils_Dataset.cpp:233-235, which keeps 8 bits of three channels);
* RGB is returned in RGB order (OpenCV reads BGR);
* an association file is read by its paths, so both column orders work
  (the reference takes word 0 as the depth name and word 2 as the RGB name,
  getAssociateContent :174-175);
* ground truth is matched to each frame by time stamp (the reference takes
  line curID + offsetLineGroundTruth, :210-221).

Images are decoded with OpenCV when it is importable, else with Pillow.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from typing import Iterator, Optional

import numpy as np

from . import trajectory


def _imread(path: str, depth: bool) -> np.ndarray:
    try:
        import cv2
    except ImportError:
        cv2 = None
    if cv2 is not None:
        img = cv2.imread(path, cv2.IMREAD_UNCHANGED)
        if img is None:
            raise IOError(f"cannot read {path}")
        if not depth and img.ndim == 3:
            img = img[:, :, 2::-1]  # BGR(A) -> RGB
    else:
        from PIL import Image
        with Image.open(path) as im:
            img = np.asarray(im if depth else im.convert("RGB"))
    if depth:
        if img.ndim != 2 or img.dtype != np.uint16:
            raise ValueError(f"{path}: depth must be a 16-bit single-channel image")
    elif img.ndim == 2:
        img = np.repeat(img[:, :, None], 3, axis=2)
    return np.ascontiguousarray(img)


def _stamp(name: str, prefix: str = "", suffix: str = ".png") -> float:
    """The number in a file name between prefix and suffix."""
    b = os.path.basename(name)
    if prefix and b.startswith(prefix):
        b = b[len(prefix):]
    if suffix and b.endswith(suffix):
        b = b[:-len(suffix)]
    return float(b)


@dataclass
class Frame:
    index: int
    stamp: float                 # depth time stamp
    depth: np.ndarray            # uint16 [rows, cols], sensor units
    rgb: Optional[np.ndarray]    # uint8 [rows, cols, 3] RGB, or None
    gt_pose: Optional[np.ndarray]  # float32 4x4 camera-to-world, or None


class TumDataset:
    """dataSet(mainDir): the frames of a TUM-layout directory in time order.

    first/last/skip select frames like the reference's firstFrameID /
    lastFrameID / skipFrameNum; gt_max_difference bounds the time difference
    of a matched ground-truth pose (seconds).  Without an association file,
    the folders list files named prefix + number + suffix (the reference's
    depthPrefix / rgbPrefix / suffixes; TUM: no prefix, ".png"), ordered by
    the number."""

    def __init__(self, main_dir: str, association: str = "association.txt",
                 groundtruth: str = "groundtruth.txt", first: int = 0,
                 last: Optional[int] = None, skip: int = 1, gt_max_difference: float = 0.02,
                 depth_prefix: str = "", rgb_prefix: str = "", suffix: str = ".png"):
        self.main_dir = main_dir
        self.depth_prefix, self.rgb_prefix, self.suffix = depth_prefix, rgb_prefix, suffix
        self.pairs = self._pairs(association)
        self.pairs = self.pairs[first:last:max(1, skip)]
        self.gt_stamps = None
        self.gt_poses = None
        gpath = os.path.join(main_dir, groundtruth)
        if os.path.exists(gpath):
            self.gt_stamps, self.gt_poses = trajectory.read_tum(gpath)
        self._gt_index = {}
        if self.gt_stamps is not None and len(self.gt_stamps):
            depth_stamps = [_stamp(d, self.depth_prefix, self.suffix) for d, _ in self.pairs]
            for i, j in trajectory.associate(depth_stamps, self.gt_stamps, gt_max_difference):
                self._gt_index[i] = j

    # (depth path, rgb path or None) per frame, in time order
    def _pairs(self, association: str):
        apath = os.path.join(self.main_dir, association)
        if os.path.exists(apath):
            out = []
            with open(apath) as f:
                for ln in f:
                    w = ln.split()
                    if not w or ln.lstrip().startswith("#"):
                        continue
                    if len(w) < 4:
                        raise ValueError(f"{apath}: expected 'stamp path stamp path' lines")
                    a, b = w[1], w[3]
                    depth, rgb = (a, b) if a.startswith("depth") else (b, a)
                    out.append((os.path.join(self.main_dir, depth),
                                os.path.join(self.main_dir, rgb)))
            return sorted(out, key=lambda p: _stamp(p[0], self.depth_prefix, self.suffix))
        dd = os.path.join(self.main_dir, "depth")
        if not os.path.isdir(dd):
            raise FileNotFoundError(f"{dd}: no depth folder and no {association}")
        def listed(folder, prefix):
            names = [n for n in os.listdir(folder)
                     if n.startswith(prefix) and n.endswith(self.suffix)
                     and len(n) > len(prefix) + len(self.suffix)]
            return sorted(names, key=lambda n: _stamp(n, prefix, self.suffix))
        depth = listed(dd, self.depth_prefix)
        rd = os.path.join(self.main_dir, "rgb")
        rgb = listed(rd, self.rgb_prefix) if os.path.isdir(rd) else []
        # the reference pairs the sorted lists by index
        return [(os.path.join(dd, d), os.path.join(rd, rgb[i]) if i < len(rgb) else None)
                for i, d in enumerate(depth)]

    def __len__(self) -> int:
        return len(self.pairs)

    def __getitem__(self, i: int) -> Frame:
        dpath, rpath = self.pairs[i]
        j = self._gt_index.get(i)
        return Frame(index=i, stamp=_stamp(dpath, self.depth_prefix, self.suffix),
                     depth=_imread(dpath, True),
                     rgb=_imread(rpath, False) if rpath else None,
                     gt_pose=self.gt_poses[j].copy() if j is not None else None)

    def __iter__(self) -> Iterator[Frame]:
        for i in range(len(self)):
            yield self[i]


def run_session(session, frames, log_path: Optional[str] = None, use_rgb: bool = True):
    """Track and map every frame with a Session (dynamap_b200.session):
    the first frame's ground-truth pose, when there is one, starts the
    trajectory; each tracked pose is appended to log_path in the TUM format
    when given.  Returns (stamps, poses)."""
    stamps, poses = [], []
    for k, fr in enumerate(frames):
        if k == 0 and fr.gt_pose is not None:
            session.set_pose(fr.gt_pose)
        pose, _ = session.process(fr.depth, fr.rgb if use_rgb else None, strict=False)
        stamps.append(fr.stamp)
        poses.append(pose)
        if log_path:
            trajectory.write_tum(log_path, [fr.stamp], [pose])
    return np.asarray(stamps), np.asarray(poses, dtype=np.float32)
