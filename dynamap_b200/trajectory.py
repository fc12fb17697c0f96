"""Trajectories in the TUM RGB-D format, and their error.

The reference logs each tracked pose with builder::writePoseToTxt
(include/builder/builder.cu:243-257) -- one line "stamp tx ty tz qx qy qz qw"
in fixed notation with 4 decimals, the quaternion of the pose's rotation --
and reads ground truth with builder::v2tRef (builder.cu:222-241) /
dataSet::getCurrentPose (include/utils/utils_Dataset.cpp:69-88): the
quaternion normalised, turned into a rotation in double, rounded to float.
The conversions are the published methods behind those Eigen calls, in the
same double-precision operation order as include/dynamap/pose_io.h (so the
C++ and Python writers print the same text):

* rotation -> quaternion: Shoemake (SIGGRAPH 1985), from the trace when it
  is positive, else from the largest diagonal element;
* quaternion -> rotation: the homogeneous form of a unit quaternion.

ate() is the absolute trajectory error of the TUM benchmark tools: the RMSE
of the translation differences after the rigid alignment of one trajectory
onto the other that minimises it (Horn 1987 / Umeyama 1991, no scale), or
without alignment when both start from the same known pose.
"""
from __future__ import annotations

import math
from typing import Iterable, Sequence

import numpy as np


def quat_from_rotation(m) -> tuple[float, float, float, float]:
    """(x, y, z, w) of the 3x3 rotation m (read in double)."""
    m = [[float(m[r][c]) for c in range(3)] for r in range(3)]
    t = m[0][0] + m[1][1] + m[2][2]
    if t > 0.0:
        s = math.sqrt(t + 1.0)
        w = 0.5 * s
        s = 0.5 / s
        return ((m[2][1] - m[1][2]) * s, (m[0][2] - m[2][0]) * s, (m[1][0] - m[0][1]) * s, w)
    i = 0
    if m[1][1] > m[0][0]:
        i = 1
    if m[2][2] > m[i][i]:
        i = 2
    j = (i + 1) % 3
    k = (j + 1) % 3
    v = [0.0, 0.0, 0.0]
    s = math.sqrt(m[i][i] - m[j][j] - m[k][k] + 1.0)
    v[i] = 0.5 * s
    s = 0.5 / s
    w = (m[k][j] - m[j][k]) * s
    v[j] = (m[j][i] + m[i][j]) * s
    v[k] = (m[k][i] + m[i][k]) * s
    return (v[0], v[1], v[2], w)


def rotation_from_quat(x: float, y: float, z: float, w: float) -> np.ndarray:
    """3x3 float64 rotation of the quaternion (x, y, z, w), normalised first."""
    n = math.sqrt(x * x + y * y + z * z + w * w)
    x, y, z, w = x / n, y / n, z / n, w / n
    tx, ty, tz = 2.0 * x, 2.0 * y, 2.0 * z
    twx, twy, twz = tx * w, ty * w, tz * w
    txx, txy, txz = tx * x, ty * x, tz * x
    tyy, tyz, tzz = ty * y, tz * y, tz * z
    return np.array([[1.0 - (tyy + tzz), txy - twz, txz + twy],
                     [txy + twz, 1.0 - (txx + tzz), tyz - twx],
                     [txz - twy, tyz + twx, 1.0 - (txx + tyy)]], dtype=np.float64)


def pose_from_tum(v: Sequence[float]) -> np.ndarray:
    """A TUM line's values {stamp, tx, ty, tz, qx, qy, qz, qw} -> float32 4x4
    camera-to-world pose (v2tRef)."""
    if len(v) < 8:
        raise ValueError("a TUM pose line has 8 values")
    p = np.eye(4, dtype=np.float32)
    p[:3, :3] = rotation_from_quat(float(v[4]), float(v[5]), float(v[6]), float(v[7]))
    p[:3, 3] = [float(v[1]), float(v[2]), float(v[3])]
    return p


def tum_line(stamp: float, pose) -> str:
    """The line writePoseToTxt writes for a 4x4 pose (its float32 values)."""
    p = np.asarray(pose, dtype=np.float32)
    q = quat_from_rotation(p[:3, :3].astype(np.float64))
    vals = (float(stamp), float(p[0, 3]), float(p[1, 3]), float(p[2, 3])) + q
    return " ".join("%.4f" % x for x in vals)


def write_tum(path: str, stamps: Iterable[float], poses: Iterable, append: bool = True) -> None:
    """Append (the reference opens its log for appending) or write one line
    per pose."""
    with open(path, "a" if append else "w") as f:
        for t, p in zip(stamps, poses):
            f.write(tum_line(t, p) + "\n")


def read_tum(path: str) -> tuple[np.ndarray, np.ndarray]:
    """(stamps float64 [n], poses float32 [n, 4, 4]) of a TUM trajectory file;
    '#' lines and blank lines are skipped, commas count as separators."""
    stamps, poses = [], []
    with open(path) as f:
        for ln in f:
            ln = ln.strip()
            if not ln or ln.startswith("#"):
                continue
            v = [float(x) for x in ln.replace(",", " ").split()]
            stamps.append(v[0])
            poses.append(pose_from_tum(v))
    return (np.asarray(stamps, dtype=np.float64),
            np.asarray(poses, dtype=np.float32).reshape(-1, 4, 4))


def associate(stamps_a: Sequence[float], stamps_b: Sequence[float],
              max_difference: float = 0.02) -> list[tuple[int, int]]:
    """Pairs (i, j) of stamps within max_difference of each other, closest
    first, each stamp used at most once; sorted by i."""
    a = np.asarray(stamps_a, dtype=np.float64)
    b = np.asarray(stamps_b, dtype=np.float64)
    order = np.argsort(b, kind="stable")
    bs = b[order]
    lo = np.searchsorted(bs, a - max_difference, side="left")
    hi = np.searchsorted(bs, a + max_difference, side="right")
    cand = sorted((abs(a[i] - bs[k]), i, int(order[k])) for i in range(len(a))
                  for k in range(lo[i], hi[i]) if abs(a[i] - bs[k]) < max_difference)
    used_a, used_b, out = set(), set(), []
    for _, i, j in cand:
        if i not in used_a and j not in used_b:
            used_a.add(i)
            used_b.add(j)
            out.append((i, j))
    return sorted(out)


def align(src: np.ndarray, dst: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Rotation R and translation t minimising sum |R src_i + t - dst_i|^2
    (points as rows, float64)."""
    src = np.asarray(src, dtype=np.float64)
    dst = np.asarray(dst, dtype=np.float64)
    ms, md = src.mean(axis=0), dst.mean(axis=0)
    h = (src - ms).T @ (dst - md)
    u, _, vt = np.linalg.svd(h)
    d = np.eye(3)
    d[2, 2] = np.sign(np.linalg.det(vt.T @ u.T)) or 1.0
    r = vt.T @ d @ u.T
    return r, md - r @ ms


def ate(est, gt, aligned: bool = True) -> dict:
    """Absolute trajectory error of estimated poses against ground truth
    (same length, matched by index): RMSE, mean, median and max of the
    translation differences in metres, after the best rigid alignment of
    the estimate when 'aligned'."""
    pe = np.asarray(est, dtype=np.float64)[:, :3, 3]
    pg = np.asarray(gt, dtype=np.float64)[:, :3, 3]
    if pe.shape != pg.shape or len(pe) == 0:
        raise ValueError("trajectories must have the same, non-zero length")
    if aligned and len(pe) >= 3:
        r, t = align(pe, pg)
        pe = pe @ r.T + t
    e = np.linalg.norm(pe - pg, axis=1)
    return {"rmse": float(np.sqrt(np.mean(e * e))), "mean": float(e.mean()),
            "median": float(np.median(e)), "max": float(e.max()), "n": int(len(e))}
