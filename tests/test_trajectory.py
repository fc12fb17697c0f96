"""TUM-format trajectory logs (builder::writePoseToTxt / v2tRef,
include/builder/builder.cu:222-257) and the absolute trajectory error:
known answers, the C++ drop-in and the Python module writing the same text,
round trips, association and alignment."""
import math
import os
import shutil
import subprocess

import numpy as np
import pytest

from dynamap_b200 import trajectory as tj

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rot(axis, ang):
    a = np.asarray(axis, dtype=np.float64)
    a = a / np.linalg.norm(a)
    k = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + math.sin(ang) * k + (1 - math.cos(ang)) * (k @ k)


def pose(r, t):
    p = np.eye(4, dtype=np.float32)
    p[:3, :3] = r
    p[:3, 3] = t
    return p


def random_poses(n, seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        if i % 5 == 0:   # rotations near 180 degrees: the negative-trace branch
            ang = math.pi - rng.uniform(0.0, 0.3)
        else:
            ang = rng.uniform(0.0, math.pi)
        out.append(pose(rot(rng.normal(size=3), ang), rng.uniform(-4, 4, size=3)))
    return out


def test_known_lines():
    assert tj.tum_line(1305031102.175304, np.eye(4)) == \
        "1305031102.1753 0.0000 0.0000 0.0000 0.0000 0.0000 0.0000 1.0000"
    rz = pose([[0, -1, 0], [1, 0, 0], [0, 0, 1]], [1.0, -2.5, 0.25])
    assert tj.tum_line(0.5, rz) == "0.5000 1.0000 -2.5000 0.2500 0.0000 0.0000 0.7071 0.7071"
    rx = pose(np.diag([1.0, -1.0, -1.0]), [0, 0, 0])   # trace -1: largest-diagonal branch
    assert tj.tum_line(2, rx) == "2.0000 0.0000 0.0000 0.0000 1.0000 0.0000 0.0000 0.0000"
    ry = pose(np.diag([-1.0, 1.0, -1.0]), [0, 0, 0])
    assert tj.tum_line(2, ry).endswith(" 0.0000 1.0000 0.0000 0.0000")


def test_quaternion_round_trip():
    for p in random_poses(200):
        r = p[:3, :3].astype(np.float64)
        q = tj.quat_from_rotation(r)
        assert abs(math.sqrt(sum(c * c for c in q)) - 1.0) < 1e-6
        np.testing.assert_allclose(tj.rotation_from_quat(*q), r, atol=2e-6)
        # q and -q are the same rotation
        np.testing.assert_allclose(tj.rotation_from_quat(*[-c for c in q]), r, atol=2e-6)


def test_write_read_round_trip(tmp_path):
    poses = random_poses(50)
    stamps = 1000.0 + 0.033 * np.arange(50)
    path = tmp_path / "traj.txt"
    path.write_text("# timestamp tx ty tz qx qy qz qw\n\n")
    tj.write_tum(str(path), stamps, poses)
    st, got = tj.read_tum(str(path))
    np.testing.assert_allclose(st, np.round(stamps, 4), atol=1e-9)
    for a, b in zip(got, poses):
        np.testing.assert_allclose(a[:3, 3], b[:3, 3], atol=5.1e-5)   # 4 decimals
        np.testing.assert_allclose(a[:3, :3], b[:3, :3], atol=4e-4)
        assert a.dtype == np.float32 and np.all(a[3] == [0, 0, 0, 1])


def test_cpp_dropin_writes_the_same_text(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path / "pose_io")
    libdir = os.path.join(ROOT, "dynamap_b200")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "pose_io_example.cpp"), "-L", libdir,
                    "-ldynamap_b200", f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    poses = random_poses(120, seed=9)
    stamps = 1305031102.0 + 0.0333 * np.arange(len(poses))
    inp = "".join("%.6f " % t + " ".join("%.9g" % x for x in p.reshape(-1)) + "\n"
                  for t, p in zip(stamps, poses))
    log = tmp_path / "log.txt"
    r = subprocess.run([exe, str(log)], input=inp, capture_output=True, text=True, check=True)
    want = [tj.tum_line(t, p) for t, p in zip(stamps, poses)]
    assert log.read_text().splitlines() == want
    # v2tRef of each written line, C++ against Python, bit for bit
    rows = [np.array([float(x) for x in ln.split()], dtype=np.float32).reshape(4, 4)
            for ln in r.stdout.splitlines()]
    assert len(rows) == len(want)
    for ln, got in zip(want, rows):
        ref = tj.pose_from_tum([float(x) for x in ln.split()])
        np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_associate():
    a = [0.00, 0.033, 0.066, 0.100, 0.5]
    b = [0.001, 0.030, 0.068, 0.140, 0.101]
    assert tj.associate(a, b, 0.02) == [(0, 0), (1, 1), (2, 2), (3, 4)]
    assert tj.associate(a, [], 0.02) == []


def test_ate():
    gt = random_poses(40, seed=3)
    # a rigid motion of the whole trajectory: zero after alignment
    g = pose(rot([0.2, 1.0, -0.3], 0.7), [0.5, -1.0, 2.0]).astype(np.float64)
    est = [g @ p.astype(np.float64) for p in gt]
    e = tj.ate(est, gt)
    assert e["rmse"] < 1e-5 and e["n"] == 40
    assert tj.ate(est, gt, aligned=False)["rmse"] > 0.1
    # a constant offset of 1 cm: 1 cm unaligned, 0 aligned
    off = [p.copy() for p in gt]
    for p in off:
        p[:3, 3] += np.float32([0.01, 0.0, 0.0])
    assert tj.ate(off, gt, aligned=False)["rmse"] == pytest.approx(0.01, abs=1e-6)
    assert tj.ate(off, gt)["rmse"] < 1e-5
    with pytest.raises(ValueError):
        tj.ate(gt[:3], gt[:4])
