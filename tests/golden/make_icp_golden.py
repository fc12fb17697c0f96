"""Generate tests/golden/ref_icp_normal_equations.npz from the REFERENCE's
own buildNLSKernel (include/solver/gnSolver/gnSolver.cu:26-196, compiled for
the CPU by oracle/ref_cpu/build_ref.sh into oracle/_ref/libdynref.so).

Two frames of a small seeded cube sequence: the target is frame 0's depth,
the source frame 1's with a 6-pixel invalid border (the reference does not
bound its projections, so every valid source pixel must land inside the
image); normals of both from the reference's rgbdImage.  For three source-
to-target transforms (identity, the true relative motion, a perturbed one)
the kernel runs at pyramid scale 1 on one host thread, so its float atomics
sum the per-pixel terms in pixel order; the 6x6 A and b are stored.  Then
gnSolver::init + solve (gnSolver.cu:12-21, 317-438) from the identity with
every level at scale 1, for three iteration / threshold settings (the last
one trips the max_increment guard); its Eigen calls are answered by the
oracle's own LDL^T and SE(3) exponential (oracle/gn_algebra.h through
oracle/ref_cpu/shim/eigen_stub.h), and the final increments are stored.
Last, the same three transforms with the kernel's photometric term on:
its hard-coded colour weight (gnSolver.cu:180) set to 0.1 through the one
substitution build_ref.sh makes, RGB from the sequence's procedural
texture; A and b are stored with both RGB images.

Usage (needs the reference tree, present only where the fixtures are made):
    bash oracle/ref_cpu/build_ref.sh && python tests/golden/make_icp_golden.py
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from dynamap_b200 import abi, scene  # noqa: E402

LIB = os.path.join(ROOT, "oracle", "_ref", "libdynref.so")
OUT = os.path.join(HERE, "ref_icp_normal_equations.npz")
BORDER = 6


def transforms(poses):
    rel = (np.linalg.inv(poses[0].astype(np.float64)) @ poses[1].astype(np.float64))
    c, s_ = np.cos(0.004), np.sin(0.004)
    bump = np.array([[c, -s_, 0, 0.002], [s_, c, 0, -0.001], [0, 0, 1, 0.003], [0, 0, 0, 1]])
    return [np.eye(4), rel, bump @ rel]


def main():
    L = C.CDLL(LIB)
    vp = C.c_void_p
    L.ref_normals.argtypes = [vp, C.POINTER(abi.Sensor), vp, vp]
    L.ref_icp_normal_equations.argtypes = [vp, vp, vp, vp, vp, vp, C.POINTER(abi.Sensor),
                                           C.POINTER(C.c_float), vp, vp]
    L.ref_gn_solve.argtypes = [vp, vp, vp, vp, C.POINTER(abi.Sensor), C.POINTER(C.c_int32),
                               C.c_float, C.c_float, C.c_float, vp, vp]
    L.ref_set_threads(1)
    L.ref_set_color_weight.argtypes = [C.c_float]
    sensor = abi.Sensor(rows=60, cols=80, fx=65.625, fy=65.625, cx=39.5, cy=29.5,
                        depth_scaler=1000.0)
    seq = scene.make_sequence(17, 2, sensor.rows, sensor.cols, sensor.fx, sensor.fy, sensor.cx,
                              sensor.cy, 0.004, 0.4, with_rgb=True, kind="cube")
    p = lambda a: a.ctypes.data_as(vp)
    depth = (seq.depth.astype(np.float32) / np.float32(sensor.depth_scaler)).astype(np.float32)
    tgt = np.ascontiguousarray(depth[0])
    src = np.ascontiguousarray(depth[1]).copy()
    src[:BORDER] = 0
    src[-BORDER:] = 0
    src[:, :BORDER] = 0
    src[:, -BORDER:] = 0
    nrm = []
    for d in (src, tgt):
        pts = np.zeros((sensor.rows, sensor.cols, 3), np.float32)
        n = np.zeros((sensor.rows, sensor.cols, 3), np.float32)
        L.ref_normals(p(d), C.byref(sensor), p(pts), p(n))
        nrm.append(n)
    Ts, As, bs = [], [], []
    for T in transforms(seq.poses):
        T = np.asarray(T, np.float32)
        A = np.zeros(36, np.float32)
        b = np.zeros(6, np.float32)
        L.ref_icp_normal_equations(p(src), p(nrm[0]), p(tgt), p(nrm[1]),
                                   p(np.ascontiguousarray(seq.rgb[1])),
                                   p(np.ascontiguousarray(seq.rgb[0])), C.byref(sensor),
                                   (C.c_float * 16)(*T.reshape(16).tolist()), p(A), p(b))
        Ts.append(T)
        As.append(A)
        bs.append(b)
    # the photometric term at weight 0.1 (the weight of the 640x480 RGB-D
    # configuration), same frames and transforms
    L.ref_set_color_weight(0.1)
    Acs, bcs = [], []
    for T in Ts:
        A = np.zeros(36, np.float32)
        b = np.zeros(6, np.float32)
        L.ref_icp_normal_equations(p(src), p(nrm[0]), p(tgt), p(nrm[1]),
                                   p(np.ascontiguousarray(seq.rgb[1])),
                                   p(np.ascontiguousarray(seq.rgb[0])), C.byref(sensor),
                                   (C.c_float * 16)(*T.reshape(16).tolist()), p(A), p(b))
        Acs.append(A)
        bcs.append(b)
    L.ref_set_color_weight(0.0)
    # whole solves: (iterations per level, min_increment, max_increment,
    # regularization)
    settings = [((5, 4, 3), 1e-3, 0.3, 0.02), ((10, 5, 4), 1e-5, 0.3, 0.02),
                ((3, 3, 3), 1e-3, 1e-9, 0.02)]
    incs, poses = [], []
    for iters, mi, ma, rg in settings:
        inc = np.zeros(6, np.float64)
        pose = np.zeros(16, np.float32)
        L.ref_gn_solve(p(src), p(tgt), None, None, C.byref(sensor), (C.c_int32 * 3)(*iters),
                       mi, ma, rg, p(inc), p(pose))
        incs.append(inc)
        poses.append(pose.reshape(4, 4))
    np.savez_compressed(
        OUT, src_depth=src, tgt_depth=tgt, src_normals=nrm[0], tgt_normals=nrm[1],
        sensor=np.array([sensor.rows, sensor.cols, sensor.fx, sensor.fy, sensor.cx, sensor.cy,
                         sensor.depth_scaler], np.float64),
        transforms=np.array(Ts), A=np.array(As), b=np.array(bs),
        src_rgb=np.ascontiguousarray(seq.rgb[1]), tgt_rgb=np.ascontiguousarray(seq.rgb[0]),
        color_weight=np.float32(0.1), A_color=np.array(Acs), b_color=np.array(bcs),
        solve_iters=np.array([s_[0] for s_ in settings], np.int32),
        solve_thresholds=np.array([s_[1:] for s_ in settings], np.float32),
        solve_inc=np.array(incs), solve_pose=np.array(poses))
    print(f"wrote {OUT}: {len(Ts)} transforms, A[1] diag {np.array(As)[1].reshape(6, 6).diagonal()}")


if __name__ == "__main__":
    main()
