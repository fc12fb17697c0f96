"""Known-answer tests of the CPU oracle's building blocks.

The reference ships no tests or golden vectors for this path, so each block
of the oracle is pinned here against an independent statement of the same
arithmetic: hand-derived values, a numpy float32 re-derivation, or (for the
parts the reference delegates to Eigen 3.3.7) an independent implementation
of the same published algorithm (scipy's matrix exponential, numpy's solve).
"""
import math

import numpy as np
import pytest

from dynamap_b200 import abi

f32 = np.float32


def py_hash(x, y, z, nb, bsz):
    """HashTable::Hash (hashTable.cu:152-163) with int32 wrap-around."""
    def mul(a, p):
        return ((a * p) & 0xFFFFFFFF)
    h = mul(x, 73856093) ^ mul(y, 19349669) ^ mul(z, 83492791)
    if h >= 1 << 31:
        h -= 1 << 32
    r = int(math.fmod(h, nb))  # C remainder: sign of the dividend
    if r < 0:
        r += nb
    return r * bsz


def test_hash_known_answers(oracle):
    L = oracle.lib()
    assert L.dyo_hash(0, 0, 0, 2500, 10) == 0
    assert L.dyo_hash(1, 0, 0, 2500, 10) == 10930        # 73856093 % 2500 = 1093
    assert L.dyo_hash(-1, 0, 0, 2500, 10) == 14070       # -1093 + 2500
    assert L.dyo_hash(100, 0, 0, 2500, 10) == 22080      # wraps: -1204325292 % 2500
    rng = np.random.default_rng(0)
    for _ in range(2000):
        x, y, z = (int(v) for v in rng.integers(-(1 << 20), 1 << 20, size=3))
        nb = int(rng.choice([2500, 1 << 18, 1 << 20, 12345]))
        assert L.dyo_hash(x, y, z, nb, 10) == py_hash(x, y, z, nb, 10)


def py_dda(start, point, trunc, bs):
    """numpy-float32 re-derivation of the DDA of AllocateFromDepthKernel
    (tsdf.cu:346-453): every operation rounded to float32 in source order."""
    s = [f32(v) for v in start]
    p = [f32(v) for v in point]
    v = [f32(p[i] - s[i]) for i in range(3)]
    dd = f32(f32(f32(v[0] * v[0]) + f32(v[1] * v[1])) + f32(v[2] * v[2]))
    inv = f32(f32(1) / f32(np.sqrt(dd)))
    d = [f32(v[i] * inv) for i in range(3)]
    w = [f32(s[i] - p[i]) for i in range(3)]
    sd = f32(np.sqrt(f32(f32(f32(w[0] * w[0]) + f32(w[1] * w[1])) + f32(w[2] * w[2]))))
    L = f32(sd + f32(trunc))
    e = [f32(s[i] + f32(d[i] * L)) for i in range(3)]
    bs = f32(bs)
    b = [int(np.floor(f32(s[i] / bs))) for i in range(3)]
    end = [int(np.floor(f32(e[i] / bs))) for i in range(3)]
    step = [int(np.sign(d[i])) for i in range(3)]
    FM = f32(3.402823466e38)
    dt = [f32(abs(f32(bs / d[i]))) if d[i] != 0 else FM for i in range(3)]
    mt = [f32(f32(f32(f32(b[i]) + f32(step[i])) * bs) - s[i]) for i in range(3)]
    mt = [f32(mt[i] / d[i]) if d[i] != 0 else FM for i in range(3)]
    out = [tuple(b)]
    diff = [0, 0, 0]
    neg = False
    for i in range(3):
        if b[i] != end[i] and d[i] < 0:
            diff[i] -= 1
            neg = True
    if neg:
        b = [b[i] + diff[i] for i in range(3)]
        out.append(tuple(b))
    for _ in range(100000):
        if b == end:
            break
        if mt[0] < mt[1]:
            k = 0 if mt[0] < mt[2] else 2
        else:
            k = 1 if mt[1] < mt[2] else 2
        b[k] += step[k]
        mt[k] = f32(mt[k] + dt[k])
        out.append(tuple(b))
    return out


def test_dda_axis_rays(oracle):
    # +x ray: blocks 0..16 along x (end = floor((1.0 + 0.032)/0.064 + ...))
    blocks, ok = oracle.dda_blocks((0.01, 0.01, 0.01), (1.0, 0.01, 0.01), 0.032, 0.064)
    assert ok
    assert [tuple(b) for b in blocks] == [(x, 0, 0) for x in range(17)]
    # -x ray exercises the 'diff' pre-step (tsdf.cu:409-429): 0, -1, ..., -9
    blocks, ok = oracle.dda_blocks((0.01, 0.01, 0.01), (-0.5, 0.01, 0.01), 0.032, 0.064)
    assert ok
    assert [tuple(b) for b in blocks] == [(x, 0, 0) for x in range(0, -10, -1)]


def test_dda_matches_float32_rederivation(oracle):
    rng = np.random.default_rng(1)
    for _ in range(400):
        start = rng.uniform(-2, 4, size=3)
        point = start + rng.normal(size=3) * rng.uniform(0.05, 3.0)
        bs = float(rng.choice([0.064, 0.04, 0.032, 0.08]))
        blocks, ok = oracle.dda_blocks(start, point, 0.032, bs)
        assert ok
        ref = py_dda(start, point, 0.032, bs)
        assert [tuple(b) for b in blocks] == ref


def test_dda_step_cap_counts_overrun(oracle):
    blocks, ok = oracle.dda_blocks((0.01, 0.02, 0.03), (3.0, 2.0, 1.0), 0.032, 0.064, cap=5)
    assert not ok


def test_merge_voxel_known_answers(oracle):
    # first merge takes the new value (w 0 -> 1)
    rgbw, sdf = oracle.merge_voxel([0, 0, 0, 0], 0.0, 0.02, [10, 20, 30], 1, 64)
    assert rgbw == [10, 20, 30, 1] and np.float32(sdf) == np.float32(0.02)
    # colour average truncates: (100*1 + 201*1)/2 = 150.5 -> 150
    rgbw, sdf = oracle.merge_voxel([100, 100, 100, 1], 0.0, 0.0, [201, 201, 201], 1, 64)
    assert rgbw[:3] == [150, 150, 150] and rgbw[3] == 2
    # weight saturates at max_sdf_weight
    rgbw, sdf = [0, 0, 0, 0], 0.0
    for _ in range(70):
        rgbw, sdf = oracle.merge_voxel(rgbw, sdf, 0.01, [0, 0, 0], 1, 64)
    assert rgbw[3] == 64
    assert sdf == pytest.approx(0.01, rel=1e-6)
    # float32 running average, as geom_Types.h:93-97 rounds it
    w, s = 5, f32(0.013)
    rgbw, sdf = oracle.merge_voxel([0, 0, 0, w], float(s), -0.007, [0, 0, 0], 1, 64)
    expect = f32(f32(f32(s * f32(w)) + f32(f32(-0.007) * f32(1))) / f32(f32(w) + f32(1)))
    assert np.float32(sdf) == expect


def test_inverse4_cofactor(oracle):
    rng = np.random.default_rng(2)
    for _ in range(50):
        xi = rng.normal(size=6) * [0.5, 0.5, 0.5, 2, 2, 2]
        T = oracle.se3_exp(xi).astype(np.float32)
        inv = oracle.inverse4(T)
        np.testing.assert_allclose(inv, np.linalg.inv(T.astype(np.float64)), atol=2e-6)


def test_se3_exp_matches_matrix_exponential(oracle):
    """Eigen's MatrixBase::exp (gnSolver.cu:443-445) is the matrix
    exponential of v2t(xi) (gnSolver.cu:446-455); scipy.linalg.expm
    computes the same function (Pade + scaling and squaring)."""
    from scipy.linalg import expm
    rng = np.random.default_rng(3)
    for scale in (1e-7, 1e-5, 1e-3, 0.05, 0.5, 2.0):
        for _ in range(20):
            xi = rng.normal(size=6) * scale
            M = np.array([[0, -xi[2], xi[1], xi[3]],
                          [xi[2], 0, -xi[0], xi[4]],
                          [-xi[1], xi[0], 0, xi[5]],
                          [0, 0, 0, 0]])
            np.testing.assert_allclose(oracle.se3_exp(xi), expm(M), atol=1e-13, rtol=1e-12)


def test_ldlt_matches_dense_solve(oracle):
    import ctypes as C
    rng = np.random.default_rng(4)
    L = oracle.lib()
    for _ in range(50):
        J = rng.normal(size=(40, 6))
        A = J.T @ J + 0.02 * np.eye(6)
        b = rng.normal(size=6)
        x = np.zeros(6)
        ok = L.dyo_ldlt_solve6(A.ctypes.data_as(C.POINTER(C.c_double)),
                               b.ctypes.data_as(C.POINTER(C.c_double)),
                               x.ctypes.data_as(C.POINTER(C.c_double)))
        assert ok
        np.testing.assert_allclose(x, np.linalg.solve(A, b), rtol=1e-10, atol=1e-12)


def test_level_sensor(oracle):
    s = abi.Sensor(rows=480, cols=640, fx=525.0, fy=525.0, cx=319.5, cy=239.5,
                   depth_scaler=1000.0)
    l2 = oracle.level_sensor(s, 4)
    assert (l2.rows, l2.cols) == (120, 160)
    assert l2.fx == pytest.approx(131.25)
    # pixel centres map: (c + 0.5)/s - 0.5
    assert l2.cx == pytest.approx((319.5 + 0.5) / 4 - 0.5)


def test_maps_normals_plane(oracle):
    """Fronto-parallel plane: normals (0, 0, 1) in the interior (cross of
    right-left and down-up, rgbdImage.cu:142-144), 0 at the borders and
    holes."""
    s = abi.Sensor(rows=24, cols=32, fx=30.0, fy=30.0, cx=15.5, cy=11.5, depth_scaler=1000.0)
    d = np.full((24, 32), 1.5, np.float32)
    d[10, 10] = 0.0
    v, n = oracle.maps(d, s)
    assert np.allclose(n[5, 5, :3], [0, 0, 1], atol=1e-6)
    assert np.all(n[0, :, :3] == 0) and np.all(n[:, 0, :3] == 0) and np.all(n[:, 1, :3] == 0)
    assert np.all(n[10, 10] == 0) and np.all(n[10, 8] == 0) and np.all(n[9, 10] == 0)
    assert v[10, 10, 3] == 0 and v[5, 5, 3] == 1


def test_bilateral_constant_and_holes(oracle):
    p = abi.BilateralParams(diameter=8, sigma_i=10.0, sigma_s=1.0, enabled=1)
    d = np.full((40, 50), 2.0, np.float32)
    d[20, 20] = 0.0
    out = oracle.bilateral(d, p)
    assert out[20, 20] == 0.0
    assert np.allclose(out[d > 0], 2.0, rtol=1e-6)


def test_downsample_valid_mean(oracle):
    d = np.array([[1.0, 3.0, 0.0, 0.0], [0.0, 2.0, 0.0, 0.0]], np.float32)
    out = oracle.downsample_depth(d)
    assert out.shape == (1, 2)
    assert out[0, 0] == pytest.approx(2.0) and out[0, 1] == 0.0
