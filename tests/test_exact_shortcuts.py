"""The exact shortcuts the FP32 kernels take, checked against the reference's
FP32 expressions with numpy (IEEE single precision, round to nearest):

* colour merge (csrc/tsdf.cu colour_merge): the byte of
  (old * w + obs) / (w + 1) computed in FP32 and truncated, as
  Voxel::mergeVoxelColor does (geom_Types.h:87-91), equals the integer
  quotient obtained from a reciprocal estimate corrected by one step, for
  every weight and byte pair and reciprocals a few ulps off;
* corner indices (csrc/common.cuh voxel_index_pair): where the fast path
  of the lower corner's index applies, the upper corner's index
  (WorldToGlobalVoxelHashing of pos_dual + vs, tsdf.cu:189-193) is the
  lower one plus one;
* pixel coordinates (csrc/icp.cu pixel_uv): the row and column of a pixel
  index from a reciprocal estimate corrected by one step equal the integer
  division's.

The GPU tests show the kernels bit-exact against the oracle on whole
frames; these check the arithmetic argument itself on every (or many)
inputs."""
import numpy as np

f = np.float32


def test_colour_merge_integer_quotient_equals_the_fp32_expression():
    w = np.arange(0, 256, dtype=np.int64)
    v = np.arange(0, 256, dtype=np.int64)
    W, R, C = (a.ravel() for a in np.meshgrid(w, v, v, indexing="ij"))
    fw = W.astype(np.float32)
    num = (R.astype(np.float32) * fw + C.astype(np.float32) * f(1.0)).astype(np.float32)
    ref = np.trunc((num / (fw + f(1.0))).astype(np.float32)).astype(np.int64)
    n, d = R * W + C, W + 1
    for k in range(-4, 5):  # the reciprocal estimate, up to 4 ulps off
        rc = (f(1.0) / d.astype(np.float32)).astype(np.float32)
        rc = (rc.astype(np.float64) * (1.0 + k * 2.0 ** -23)).astype(np.float32)
        q = np.trunc((n.astype(np.float32) * rc).astype(np.float32)).astype(np.int64)
        r = n - q * d
        q = q + (r >= d) - (r < 0)
        assert np.array_equal(q, ref), k


def _ref_index(p, vs):
    """(int)(p / vs + sign(p) * 0.5) in FP32, truncated toward zero."""
    s = ((p / vs).astype(np.float32) + np.sign(p).astype(np.float32) * f(0.5)).astype(np.float32)
    return np.trunc(s).astype(np.int64)


def test_upper_corner_index_follows_from_the_lower_one():
    rng = np.random.default_rng(3)
    used = 0
    for vs in (f(0.004), f(0.005), f(0.008), f(0.0123)):
        inv = (f(1.0) / vs).astype(np.float32)
        k = rng.integers(-1500, 1500, 1_000_000)
        near = ((k * 0.5) * float(vs) + rng.normal(0, 1e-6, k.size) * float(vs)).astype(np.float32)
        for pd in (rng.uniform(-6, 6, 1_000_000).astype(np.float32), near, -near):
            p0 = (pd + f(0.0)).astype(np.float32)
            p1 = (pd + vs).astype(np.float32)
            t = ((p0 * inv).astype(np.float32) + np.copysign(f(0.5), p0)).astype(np.float32)
            margin = (np.abs(t).astype(np.float64) * 1.9073486328125e-6
                      + 1.9073486328125e-6).astype(np.float32)
            fast = (np.abs((t - np.rint(t)).astype(np.float32)) > margin) & \
                ((p0 > 0) | ((p1 < 0) & (t < -1)))
            g0 = np.trunc(t).astype(np.int64)
            assert np.array_equal(g0[fast], _ref_index(p0, vs)[fast])
            assert np.array_equal(g0[fast] + 1, _ref_index(p1, vs)[fast])
            used += int(fast.sum())
    assert used > 5_000_000


def test_pixel_coordinates_from_a_reciprocal_estimate():
    """pixel_uv (csrc/icp.cu): the row of pixel index idx as the truncated
    product of idx and an approximate reciprocal of the column count, then
    one correction step, equals idx / cols and idx % cols for images of up
    to 8192 x 8192 pixels and reciprocals a few ulps off."""
    rng = np.random.default_rng(5)
    for rows, cols in ((120, 160), (240, 320), (480, 640), (720, 1280), (60, 80), (30, 40),
                       (8192, 8192), (8192, 7), (3, 8191)):
        n = rows * cols
        idx = np.arange(n, dtype=np.int64) if n <= 2_000_000 else \
            np.concatenate([rng.integers(0, n, 2_000_000), np.arange(n - 100_000, n)])
        for k in (-4, -1, 0, 1, 4):
            rc = (f(1.0) / f(cols)).astype(np.float32)
            rc = f(float(rc) * (1.0 + k * 2.0 ** -23))
            v = np.trunc((idx.astype(np.float32) * rc).astype(np.float32)).astype(np.int64)
            u = idx - v * cols
            v = np.where(u < 0, v - 1, np.where(u >= cols, v + 1, v))
            u = idx - v * cols
            assert np.array_equal(v, idx // cols) and np.array_equal(u, idx % cols), (rows, cols, k)
