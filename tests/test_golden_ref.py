"""The oracle reproduces the reference's own outputs (golden vectors made
by tests/golden/make_golden.py and make_icp_golden.py from the reference
sources compiled for the CPU): allocation, integration, raycast,
vertex/normal maps, the hash, the ICP normal equations of buildNLSKernel,
gnSolver::solve's increments and the vertices of MeshExtractor's mesh bit
for bit; the bilateral filter within 2 ulp-scale relative error (the
oracle's range weight uses a portable FP32 exp, the reference libm's FP64
exp)."""
import os

import numpy as np
import pytest

from dynamap_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "ref_rigid_small.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def structs(g):
    s = g["sensor"]
    t = g["tsdf"]
    sensor = abi.Sensor(rows=int(s[0]), cols=int(s[1]), fx=s[2], fy=s[3], cx=s[4], cy=s[5],
                        depth_scaler=s[6])
    tsdf = abi.TsdfParams(voxel_size=t[0], num_buckets=int(t[1]), bucket_size=int(t[2]),
                          num_blocks=int(t[3]), block_size=int(t[4]), max_sdf_weight=int(t[5]),
                          truncation_distance=t[6], max_sensor_depth=t[7], min_sensor_depth=t[8])
    return sensor, tsdf


def block_crc(rgbw, sdf):
    import zlib
    return zlib.crc32(np.ascontiguousarray(sdf, "<f4").tobytes(),
                      zlib.crc32(np.ascontiguousarray(rgbw, np.uint8).tobytes()))


@pytest.fixture(scope="module")
def oracle_volume(gold, oracle):
    sensor, tsdf = structs(gold)
    vol = oracle.Volume(tsdf)
    for k in range(3):
        d = oracle.depth_from_raw(gold["depth"][k], sensor.depth_scaler)
        c1 = vol.allocate(d, sensor, gold["poses"][k])
        c2 = vol.integrate(d, gold["rgb"][k], sensor, gold["poses"][k])
        assert c1[oracle.C_BUCKET_FULL] == 0 and c1[oracle.C_DDA] == 0
        assert c2[oracle.C_REHASH] == 0
    return vol, sensor


def test_reference_block_set_and_voxels(gold, oracle_volume):
    vol, _ = oracle_volume
    coords, rgbw, sdf = vol.download()
    order = np.lexsort((coords[:, 2], coords[:, 1], coords[:, 0]))
    coords, rgbw, sdf = coords[order], rgbw[order], sdf[order]
    np.testing.assert_array_equal(coords, gold["block_coords"])
    sub = gold["subset"]
    np.testing.assert_array_equal(rgbw[sub], gold["subset_rgbw"])
    np.testing.assert_array_equal(sdf[sub].view(np.uint32), gold["subset_sdf"].view(np.uint32))
    crc = np.array([block_crc(rgbw[i], sdf[i]) for i in range(len(coords))], np.uint32)
    np.testing.assert_array_equal(crc, gold["block_crc"])


def test_reference_raycast(gold, oracle_volume):
    vol, sensor = oracle_volume
    for name, pose, s in (("ray_pose2", gold["poses"][2], sensor),
                          ("ray_pose0", gold["poses"][0], sensor),
                          ("ray_half", gold["poses"][1],
                           abi.Sensor(rows=30, cols=40, fx=32.8125, fy=32.8125, cx=19.75,
                                      cy=14.75, depth_scaler=1000.0))):
        d, c, _ = vol.raycast(pose, s, rgb=True)
        np.testing.assert_array_equal(d.view(np.uint32), gold[name + "_depth"].view(np.uint32))
        np.testing.assert_array_equal(c, gold[name + "_rgb"])


def test_reference_normals(gold, oracle):
    sensor, _ = structs(gold)
    d = oracle.depth_from_raw(gold["depth"][0], sensor.depth_scaler)
    v, n = oracle.maps(d, sensor)
    valid = d > 0
    np.testing.assert_array_equal(v[valid][:, :3].view(np.uint32),
                                  gold["normals_points"][valid].view(np.uint32))
    # normals agree wherever the oracle has one (centre and all four
    # neighbours valid, inside the row); elsewhere the reference reads
    # wrapped or stale vertices (rgbdImage.cu:126-145)
    has = np.any(n[..., :3] != 0, axis=-1)
    assert has.sum() > 1000
    np.testing.assert_array_equal(n[has][:, :3].view(np.uint32), gold["normals"][has].view(np.uint32))


def test_reference_bilateral(gold, oracle):
    sensor, _ = structs(gold)
    d = oracle.depth_from_raw(gold["depth"][int(gold["bilateral_src_frame"])], sensor.depth_scaler)
    out = oracle.bilateral(d, abi.BilateralParams(diameter=8, sigma_i=10.0, sigma_s=1.0, enabled=1))
    ref = gold["bilateral"]
    # compare where the reference window is fully inside and fully valid
    r = 8
    ok = np.zeros_like(d, bool)
    for x in range(r, d.shape[0] - r + 1):
        for y in range(r, d.shape[1] - r + 1):
            ok[x, y] = np.all(d[x - r:x + r, y - r:y + r] > 0)
    assert ok.sum() > 100
    np.testing.assert_allclose(out[ok], ref[ok], rtol=3e-7, atol=0)


def test_reference_hash(gold, oracle):
    _, tsdf = structs(gold)
    L = oracle.lib()
    for (x, y, z), h in zip(gold["hash_coords"], gold["hash_values"]):
        assert L.dyo_hash(int(x), int(y), int(z), tsdf.num_buckets, tsdf.bucket_size) == h


def test_reference_icp_normal_equations(oracle):
    """buildNLSKernel's 6x6 A and b (gnSolver.cu:26-196) for three
    transforms: the oracle's per-pixel terms summed in the reference's order
    (FP32, pixel order) are bit-identical; its FP64 sums agree to FP32
    summation error."""
    z = np.load(os.path.join(HERE, "golden", "ref_icp_normal_equations.npz"))
    r, c, fx, fy, cx, cy, ds = z["sensor"]
    s = abi.Sensor(rows=int(r), cols=int(c), fx=fx, fy=fy, cx=cx, cy=cy, depth_scaler=ds)
    _, g, _, _ = abi.defaults()
    # the reference's constants: depth window 0.15-2.0 m (pyramid.h:15-16),
    # colour weight 0 (gnSolver.cu:180), |cos| > cos(pi/10) compared in
    # double -- for a float cosine, > the float just below float(cos(pi/10))
    g.icp_min_depth, g.icp_max_depth, g.color_weight = 0.15, 2.0, 0.0
    thr = np.float32(np.cos(np.pi / 10))
    g.normal_cos_thresh = float(np.nextafter(thr, np.float32(0)))

    def n4(n3):
        n = np.zeros(n3.shape[:2] + (4,), np.float32)
        n[..., :3] = n3
        return n

    sn, tn = n4(z["src_normals"]), n4(z["tgt_normals"])
    for k in range(len(z["transforms"])):
        A, b, cnt = oracle.icp_normal_equations_refsum(z["src_depth"], sn, None, z["tgt_depth"],
                                                        tn, None, s, g, z["transforms"][k])
        assert cnt > 250
        np.testing.assert_array_equal(A.view(np.uint32), z["A"][k].view(np.uint32))
        np.testing.assert_array_equal(b.view(np.uint32), z["b"][k].view(np.uint32))
        out = oracle.icp_normal_equations(z["src_depth"], sn, None, z["tgt_depth"], tn, None,
                                          s, g, z["transforms"][k])
        Af = z["A"][k].astype(np.float64).reshape(6, 6)
        up = np.array([Af[i, j] for i in range(6) for j in range(i, 6)])
        np.testing.assert_allclose(out[:21], up, rtol=1e-5, atol=1e-4)
        np.testing.assert_allclose(out[21:27], z["b"][k], rtol=1e-5, atol=1e-4)
        assert out[28] == cnt


def test_reference_icp_photometric(oracle):
    """buildNLSKernel with its photometric term on (gnSolver.cu:136-193):
    the reference's colour weight (a constant 0 at :180) set to 0.1, RGB
    from the sequence's texture.  The oracle's per-pixel terms -- luma
    intensities, the one-sided gradient at (x-1) and (y-1) halved, the
    Jacobian grad(I) [-p^ | I], the blend (1-w) A + w Jc^T Jc and
    (1-w) b + w Jc^T (I_t - I_s) -- summed in the reference's order are
    bit-identical for three transforms."""
    z = np.load(os.path.join(HERE, "golden", "ref_icp_normal_equations.npz"))
    r, c, fx, fy, cx, cy, ds = z["sensor"]
    s = abi.Sensor(rows=int(r), cols=int(c), fx=fx, fy=fy, cx=cx, cy=cy, depth_scaler=ds)
    _, g, _, _ = abi.defaults()
    g.icp_min_depth, g.icp_max_depth = 0.15, 2.0
    g.color_weight = float(z["color_weight"])
    thr = np.float32(np.cos(np.pi / 10))
    g.normal_cos_thresh = float(np.nextafter(thr, np.float32(0)))

    def n4(n3):
        n = np.zeros(n3.shape[:2] + (4,), np.float32)
        n[..., :3] = n3
        return n

    sn, tn = n4(z["src_normals"]), n4(z["tgt_normals"])
    si, ti = oracle.intensity(z["src_rgb"]), oracle.intensity(z["tgt_rgb"])
    for k in range(len(z["transforms"])):
        A, b, cnt = oracle.icp_normal_equations_refsum(z["src_depth"], sn, si, z["tgt_depth"],
                                                        tn, ti, s, g, z["transforms"][k])
        assert cnt > 250
        # the colour term changes the system
        assert not np.array_equal(z["A_color"][k], z["A"][k])
        np.testing.assert_array_equal(A.view(np.uint32), z["A_color"][k].view(np.uint32))
        np.testing.assert_array_equal(b.view(np.uint32), z["b_color"][k].view(np.uint32))
        out = oracle.icp_normal_equations(z["src_depth"], sn, si, z["tgt_depth"], tn, ti,
                                          s, g, z["transforms"][k])
        Af = z["A_color"][k].astype(np.float64).reshape(6, 6)
        up = np.array([Af[i, j] for i in range(6) for j in range(i, 6)])
        np.testing.assert_allclose(out[:21], up, rtol=1e-5, atol=1e-4)
        np.testing.assert_allclose(out[21:27], z["b_color"][k], rtol=1e-5, atol=1e-4)
        assert out[28] == cnt


def test_reference_gn_solve(oracle):
    """gnSolver::solve (gnSolver.cu:317-438) from the identity, every level
    at full resolution, for three settings (the last trips the
    max_increment guard): the oracle's GN loop over the reference-order sums
    reproduces the reference's final increment bit for bit.  The Eigen calls
    are the shared LDL^T / SE(3) exponential of oracle/gn_algebra.h, so this
    pins the reference's own loop: scaling, damping, convergence test,
    iteration counts and guards."""
    z = np.load(os.path.join(HERE, "golden", "ref_icp_normal_equations.npz"))
    r, c, fx, fy, cx, cy, ds = z["sensor"]
    s = abi.Sensor(rows=int(r), cols=int(c), fx=fx, fy=fy, cx=cx, cy=cy, depth_scaler=ds)

    def n4(n3):
        n = np.zeros(n3.shape[:2] + (4,), np.float32)
        n[..., :3] = n3
        return n

    sn, tn = n4(z["src_normals"]), n4(z["tgt_normals"])
    moved = 0
    for iters, (mi, ma, rg), inc in zip(z["solve_iters"], z["solve_thresholds"], z["solve_inc"]):
        _, g, _, _ = abi.defaults()
        g.icp_min_depth, g.icp_max_depth, g.color_weight = 0.15, 2.0, 0.0
        g.normal_cos_thresh = float(np.nextafter(np.float32(np.cos(np.pi / 10)), np.float32(0)))
        g.lvl_iteration_num[:] = [int(x) for x in iters]
        g.lvl_scale[:] = [1, 1, 1]
        g.min_increment, g.max_increment, g.regularization = float(mi), float(ma), float(rg)
        got = oracle.gn_solve_refsum(z["src_depth"], sn, z["tgt_depth"], tn, s, g)
        np.testing.assert_array_equal(got.view(np.uint64), inc.view(np.uint64))
        moved += int(np.any(inc != 0))
    assert moved == 2  # two settings converge to a motion, the guard zeroes the third


def test_reference_mesh_vertices(oracle_volume):
    """MeshExtractor::ExtractMesh (meshExtractor.cu:22-214, 364-407) over a
    box of the pinned volume: the oracle's vertices -- corner samples that
    give up at an unobserved corner, the cube edges that cross zero, the
    reference's edge interpolation and centre-voxel colour -- are exactly
    the distinct vertices of the reference's triangles."""
    vol, _ = oracle_volume
    z = np.load(os.path.join(HERE, "golden", "ref_mesh_vertices.npz"))
    lo, hi = z["box"]
    got = vol.mesh_vertices(lo, hi)
    uniq = np.unique(np.ascontiguousarray(got).view(np.uint32), axis=0)
    assert len(got) >= len(uniq) > 1000
    np.testing.assert_array_equal(uniq, z["vertices"].view(np.uint32))


def test_mesh_with_own_table_against_reference(oracle_volume):
    """The same box meshed with this project's generated marching-cubes
    table (the reference's table is not copied): its vertices are the
    reference's, and its triangle count and area match the reference's
    mesh (the tables may split a cell's polygons differently)."""
    vol, _ = oracle_volume
    z = np.load(os.path.join(HERE, "golden", "ref_mesh_vertices.npz"))
    lo, hi = z["box"]
    tris = vol.mesh_triangles(lo, hi)
    uniq = np.unique(np.ascontiguousarray(tris.reshape(-1, 6)).view(np.uint32), axis=0)
    np.testing.assert_array_equal(uniq, z["vertices"].view(np.uint32))
    assert len(tris) == int(z["triangles"])
    p = tris[:, :, :3].astype(np.float64)
    area = 0.5 * np.linalg.norm(np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), axis=1).sum()
    assert abs(area - float(z["area"])) < 5e-3 * float(z["area"])
