"""Parity of the CUDA path (libdynamap_b200.so, through its C ABI) with the
CPU oracle on identical seeded inputs.

Bars: allocation (block set), integration (voxel sdf bits, weights, colours)
and raycast are bit-exact; bilateral-filtered depth within 2e-6 relative
(the range weight uses FP32 exp where the reference uses FP64); the normal
equations within 1e-6 relative; tracked poses within 1e-4 m / 1e-4 rad.
"""
import ctypes as C

import numpy as np
import pytest

from dynamap_b200 import abi, configs
from dynamap_b200.session import Session

pytestmark = pytest.mark.gpu


def small_cfg1(**over):
    p = configs.preset("cfg1")
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    for k, v in over.items():
        p[k].update(v)
    return p


@pytest.fixture(scope="module")
def seq_cfg1():
    return configs.sequence(configs.preset("cfg1"), seed=3, n_frames=12)


def sort_blocks(coords, *arrs):
    order = np.lexsort((coords[:, 2], coords[:, 1], coords[:, 0]))
    return (coords[order],) + tuple(a[order] for a in arrs)


def assert_volume_equal(gpu: Session, ovol):
    gc, grgbw, gsdf = gpu.download_blocks()
    oc, orgbw, osdf = ovol.download()
    assert gc.shape == oc.shape, f"block count gpu {len(gc)} oracle {len(oc)}"
    gc, grgbw, gsdf = sort_blocks(gc, grgbw, gsdf)
    oc, orgbw, osdf = sort_blocks(oc, orgbw, osdf)
    np.testing.assert_array_equal(gc, oc)
    np.testing.assert_array_equal(grgbw[..., 3], orgbw[..., 3])        # weights
    np.testing.assert_array_equal(grgbw, orgbw)                          # colours
    np.testing.assert_array_equal(gsdf.view(np.uint32), osdf.view(np.uint32))  # sdf bits


def test_integration_bitexact(gpu_lib, oracle, seq_cfg1):
    p = small_cfg1()
    t, g, b, s = configs.structs(p)
    ovol = oracle.Volume(t)
    with Session(t, g, b, s) as m:
        for k in range(4):
            pose = seq_cfg1.poses[k].astype(np.float32)
            m.integrate_with_pose(seq_cfg1.depth[k], None, pose)
            d = oracle.depth_from_raw(seq_cfg1.depth[k], s.depth_scaler)
            c1 = ovol.allocate(d, s, pose)
            c2 = ovol.integrate(d, None, s, pose)
            assert c1[oracle.C_BUCKET_FULL] == 0 and c1[oracle.C_HEAP] == 0
            assert c2[oracle.C_REHASH] == 0  # the camera->world round trip is the identity
        assert_volume_equal(m, ovol)


def test_integration_rgb_bitexact(gpu_lib, oracle):
    p = configs.preset("cfg2")
    p["sensor"].update(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5)
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    seq = configs.sequence(p, seed=5, n_frames=3)
    t, g, b, s = configs.structs(p)
    ovol = oracle.Volume(t)
    with Session(t, g, b, s) as m:
        for k in range(3):
            pose = seq.poses[k].astype(np.float32)
            m.integrate_with_pose(seq.depth[k], seq.rgb[k], pose)
            d = oracle.depth_from_raw(seq.depth[k], s.depth_scaler)
            ovol.allocate(d, s, pose)
            ovol.integrate(d, seq.rgb[k], s, pose)
        assert_volume_equal(m, ovol)
        # raycast depth and colour
        pose = seq.poses[2].astype(np.float32)
        gd, grgb = m.raycast(pose, rgb=True)
        od, orgb, _ = ovol.raycast(pose, s, rgb=True)
        np.testing.assert_array_equal(gd.view(np.uint32), od.view(np.uint32))
        np.testing.assert_array_equal(grgb, orgb)


def test_raycast_bitexact(gpu_lib, oracle, seq_cfg1):
    p = small_cfg1()
    t, g, b, s = configs.structs(p)
    ovol = oracle.Volume(t)
    with Session(t, g, b, s) as m:
        for k in range(3):
            pose = seq_cfg1.poses[k].astype(np.float32)
            m.integrate_with_pose(seq_cfg1.depth[k], None, pose)
            d = oracle.depth_from_raw(seq_cfg1.depth[k], s.depth_scaler)
            ovol.allocate(d, s, pose)
            ovol.integrate(d, None, s, pose)
        for k in (2, 5):
            pose = seq_cfg1.poses[k].astype(np.float32)
            gd, _ = m.raycast(pose)
            od, _, c = ovol.raycast(pose, s)
            assert c[oracle.C_RC] == 0
            np.testing.assert_array_equal(gd.view(np.uint32), od.view(np.uint32))
        # a virtual sensor at half resolution (builder::GenerateDepth scales
        # the intrinsics, builder.cu:179-196)
        vs = oracle.level_sensor(s, 2)
        gd, _ = m.raycast(seq_cfg1.poses[2].astype(np.float32), sensor=vs)
        od, _, _ = ovol.raycast(seq_cfg1.poses[2].astype(np.float32), vs)
        np.testing.assert_array_equal(gd.view(np.uint32), od.view(np.uint32))


def _torch():
    import torch
    return torch


def test_bilateral_and_maps(gpu_lib, oracle, seq_cfg1):
    torch = _torch()
    p = small_cfg1()
    t, g, b, s = configs.structs(p)
    raw = oracle.depth_from_raw(seq_cfg1.depth[0], s.depth_scaler)
    # stage entry point on caller device buffers
    dsrc = torch.from_numpy(raw).cuda()
    dout = torch.empty_like(dsrc)
    abi.check("dyn_bilateral_filter", gpu_lib.dyn_bilateral_filter(
        dsrc.data_ptr(), dout.data_ptr(), s.rows, s.cols, C.byref(b), None))
    torch.cuda.synchronize()
    ob = oracle.bilateral(raw, b)
    gb = dout.cpu().numpy()
    assert np.array_equal(gb == 0, ob == 0)
    np.testing.assert_allclose(gb, ob, rtol=2e-6, atol=0)
    # maps from the same (oracle) depth are bit-exact
    for scale in (1, 2, 4):
        ls = oracle.level_sensor(s, scale)
        dl = ob
        for _ in range({1: 0, 2: 1, 4: 2}[scale]):
            dl = oracle.downsample_depth(dl)
        ov, on = oracle.maps(dl, ls)
        dd = torch.from_numpy(np.ascontiguousarray(dl)).cuda()
        gv = torch.empty((ls.rows, ls.cols, 4), dtype=torch.float32, device="cuda")
        gn = torch.empty_like(gv)
        abi.check("dyn_depth_to_maps", gpu_lib.dyn_depth_to_maps(
            dd.data_ptr(), C.byref(ls), gv.data_ptr(), gn.data_ptr(), None))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(gv.cpu().numpy().view(np.uint32), ov.view(np.uint32))
        np.testing.assert_array_equal(gn.cpu().numpy().view(np.uint32), on.view(np.uint32))


def test_session_images_match_oracle(gpu_lib, oracle, seq_cfg1):
    """Pyramid depth, normals and the raycast target after one frame."""
    p = small_cfg1()
    t, g, b, s = configs.structs(p)
    os_ = oracle.Session(t, g, b, s)
    os_.set_pose(seq_cfg1.poses[0])
    os_.frame(seq_cfg1.depth[0])
    with Session(t, g, b, s) as m:
        m.set_pose(seq_cfg1.poses[0])
        m.process(seq_cfg1.depth[0])
        raw = m.image(0, 0, (s.rows, s.cols), np.float32)
        np.testing.assert_array_equal(raw, os_.image(0, 0, (s.rows, s.cols), np.float32))
        filt = m.image(1, 0, (s.rows, s.cols), np.float32)
        np.testing.assert_allclose(filt, os_.image(1, 0, (s.rows, s.cols), np.float32),
                                   rtol=2e-6, atol=0)
        # target (raycast) depth is bit-exact: same volume, same pose
        for lvl in range(3):
            sh = (s.rows >> lvl, s.cols >> lvl)
            gt = m.image(5, lvl, sh, np.float32)
            ot = os_.image(5, lvl, sh, np.float32)
            np.testing.assert_array_equal(gt.view(np.uint32), ot.view(np.uint32))
            gn = m.image(7, lvl, sh + (4,), np.float32)
            on = os_.image(7, lvl, sh + (4,), np.float32)
            np.testing.assert_array_equal(gn.view(np.uint32), on.view(np.uint32))


def test_icp_normal_equations(gpu_lib, oracle, seq_cfg1):
    torch = _torch()
    p = small_cfg1()
    t, g, b, s = configs.structs(p)
    for scale in (4, 1):
        ls = oracle.level_sensor(s, scale)
        def level(depth):
            d = oracle.bilateral(oracle.depth_from_raw(depth, s.depth_scaler), b)
            while d.shape[0] > ls.rows:
                d = oracle.downsample_depth(d)
            return d
        sd, td = level(seq_cfg1.depth[1]), level(seq_cfg1.depth[0])
        _, sn = oracle.maps(sd, ls)
        _, tn = oracle.maps(td, ls)
        rel = np.linalg.inv(seq_cfg1.poses[0]) @ seq_cfg1.poses[1]
        T = rel.astype(np.float32)
        ref = oracle.icp_normal_equations(sd, sn, None, td, tn, None, ls, g, T)
        assert ref[28] > 100
        dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (sd, sn, td, tn)]
        out = (C.c_double * 29)()
        Tc = (C.c_float * 16)(*T.reshape(16).tolist())
        abi.check("dyn_icp_normal_equations", gpu_lib.dyn_icp_normal_equations(
            dev[0].data_ptr(), dev[1].data_ptr(), None, dev[2].data_ptr(), dev[3].data_ptr(),
            None, C.byref(ls), C.byref(g), Tc, out, None))
        got = np.array(out)
        assert got[28] == ref[28]
        np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-9 * np.abs(ref).max())


def rot_angle(R):
    """Angle of a near-identity rotation from its skew part (accurate for
    small angles, unlike arccos of the trace)."""
    w = np.array([R[2, 1] - R[1, 2], R[0, 2] - R[2, 0], R[1, 0] - R[0, 1]]) / 2
    return float(np.arcsin(min(1.0, np.linalg.norm(w))))


@pytest.mark.parametrize("bilateral", [1, 0])
def test_tracking_matches_oracle(gpu_lib, oracle, seq_cfg1, bilateral):
    p = small_cfg1(bilateral=dict(enabled=bilateral))
    t, g, b, s = configs.structs(p)
    os_ = oracle.Session(t, g, b, s)
    os_.set_pose(seq_cfg1.poses[0])
    with Session(t, g, b, s) as m:
        m.set_pose(seq_cfg1.poses[0])
        for k in range(len(seq_cfg1.depth)):
            gp, gst = m.process(seq_cfg1.depth[k])
            op, ost = os_.frame(seq_cfg1.depth[k])
            dt = np.linalg.norm(gp[:3, 3] - op[:3, 3])
            dr = rot_angle(gp[:3, :3].astype(np.float64).T @ op[:3, :3].astype(np.float64))
            assert dt < 1e-4 and dr < 1e-4, (k, dt, dr)
            assert list(gst.icp_iterations) == list(ost.icp_iterations)
        # and the tracked trajectory follows the ground truth
        te = np.linalg.norm(gp[:3, 3] - seq_cfg1.poses[-1][:3, 3])
        assert te < 0.02


def test_deterministic(gpu_lib, seq_cfg1):
    p = small_cfg1()
    t, g, b, s = configs.structs(p)
    outs = []
    for _ in range(2):
        with Session(t, g, b, s) as m:
            m.set_pose(seq_cfg1.poses[0])
            for k in range(5):
                pose, _ = m.process(seq_cfg1.depth[k])
            c, rgbw, sdf = m.download_blocks()
            c, rgbw, sdf = sort_blocks(c, rgbw, sdf)
            outs.append((pose, c, rgbw, sdf))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    for a, b_ in zip(outs[0][1:], outs[1][1:]):
        np.testing.assert_array_equal(a, b_)


def test_empty_frame_and_odd_sizes(gpu_lib, oracle):
    p = small_cfg1()
    p["sensor"].update(rows=123, cols=161, cx=80.0, cy=61.0)
    seq = configs.sequence(p, seed=9, n_frames=3)
    t, g, b, s = configs.structs(p)
    ovol = oracle.Volume(t)
    with Session(t, g, b, s) as m:
        m.set_pose(seq.poses[0])
        pose, st = m.process(np.zeros((s.rows, s.cols), np.uint16))
        assert st.blocks_total == 0 and st.blocks_new == 0
        pose, st = m.process(seq.depth[1])  # no target yet after an empty map
        m.integrate_with_pose(seq.depth[2], None, seq.poses[2].astype(np.float32))
        d = oracle.depth_from_raw(seq.depth[2], s.depth_scaler)
        # the empty frame allocated nothing; frame 1 integrated at pose 0
        ovol.allocate(oracle.depth_from_raw(seq.depth[1], s.depth_scaler), s,
                      seq.poses[0].astype(np.float32))
        ovol.integrate(oracle.depth_from_raw(seq.depth[1], s.depth_scaler), None, s,
                       seq.poses[0].astype(np.float32))
        ovol.allocate(d, s, seq.poses[2].astype(np.float32))
        ovol.integrate(d, None, s, seq.poses[2].astype(np.float32))
        assert_volume_equal(m, ovol)


def test_bucket_full_and_heap_exhausted_are_reported(gpu_lib, oracle, seq_cfg1):
    # tiny heap: the frame reports HEAP_EXHAUSTED, never corrupts memory
    p = small_cfg1()
    p["tsdf"].update(num_blocks=512)
    t, g, b, s = configs.structs(p)
    with Session(t, g, b, s) as m:
        with pytest.raises(abi.DynError) as e:
            m.integrate_with_pose(seq_cfg1.depth[0], None, seq_cfg1.poses[0].astype(np.float32))
        assert e.value.status == abi.DYN_ERR_HEAP_EXHAUSTED
        assert m.num_blocks() == 512
    # tiny table: buckets overflow and are counted
    p = small_cfg1()
    p["tsdf"].update(num_buckets=64, bucket_size=4)
    t, g, b, s = configs.structs(p)
    with Session(t, g, b, s) as m:
        with pytest.raises(abi.DynError) as e:
            m.integrate_with_pose(seq_cfg1.depth[0], None, seq_cfg1.poses[0].astype(np.float32))
        assert e.value.status == abi.DYN_ERR_HASH_FULL
        assert m.num_blocks() <= 64 * 4


def test_large_frame_1280x720(gpu_lib, oracle):
    """Largest sensor of the serving configuration: integration bit-exact."""
    p = configs.preset("cfg1")
    p["sensor"].update(rows=720, cols=1280, fx=900.0, fy=900.0, cx=639.5, cy=359.5)
    p["tsdf"].update(num_blocks=1 << 17, num_buckets=1 << 18)
    seq = configs.sequence(p, seed=11, n_frames=1)
    t, g, b, s = configs.structs(p)
    ovol = oracle.Volume(t)
    with Session(t, g, b, s) as m:
        pose = seq.poses[0].astype(np.float32)
        m.integrate_with_pose(seq.depth[0], None, pose)
        d = oracle.depth_from_raw(seq.depth[0], s.depth_scaler)
        ovol.allocate(d, s, pose)
        ovol.integrate(d, None, s, pose)
        assert_volume_equal(m, ovol)
