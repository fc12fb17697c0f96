"""Boundary entries beside the reference's: the raycast's vertex and normal
maps (dyn_raycast_maps) and tracking from a pose hint
(dyn_frame_submit_hint)."""
import numpy as np
import pytest

from dynamap_b200 import abi, configs
from dynamap_b200.session import Session

pytestmark = pytest.mark.gpu


def small():
    p = configs.preset("cfg1")
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    return p


def test_raycast_maps_match_the_oracle(gpu_lib, oracle):
    p = small()
    seq = configs.sequence(p, seed=31, n_frames=4)
    t, g, b, s = configs.structs(p)
    with Session(t, g, b, s) as m:
        m.set_pose(seq.poses[0])
        for k in range(4):
            m.process(seq.depth[k])
        pose = m.pose()
        d0, _ = m.raycast(pose)
        d, v, n, _ = m.raycast_maps(pose)
    np.testing.assert_array_equal(d.view(np.uint32), d0.view(np.uint32))
    valid = np.where(d < t.max_sensor_depth, d, 0).astype(np.float32)
    ov, on = oracle.maps(valid, s)
    np.testing.assert_array_equal(v.view(np.uint32), ov.view(np.uint32))
    np.testing.assert_array_equal(n.view(np.uint32), on.view(np.uint32))
    assert np.count_nonzero(n[..., 2]) > 0.3 * n[..., 2].size


def test_pose_hint(gpu_lib):
    p = small()
    seq = configs.sequence(p, seed=32, n_frames=8)
    t, g, b, s = configs.structs(p)
    gt = seq.poses
    with Session(t, g, b, s) as plain, Session(t, g, b, s) as same, \
            Session(t, g, b, s) as hinted:
        for m in (plain, same):
            m.set_pose(gt[0])
        # before the first target exists the hint becomes the pose
        hinted.process(seq.depth[0], pose_hint=gt[0])
        np.testing.assert_allclose(hinted.pose(), gt[0].astype(np.float32), atol=1e-6)
        plain.process(seq.depth[0])
        same.process(seq.depth[0])
        for k in range(1, len(seq.depth)):
            a = plain.process(seq.depth[k])[0]
            # a hint equal to the current pose (rounded to float): the same
            # tracking as no hint, up to where the solver's 1e-3 increment
            # threshold stops it
            c = same.process(seq.depth[k], pose_hint=same.pose())[0]
            assert np.linalg.norm(c[:3, 3] - a[:3, 3]) < 5e-4
            R = c[:3, :3].T @ a[:3, :3]
            assert np.arccos(np.clip((np.trace(R) - 1) / 2, -1, 1)) < 1e-3
            # the true pose as the hint: tracking stays at the truth
            h = hinted.process(seq.depth[k], pose_hint=gt[k])[0]
            assert np.linalg.norm(h[:3, 3] - gt[k][:3, 3]) < 1e-2


def test_two_frames_in_flight_give_the_sequential_results(gpu_lib):
    """dyn_frame_submit of frame k+1 before frame k's dyn_frame_result (the
    copy of k+1 overlapping frame k's work, through the second input slot):
    every frame's pose and statistics equal those of one frame at a time,
    from pageable and from page-locked frames, and device frames too."""
    import torch
    p = small()
    p["sensor"].update(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5)
    seq = configs.sequence(p, seed=35, n_frames=9)
    t, g, b, s = configs.structs(p)
    with Session(t, g, b, s) as m:
        m.set_pose(seq.poses[0])
        ref = [m.process(seq.depth[k]) for k in range(len(seq.depth))]
    pinned = torch.from_numpy(seq.depth).pin_memory().numpy()
    dev = torch.from_numpy(seq.depth).cuda()
    nb = seq.depth.shape[1] * seq.depth.shape[2] * 2
    for source in ("pageable", "pinned", "device"):
        with Session(t, g, b, s) as m:
            m.set_pose(seq.poses[0])
            got = []

            def submit(k):
                if source == "device":
                    m.submit_device(dev.data_ptr() + k * nb)
                else:
                    m.submit((seq.depth if source == "pageable" else pinned)[k])
            submit(0)
            for k in range(1, len(seq.depth)):
                submit(k)
                got.append(m.result())
            got.append(m.result())
            with pytest.raises(abi.DynError):
                m.result()  # nothing in flight
        for k, ((pa, sa), (pb, sb)) in enumerate(zip(ref, got)):
            np.testing.assert_array_equal(pa, pb, err_msg=f"{source} frame {k}")
            assert list(sa.icp_iterations) == list(sb.icp_iterations)
            assert sa.blocks_total == sb.blocks_total
