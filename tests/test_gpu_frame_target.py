"""The frame's raycast (the fused per-frame launch) must equal the stage
entry point dyn_raycast at the same pose, after several frames, for a
camera looking into a box (cube) and inside a room (blocks beside and
behind the camera).  The frame raycast skips the lookups outside its
per-tile depth bounds, which dyn_raycast does not use.  FP32 and mixed
with band allocation: bit for bit, in depth and colour.  Mixed with
carving: its near bound is the nearest block holding observed non-saturated
voxels, and before it the frame's march steps exactly the truncation where
the full march may interpolate saturated voxels (the truncation up to the
rounding of the weights), so the two agree bit for bit on nearly every
pixel and within the mixed raycast's tolerance everywhere."""
import numpy as np
import pytest

from dynamap_b200 import abi, configs
from dynamap_b200.session import Session
from raycast_check import assert_raycast_close

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["cube", "room"])
@pytest.mark.parametrize("prec", [abi.PRECISION_FP32, abi.PRECISION_MIXED,
                                  abi.PRECISION_MIXED_BAND])
def test_frame_target_equals_full_march(gpu_lib, kind, prec):
    p = configs.preset("cfg2")
    p["sensor"].update(rows=240, cols=320, fx=262.5, fy=262.5, cx=159.5, cy=119.5)
    p["tsdf"].update(num_blocks=1 << 17, num_buckets=1 << 18)
    p["seq"].update(kind=kind)
    seq = configs.sequence(p, seed=61, n_frames=6)
    t, g, b, s = configs.structs(p)
    with Session(t, g, b, s, precision=prec) as m:
        m.set_pose(seq.poses[0])
        for k in range(len(seq.depth)):
            m.process(seq.depth[k], seq.rgb[k])
            if k < 2:
                continue
            pose = m.pose()
            full, rgb = m.raycast(pose, rgb=True)
            full0 = np.where(full < t.max_sensor_depth, full, 0).astype(np.float32)
            tgt = m.image(5, 0, (s.rows, s.cols), np.float32)
            trgb = m.image(8, 0, (s.rows, s.cols, 3), np.uint8)
            assert np.count_nonzero(tgt) > 0.3 * tgt.size
            if prec != abi.PRECISION_MIXED:
                np.testing.assert_array_equal(tgt.view(np.uint32), full0.view(np.uint32))
                np.testing.assert_array_equal(trgb, rgb)
                continue
            same = float(np.mean(tgt.view(np.uint32) == full0.view(np.uint32)))
            assert same >= 0.99, same
            far = np.float32(t.max_sensor_depth)
            assert_raycast_close(np.where(tgt > 0, tgt, far), np.where(full0 > 0, full0, far),
                                 t.voxel_size, t.max_sensor_depth, trgb, rgb)
