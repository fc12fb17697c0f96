"""The frame's raycast (the fused per-frame launch) must equal the stage
entry point dyn_raycast at the same pose bit for bit, in depth and colour,
FP32, mixed and mixed with band allocation (the frame raycast skips the
lookups outside its per-tile depth bounds, which dyn_raycast does not use),
after several frames, for a camera looking into a box (cube) and inside a
room (blocks beside and behind the camera)."""
import numpy as np
import pytest

from dynamap_b200 import abi, configs
from dynamap_b200.session import Session

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
            np.testing.assert_array_equal(tgt.view(np.uint32), full0.view(np.uint32))
            trgb = m.image(8, 0, (s.rows, s.cols, 3), np.uint8)
            np.testing.assert_array_equal(trgb, rgb)
            assert np.count_nonzero(tgt) > 0.3 * tgt.size
