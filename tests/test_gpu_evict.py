"""Block eviction and streaming on the GPU (dyn_evict_blocks,
dyn_delete_blocks, dyn_upload_blocks; dynamap_b200/csrc/evict.cu) on a
session's volume: deleted blocks come out with their voxels in heap order,
the rest stay as they were, and uploading the removed blocks restores the
map -- the same block set and voxels bit for bit, and the same raycast (bit
for bit in the FP32 form; within the raycast tolerance in the mixed form,
whose free-cell flags the upload leaves cleared); eviction by age keeps exactly the blocks
the last frames' allocation touched (the oracle's allocation of those
frames alone), and the session integrates on afterwards."""
import numpy as np
import pytest

from dynamap_b200 import abi, configs
from dynamap_b200.session import Session
from raycast_check import assert_raycast_close

pytestmark = pytest.mark.gpu


def small_rgb():
    p = configs.preset("cfg2")
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    p["sensor"].update(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5)
    return p


def as_map(coords, rgbw, sdf):
    return {tuple(c): (w.tobytes(), s.tobytes()) for c, w, s in zip(coords.tolist(), rgbw, sdf)}


@pytest.mark.parametrize("precision", [abi.PRECISION_FP32, abi.PRECISION_MIXED])
def test_delete_then_upload_restores_the_map(gpu_lib, precision):
    p = small_rgb()
    seq = configs.sequence(p, seed=41, n_frames=4)
    t, g, b, s = configs.structs(p)
    with Session(t, g, b, s, precision=precision) as m:
        for k in range(4):
            m.integrate_with_pose(seq.depth[k], seq.rgb[k], seq.poses[k].astype(np.float32))
        pose = seq.poses[3].astype(np.float32)
        d0, c0 = m.raycast(pose, rgb=True)
        pre = m.download_blocks()
        n = len(pre[0])
        sel = np.sort(np.random.default_rng(5).choice(n, n // 3, replace=False))
        extra = np.array([[900, 900, 900]], np.int32)  # no block there
        out = m.delete_blocks(np.concatenate([pre[0][sel], pre[0][sel[:7]], extra]))
        # removed in heap order, with their voxels
        for a, want in zip(out, pre):
            np.testing.assert_array_equal(a, want[sel])
        rest = np.setdiff1d(np.arange(n), sel)
        post = m.download_blocks()
        assert m.num_blocks() == len(rest)
        assert as_map(*post) == as_map(*(a[rest] for a in pre))
        counts = m.upload_blocks(*out)
        assert list(counts) == [len(sel), 0, 0, 0]
        assert as_map(*m.download_blocks()) == as_map(*pre)
        d1, c1 = m.raycast(pose, rgb=True)
        if precision == abi.PRECISION_FP32:  # the same voxels: the same raycast
            np.testing.assert_array_equal(d1.view(np.uint32), d0.view(np.uint32))
            np.testing.assert_array_equal(c1, c0)
        else:
            # the mixed march steps through free cells by their flags, and
            # the uploaded blocks' flags start cleared: the same steps up
            # to rounding
            assert_raycast_close(d1, d0, t.voxel_size, t.max_sensor_depth, c1, c0)
        # present keys are left as they are
        assert list(m.upload_blocks(*(a[:5] for a in out))) == [0, 5, 0, 0]


def test_evict_by_age_keeps_the_last_frames_blocks(gpu_lib, oracle):
    p = small_rgb()
    p["tsdf"].update(num_blocks=1 << 17, num_buckets=1 << 18)  # the far views hold more
    seq = configs.sequence(p, seed=42, n_frames=51)
    t, g, b, s = configs.structs(p)
    order = [0, 1, 2, 3, 40, 45, 50]  # the last views far from the first ones

    def frame_blocks(k):
        vol = oracle.Volume(t)
        vol.allocate(oracle.depth_from_raw(seq.depth[k], s.depth_scaler), s,
                     seq.poses[k].astype(np.float32))
        return {tuple(c) for c in vol.download()[0].tolist()}

    with Session(t, g, b, s) as m:
        for k in order[:6]:
            m.integrate_with_pose(seq.depth[k], seq.rgb[k], seq.poses[k].astype(np.float32))
        before = {tuple(c) for c in m.download_blocks()[0].tolist()}
        assert m.evict_blocks(10, out=False) == 0  # all within ten frames
        keep = frame_blocks(order[4]) | frame_blocks(order[5])
        assert keep < before
        gone = m.evict_blocks(1)
        assert {tuple(c) for c in gone[0].tolist()} == before - keep
        after = m.download_blocks()[0]
        assert {tuple(c) for c in after.tolist()} == keep
        assert len(after) == len(keep)
        # integration goes on from the freed heap
        k = order[6]
        m.integrate_with_pose(seq.depth[k], seq.rgb[k], seq.poses[k].astype(np.float32))
        c6 = m.download_blocks()[0]
        got = {tuple(c) for c in c6.tolist()}
        assert len(got) == len(c6) and got == keep | frame_blocks(k)
