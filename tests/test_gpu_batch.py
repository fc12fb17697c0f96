"""dyn_batch: sessions stepped together (one fused launch per stage, one
graph per frame) give bit-identical results to the same sessions stepped
alone.  Members differ in sensor size, RGB, precision, mode and filtering."""
import numpy as np
import pytest

from dynamap_b200 import abi, configs
from dynamap_b200.session import Batch, Session

pytestmark = pytest.mark.gpu


def member_params():
    out = []
    p = configs.preset("cfg1")  # 320x240 depth only, FP32
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    out.append((p, abi.PRECISION_FP32))
    p = configs.preset("cfg2")  # 160x120 RGB + photometric term, FP32
    p["sensor"].update(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5)
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    out.append((p, abi.PRECISION_FP32))
    p = configs.preset("cfg1")  # mixed precision, no bilateral filter
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    p["bilateral"].update(enabled=0)
    out.append((p, abi.PRECISION_MIXED))
    p = configs.preset("cfg2")  # mixed, frame-to-frame, RGB, other level scales
    p["sensor"].update(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5)
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    p["gn"].update(mode=0, lvl_scale=[4, 2, 1], lvl_iteration_num=[6, 4, 3])
    out.append((p, abi.PRECISION_MIXED))
    p = configs.preset("cfg1")  # band allocation (ray-start bound in the raycast)
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    out.append((p, abi.PRECISION_MIXED_BAND))
    return out


N_FRAMES = 5


@pytest.fixture(scope="module")
def members():
    ms = []
    for i, (p, prec) in enumerate(member_params()):
        seq = configs.sequence(p, seed=40 + i, n_frames=N_FRAMES)
        rgb = getattr(seq, "rgb", None)
        frames = []
        for k in range(N_FRAMES):
            # member 1 drops its RGB on frame 2 (the per-frame RGB flag)
            c = None if rgb is None or (i == 1 and k == 2) else rgb[k]
            frames.append((seq.depth[k], c))
        ms.append((p, prec, seq.poses[0].astype(np.float32), frames))
    return ms


def sorted_blocks(coords, rgbw, sdf):
    o = np.lexsort((coords[:, 2], coords[:, 1], coords[:, 0]))
    return coords[o], rgbw[o], sdf[o]


def make(p, prec, pose0):
    t, g, b, s = configs.structs(p)
    m = Session(t, g, b, s, precision=prec)
    m.set_pose(pose0)
    return m


STAT_KEYS = ("blocks_total", "blocks_new", "blocks_visible", "icp_iterations", "icp_inliers")


def stats_tuple(st):
    d = st.as_dict()
    return tuple(np.asarray(d[k]).tolist() for k in STAT_KEYS)


def test_batch_matches_sessions_alone(gpu_lib, members):
    alone_poses, alone_stats, alone_maps = [], [], []
    for p, prec, pose0, frames in members:
        with make(p, prec, pose0) as m:
            poses, stats = [], []
            for d, c in frames:
                pose, st = m.process(d, c)
                poses.append(pose)
                stats.append(stats_tuple(st))
            alone_poses.append(poses)
            alone_stats.append(stats)
            alone_maps.append(sorted_blocks(*m.download_blocks()))
    sess = [make(p, prec, pose0) for p, prec, pose0, _ in members]
    try:
        with Batch(sess) as b:
            assert b.kernels_per_frame() == 0  # graph captured on the first frame
            for k in range(N_FRAMES):
                poses, stats, status = b.process([m[3][k][0] for m in members],
                                                 [m[3][k][1] for m in members])
                assert status == [0] * len(members)
                for i in range(len(members)):
                    assert np.array_equal(poses[i], alone_poses[i][k]), (i, k)
                    assert stats_tuple(stats[i]) == alone_stats[i][k], (i, k)
            # one launch per stage for all members, however many members:
            # the ICP is one persistent launch per summation kind present
            # for every level and iteration (per GN iteration and kind when
            # a table does not fit the resident blocks), the raycast one
            # launch per voxel form present, and at most 18 other stage
            # launches (pyramid levels included)
            iters = sum(max(m[0]["gn"]["lvl_iteration_num"][pl] for m in members) - 1
                        for pl in range(3))
            kpf = b.kernels_per_frame()
            assert 3 <= kpf <= 2 + 2 + 18 or 2 * iters + 2 < kpf <= 2 * iters + 2 + 18, (kpf, iters)
            # member pose readable after the batch frame
            for i, m in enumerate(sess):
                np.testing.assert_array_equal(m.pose(), alone_poses[i][-1])
        for i, m in enumerate(sess):
            gc, grgbw, gsdf = sorted_blocks(*m.download_blocks())
            ac, argbw, asdf = alone_maps[i]
            np.testing.assert_array_equal(gc, ac)
            np.testing.assert_array_equal(grgbw, argbw)
            np.testing.assert_array_equal(gsdf.view(np.uint32), asdf.view(np.uint32))
    finally:
        for m in sess:
            m.close()


def test_batch_membership_rules(gpu_lib, members):
    p, prec, pose0, frames = members[0]
    a = make(p, prec, pose0)
    c = make(*members[1][:3])
    try:
        with pytest.raises(abi.DynError):
            Batch([a, a])  # duplicate member
        b = Batch([a, c])
        with pytest.raises(abi.DynError):
            Batch([a])  # already in a batch
        with pytest.raises(abi.DynError):
            a.submit(frames[0][0])  # frames go through the batch
        with pytest.raises(abi.DynError):
            b.result()  # nothing submitted
        b.process([frames[0][0], members[1][3][0][0]], [None, members[1][3][0][1]])
        b.close()
        # released: the session steps alone again
        a.process(frames[1][0])
    finally:
        a.close()
        c.close()


def test_batch_profile_stage_times(gpu_lib, members):
    sess = [make(p, prec, pose0) for p, prec, pose0, _ in members]
    try:
        with Batch(sess) as b:
            b.profile(True)
            for k in range(3):
                b.process([m[3][k][0] for m in members], [m[3][k][1] for m in members])
            ms, n = b.stage_times()
            assert n == 3
            assert ms[abi.STAGES.index("frame")] > 0
            assert abs(sum(ms[:-1]) - ms[-1]) <= 0.05 * ms[-1] + 1e-3
    finally:
        for m in sess:
            m.close()


def test_grouped_batch_matches_sessions_alone(gpu_lib):
    """17 members: the batch splits them into groups on separate streams."""
    p = configs.preset("cfg1")
    p["sensor"].update(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5)
    p["tsdf"].update(voxel_size=0.01, truncation_distance=0.04, num_blocks=1 << 13,
                     num_buckets=1 << 14)
    n = 17
    seqs = [configs.sequence(p, seed=90 + i, n_frames=3) for i in range(n)]
    t, g, b, s = configs.structs(p)
    precs = [abi.PRECISION_MIXED if i % 3 == 0 else abi.PRECISION_FP32 for i in range(n)]
    alone = []
    for i in range(n):
        with Session(t, g, b, s, precision=precs[i]) as m:
            m.set_pose(seqs[i].poses[0])
            alone.append([m.process(d)[0] for d in seqs[i].depth])
    sess = [Session(t, g, b, s, precision=precs[i]) for i in range(n)]
    try:
        for i, m in enumerate(sess):
            m.set_pose(seqs[i].poses[0])
        with Batch(sess) as bt:
            for k in range(3):
                poses, _, status = bt.process([q.depth[k] for q in seqs])
                assert status == [0] * n
                for i in range(n):
                    assert np.array_equal(poses[i], alone[i][k]), (i, k)
    finally:
        for m in sess:
            m.close()


def test_autotune_keeps_results(gpu_lib):
    """The autotuner times nine launch shapes (integration grid x raycast
    tile), then two more ICP shapes (the persistent launch on half its block
    share, the chained kernels) with the best of them, on the batch's own
    frames and keeps the fastest; the shapes change no result, so every
    frame matches the sessions stepped alone."""
    p = configs.preset("cfg1")
    p["sensor"].update(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5)
    p["tsdf"].update(voxel_size=0.01, truncation_distance=0.04, num_blocks=1 << 13,
                     num_buckets=1 << 14)
    n, nf = 3, 26
    seqs = [configs.sequence(p, seed=120 + i, n_frames=nf) for i in range(n)]
    t, g, b, s = configs.structs(p)
    precs = [abi.PRECISION_FP32, abi.PRECISION_MIXED, abi.PRECISION_MIXED_BAND]
    alone = []
    for i in range(n):
        with Session(t, g, b, s, precision=precs[i]) as m:
            m.set_pose(seqs[i].poses[0])
            alone.append([m.process(d)[0] for d in seqs[i].depth])
    sess = [Session(t, g, b, s, precision=precs[i]) for i in range(n)]
    try:
        for i, m in enumerate(sess):
            m.set_pose(seqs[i].poses[0])
        with Batch(sess) as bt:
            bt.autotune(2)
            assert not bt.tuning()[0]
            for k in range(nf):
                poses, _, _ = bt.process([q.depth[k] for q in seqs])
                for i in range(n):
                    assert np.array_equal(poses[i], alone[i][k]), (i, k)
            done, ctas, tile = bt.tuning()
            assert done and ctas in (592, 1184, 2368) and tile in (0, 1, 2)
    finally:
        for m in sess:
            m.close()
