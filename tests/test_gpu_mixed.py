"""The mixed-precision form (f16 sdf + u16 weight voxels, compensated FP32
normal equations, the fast raycast) against the plain FP32 path and the
FP64 oracle.  Bars: weights and colours exact, sdf within 1e-3 x truncation
of the FP32 path; raycast depth within one voxel where both paths hit;
tracked trajectory within 1 mm (ATE) of the plain path."""
import numpy as np
import pytest

from dynamap_b200 import abi, configs
from dynamap_b200.session import Session

pytestmark = pytest.mark.gpu


def small(name="cfg1", **over):
    p = configs.preset(name)
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    for k, v in over.items():
        p[k].update(v)
    return p


def sorted_blocks(coords, *arrs):
    o = np.lexsort((coords[:, 2], coords[:, 1], coords[:, 0]))
    return (coords[o],) + tuple(a[o] for a in arrs)


@pytest.mark.parametrize("rgb", [False, True])
def test_mixed_integration_close_to_fp32(gpu_lib, oracle, rgb):
    if rgb:
        p = small("cfg2")
        p["sensor"].update(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5)
    else:
        p = small()
    seq = configs.sequence(p, seed=12, n_frames=4)
    t, g, b, s = configs.structs(p)
    ovol = oracle.Volume(t)
    with Session(t, g, b, s, precision=abi.PRECISION_MIXED) as m:
        for k in range(4):
            pose = seq.poses[k].astype(np.float32)
            c = seq.rgb[k] if rgb else None
            m.integrate_with_pose(seq.depth[k], c, pose)
            d = oracle.depth_from_raw(seq.depth[k], s.depth_scaler)
            ovol.allocate(d, s, pose)
            ovol.integrate(d, c, s, pose)
        gc, grgbw, gsdf = sorted_blocks(*m.download_blocks())
    oc, orgbw, osdf = sorted_blocks(*ovol.download())
    np.testing.assert_array_equal(gc, oc)
    np.testing.assert_array_equal(grgbw[..., 3], orgbw[..., 3])
    if rgb:
        np.testing.assert_array_equal(grgbw[..., :3], orgbw[..., :3])
    assert np.max(np.abs(gsdf - osdf)) <= 1e-3 * t.truncation_distance


def test_mixed_raycast_close_to_fp32(gpu_lib, oracle):
    p = small()
    seq = configs.sequence(p, seed=13, n_frames=3)
    t, g, b, s = configs.structs(p)
    ovol = oracle.Volume(t)
    with Session(t, g, b, s, precision=abi.PRECISION_MIXED) as m:
        for k in range(3):
            pose = seq.poses[k].astype(np.float32)
            m.integrate_with_pose(seq.depth[k], None, pose)
            d = oracle.depth_from_raw(seq.depth[k], s.depth_scaler)
            ovol.allocate(d, s, pose)
            ovol.integrate(d, None, s, pose)
        pose = seq.poses[2].astype(np.float32)
        gd, _ = m.raycast(pose)
    od, _, _ = ovol.raycast(pose, s)
    hit_g, hit_o = gd < t.max_sensor_depth, od < t.max_sensor_depth
    assert np.mean(hit_g == hit_o) > 0.99
    both = hit_g & hit_o
    err = np.abs(gd[both] - od[both])
    assert np.quantile(err, 0.99) <= t.voxel_size
    assert np.median(err) <= 0.1 * t.voxel_size


def test_mixed_tracking_within_1mm_of_plain(gpu_lib):
    p = small()
    seq = configs.sequence(p, seed=14, n_frames=20)
    t, g, b, s = configs.structs(p)
    tracks = {}
    for prec in (abi.PRECISION_FP32, abi.PRECISION_MIXED):
        with Session(t, g, b, s, precision=prec) as m:
            m.set_pose(seq.poses[0])
            tracks[prec] = [m.process(seq.depth[k])[0] for k in range(len(seq.depth))]
    def ate(tr):
        return float(np.sqrt(np.mean([np.sum((a[:3, 3] - gt[:3, 3]) ** 2)
                                      for a, gt in zip(tr, seq.poses)])))
    a32, a16 = ate(tracks[abi.PRECISION_FP32]), ate(tracks[abi.PRECISION_MIXED])
    assert abs(a16 - a32) < 1e-3, (a32, a16)
    diff = max(np.linalg.norm(a[:3, 3] - b_[:3, 3])
               for a, b_ in zip(tracks[abi.PRECISION_FP32], tracks[abi.PRECISION_MIXED]))
    assert diff < 2e-3


def test_band_allocation_tracking_within_1mm_of_plain(gpu_lib):
    """Mixed form with band allocation: no carving of free space; the
    trajectory stays within 1 mm ATE of the FP32 drop-in and the map holds
    only blocks the carving form also allocates."""
    p = small()
    seq = configs.sequence(p, seed=14, n_frames=20)
    t, g, b, s = configs.structs(p)
    tracks, maps = {}, {}
    for prec in (abi.PRECISION_FP32, abi.PRECISION_MIXED_BAND):
        with Session(t, g, b, s, precision=prec) as m:
            m.set_pose(seq.poses[0])
            tracks[prec] = [m.process(seq.depth[k])[0] for k in range(len(seq.depth))]
            maps[prec] = m.download_blocks()[0]
    def ate(tr):
        return float(np.sqrt(np.mean([np.sum((a[:3, 3] - gt[:3, 3]) ** 2)
                                      for a, gt in zip(tr, seq.poses)])))
    a32, aband = ate(tracks[abi.PRECISION_FP32]), ate(tracks[abi.PRECISION_MIXED_BAND])
    assert abs(aband - a32) < 1e-3, (a32, aband)
    full = {tuple(c) for c in maps[abi.PRECISION_FP32]}
    band = {tuple(c) for c in maps[abi.PRECISION_MIXED_BAND]}
    assert len(band) < 0.7 * len(full)
    assert len(band - full) <= 0.01 * len(band)  # poses differ slightly: nearly a subset
