"""Workload presets: the five configurations the rigid path is measured on.

Each preset gives the sensor, TSDF, ICP and bilateral parameters and the
synthetic sequence that stands in for a recording (see scene.py).  Sizes
follow the configuration texts; where a text leaves a value open the choice
is written next to it.
"""
from __future__ import annotations

import math

from . import abi

COS_PI_10 = math.cos(math.pi / 10)


def _gn(iters, color_weight=0.0, dmin=0.15, dmax=3.0):
    return dict(lvl_iteration_num=iters, lvl_scale=[4, 2, 1], min_increment=1e-3,
                max_increment=0.3, regularization=0.02, huber_constant=0.3,
                color_weight=color_weight, icp_min_depth=dmin, icp_max_depth=dmax,
                normal_cos_thresh=COS_PI_10, mode=1, compose_left=0)


PRESETS = {
    # 50 frames 320x240, 8 mm voxels, trunc 4 voxels, 2^18 buckets x 10,
    # 3 levels with lvlIterationNum 10/5/4 (9/4/3 executed).
    "cfg1": dict(
        sensor=dict(rows=240, cols=320, fx=262.5, fy=262.5, cx=159.5, cy=119.5,
                    depth_scaler=1000.0),
        tsdf=dict(voxel_size=0.008, num_buckets=1 << 18, bucket_size=10,
                  num_blocks=1 << 17, block_size=8, max_sdf_weight=64,
                  truncation_distance=0.032, max_sensor_depth=3.0,
                  min_sensor_depth=0.15),
        gn=_gn([10, 5, 4]),
        bilateral=dict(diameter=8, sigma_i=10.0, sigma_s=1.0, enabled=1),
        seq=dict(n_frames=50, trans=0.005, rot=0.5, rgb=False, kind="cube"),
    ),
    # 500 frames 640x480 + RGB, 5 mm voxels (trunc 4 voxels), 2^20 buckets,
    # photometric weight 0.1.
    "cfg2": dict(
        sensor=dict(rows=480, cols=640, fx=525.0, fy=525.0, cx=319.5, cy=239.5,
                    depth_scaler=1000.0),
        tsdf=dict(voxel_size=0.005, num_buckets=1 << 20, bucket_size=10,
                  num_blocks=1 << 19, block_size=8, max_sdf_weight=64,
                  truncation_distance=0.02, max_sensor_depth=3.0,
                  min_sensor_depth=0.15),
        gn=_gn([10, 5, 4], color_weight=0.1),
        bilateral=dict(diameter=8, sigma_i=10.0, sigma_s=1.0, enabled=1),
        seq=dict(n_frames=500, trans=0.01, rot=1.0, rgb=True, kind="cube"),
    ),
    # Large-scene stress: 1280x720 depth + RGB through the 8 x 8 x 3 m room
    # (walls, 40 primitives), 4 mm voxels, 2^23 buckets, 2^22 blocks,
    # ranges to 8 m; run in the mixed form with band allocation, batched with
    # eight 640x480 sessions (cfg2 sensor, cube scenes).
    "cfg5": dict(
        sensor=dict(rows=720, cols=1280, fx=910.0, fy=910.0, cx=639.5, cy=359.5,
                    depth_scaler=1000.0),
        tsdf=dict(voxel_size=0.004, num_buckets=1 << 23, bucket_size=10,
                  num_blocks=1 << 22, block_size=8, max_sdf_weight=64,
                  truncation_distance=0.016, max_sensor_depth=8.0,
                  min_sensor_depth=0.15),
        gn=_gn([10, 5, 4], color_weight=0.1, dmax=8.0),
        bilateral=dict(diameter=8, sigma_i=10.0, sigma_s=1.0, enabled=1),
        seq=dict(n_frames=2000, trans=0.01, rot=1.0, rgb=True, kind="room", max_range=8.0),
    ),
}


def session_mix(n_sessions: int = 32, n_frames: int = 200, base_seed: int = 100):
    """The batched configuration: n independent sessions, resolutions
    160x120 / 320x240 / 640x480 in the ratio 1:2:1, voxel sizes 5-10 mm,
    2^18-2^20 buckets, each with its own seeded scene and trajectory.
    Returns a list of (name, preset dict, seed)."""
    out = []
    kinds = ["s160", "s320", "s320", "s640"]
    for i in range(n_sessions):
        k = kinds[i % 4]
        if k == "s160":
            sensor = dict(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5,
                          depth_scaler=1000.0)
            tsdf = dict(voxel_size=0.01, num_buckets=1 << 18, num_blocks=1 << 14)
        elif k == "s320":
            sensor = dict(rows=240, cols=320, fx=262.5, fy=262.5, cx=159.5, cy=119.5,
                          depth_scaler=1000.0)
            tsdf = dict(voxel_size=0.008, num_buckets=1 << 19, num_blocks=1 << 16)
        else:
            sensor = dict(rows=480, cols=640, fx=525.0, fy=525.0, cx=319.5, cy=239.5,
                          depth_scaler=1000.0)
            tsdf = dict(voxel_size=0.005, num_buckets=1 << 20, num_blocks=1 << 18)
        tsdf.update(bucket_size=10, block_size=8, max_sdf_weight=64,
                    truncation_distance=4 * tsdf["voxel_size"], max_sensor_depth=3.0,
                    min_sensor_depth=0.15)
        p = dict(sensor=sensor, tsdf=tsdf, gn=_gn([10, 5, 4]),
                 bilateral=dict(diameter=8, sigma_i=10.0, sigma_s=1.0, enabled=1),
                 seq=dict(n_frames=n_frames, trans=0.005, rot=0.5, rgb=False, kind="cube"))
        out.append((k, p, base_seed + i))
    return out


# The serving configuration: sessions arrive as a Poisson process (rate
# 4/s), each streams depth at 30 Hz for U[5, 60] s; resolutions 320x240 /
# 640x480 / 1280x720 (ratio 2:2:1); each session's hash table holds 84 /
# 168 / 336 MB of entries (2^19 / 2^20 / 2^21 buckets x 10); mixed
# precision; a 150 GB device budget.
SERVING = dict(rate_per_s=4.0, duration_s=(5.0, 60.0), fps=30.0, budget_gb=150.0,
               kinds=["s320", "s320", "s640", "s640", "s1280"])


def serving_kind(kind: str, n_frames: int = 24):
    """Preset of one serving session kind."""
    if kind == "s320":
        sensor = dict(rows=240, cols=320, fx=262.5, fy=262.5, cx=159.5, cy=119.5,
                      depth_scaler=1000.0)
        tsdf = dict(voxel_size=0.008, num_buckets=1 << 19, num_blocks=1 << 16)
    elif kind == "s640":
        sensor = dict(rows=480, cols=640, fx=525.0, fy=525.0, cx=319.5, cy=239.5,
                      depth_scaler=1000.0)
        tsdf = dict(voxel_size=0.005, num_buckets=1 << 20, num_blocks=1 << 18)
    else:
        sensor = dict(rows=720, cols=1280, fx=910.0, fy=910.0, cx=639.5, cy=359.5,
                      depth_scaler=1000.0)
        tsdf = dict(voxel_size=0.004, num_buckets=1 << 21, num_blocks=1 << 19)
    tsdf.update(bucket_size=10, block_size=8, max_sdf_weight=64,
                truncation_distance=4 * tsdf["voxel_size"], max_sensor_depth=3.0,
                min_sensor_depth=0.15)
    return dict(sensor=sensor, tsdf=tsdf, gn=_gn([10, 5, 4]),
                bilateral=dict(diameter=8, sigma_i=10.0, sigma_s=1.0, enabled=1),
                seq=dict(n_frames=n_frames, trans=0.005, rot=0.5, rgb=False, kind="cube"))


def preset(name: str, **over):
    p = {k: (dict(v) if isinstance(v, dict) else v) for k, v in PRESETS[name].items()}
    for k, v in over.items():
        p[k].update(v)
    return p


def structs(p: dict):
    return abi.make_params(p["sensor"], p["tsdf"], p["gn"], p["bilateral"])


def sequence(p: dict, seed: int = 1, n_frames: int | None = None, noise: bool = True):
    from . import scene
    s, q = p["sensor"], p["seq"]
    return scene.make_sequence(
        seed, n_frames if n_frames is not None else q["n_frames"], s["rows"], s["cols"],
        s["fx"], s["fy"], s["cx"], s["cy"], q["trans"], q["rot"], with_rgb=q["rgb"],
        kind=q["kind"], noise=noise, depth_scaler=s["depth_scaler"],
        max_range=q.get("max_range", 4.0))
