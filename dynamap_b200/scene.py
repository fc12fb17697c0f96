"""Seeded synthetic RGB-D sequences for the rigid mapping path.

The reference is exercised on TUM/NUIM recordings, which are not available
here; these analytic scenes stand in for them.  A scene is a floor plane,
axis-aligned boxes and spheres inside a cube (or a walled room), seen by a
pinhole camera on a smooth seeded trajectory.  Depth is the exact z-depth of
the first surface hit plus Gaussian noise with sigma(z) = 0.0012 +
0.0019 (z - 0.4)^2 metres, quantised to sensor units; pixels that hit nothing
within range are 0.  Colour is a per-primitive base colour modulated by 3-D
Perlin noise (albedo only, no shading).

World axes: y points down (the camera convention of the reference's pinhole
model, include/utils/utils.h:104-119), so the floor is the plane y = floor_y
with the scene above it (smaller y).  The scene is placed away from the world
origin and every camera looks away from it.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Sphere:
    center: np.ndarray
    radius: float
    color: np.ndarray


@dataclasses.dataclass
class Box:
    lo: np.ndarray
    hi: np.ndarray
    color: np.ndarray
    inside: bool = False  # True: a room; rays hit the inner walls


@dataclasses.dataclass
class Scene:
    floor_y: float
    floor_lo: np.ndarray  # xz extent of the floor
    floor_hi: np.ndarray
    floor_color: np.ndarray
    boxes: list
    spheres: list
    center: np.ndarray
    perm: np.ndarray      # Perlin permutation table (seeded)


def make_scene(seed: int, kind: str = "cube") -> Scene:
    """kind 'cube': floor, 1 box, 3 spheres (r 0.1-0.3 m) in a 2 m cube.
    kind 'room': 8 x 8 x 3 m room with walls and 40 primitives."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(256).astype(np.int64)
    perm = np.concatenate([perm, perm])
    if kind == "cube":
        c = np.array([3.0, 0.0, 3.0])
        floor_y = 1.0
        boxes, spheres = [], []
        sz = rng.uniform(0.3, 0.6, size=3)
        bxz = c[[0, 2]] + rng.uniform(-0.45, 0.45, size=2)
        lo = np.array([bxz[0] - sz[0] / 2, floor_y - sz[1], bxz[1] - sz[2] / 2])
        hi = np.array([bxz[0] + sz[0] / 2, floor_y, bxz[1] + sz[2] / 2])
        boxes.append(Box(lo, hi, rng.uniform(0.2, 0.9, size=3)))
        for _ in range(3):
            r = rng.uniform(0.1, 0.3)
            xz = c[[0, 2]] + rng.uniform(-0.6, 0.6, size=2)
            y = floor_y - r - rng.uniform(0.0, 0.6)
            spheres.append(Sphere(np.array([xz[0], y, xz[1]]), r,
                                  rng.uniform(0.2, 0.9, size=3)))
        return Scene(floor_y, c[[0, 2]] - 2.5, c[[0, 2]] + 2.5,
                     rng.uniform(0.3, 0.8, size=3), boxes, spheres, c, perm)
    if kind == "room":
        c = np.array([6.0, 0.0, 6.0])
        floor_y = 1.5
        lo = np.array([c[0] - 4.0, floor_y - 3.0, c[2] - 4.0])
        hi = np.array([c[0] + 4.0, floor_y, c[2] + 4.0])
        boxes = [Box(lo, hi, rng.uniform(0.4, 0.8, size=3), inside=True)]
        spheres = []
        for _ in range(20):
            sz = rng.uniform(0.2, 0.9, size=3)
            xz = c[[0, 2]] + rng.uniform(-3.3, 3.3, size=2)
            blo = np.array([xz[0] - sz[0] / 2, floor_y - sz[1], xz[1] - sz[2] / 2])
            bhi = np.array([xz[0] + sz[0] / 2, floor_y, xz[1] + sz[2] / 2])
            boxes.append(Box(blo, bhi, rng.uniform(0.2, 0.9, size=3)))
        for _ in range(20):
            r = rng.uniform(0.1, 0.4)
            xz = c[[0, 2]] + rng.uniform(-3.5, 3.5, size=2)
            y = floor_y - r - rng.uniform(0.0, 1.5)
            spheres.append(Sphere(np.array([xz[0], y, xz[1]]), r,
                                  rng.uniform(0.2, 0.9, size=3)))
        return Scene(floor_y, lo[[0, 2]], hi[[0, 2]],
                     rng.uniform(0.3, 0.8, size=3), boxes, spheres, c, perm)
    raise ValueError(kind)


def look_at(pos: np.ndarray, target: np.ndarray) -> np.ndarray:
    """Camera-to-world 4x4 (float64) with z forward, y down, x right."""
    z = target - pos
    z = z / np.linalg.norm(z)
    down = np.array([0.0, 1.0, 0.0])
    x = np.cross(down, z)
    x = x / np.linalg.norm(x)
    y = np.cross(z, x)
    T = np.eye(4)
    T[:3, 0], T[:3, 1], T[:3, 2], T[:3, 3] = x, y, z, pos
    return T


def trajectory(scene: Scene, n_frames: int, seed: int, trans_per_frame: float,
               rot_per_frame_deg: float, radius: float = 1.6,
               height: float = 0.2) -> np.ndarray:
    """n_frames camera-to-world poses (n, 4, 4) float64.

    The camera sweeps back and forth on an arc around the scene centre that
    keeps the world origin behind it, looking at a point that wanders slowly
    around the centre.  The sweep amplitude and the wander amplitude are
    scaled so that the mean translation per frame is trans_per_frame and the
    mean rotation per frame is rot_per_frame_deg."""
    rng = np.random.default_rng(seed + 7919)
    c = scene.center
    th0 = math.radians(225.0)
    ph = rng.uniform(0, 2 * math.pi, size=6)
    k = np.arange(n_frames, dtype=np.float64)
    max_span = math.radians(40.0)
    # the sweep's period follows from the motion per frame alone, so that a
    # short sequence is the start of a long one (same motion per frame)
    period = max(4.0 * radius * max_span / max(trans_per_frame, 1e-9), 8.0)
    pw = 60.0
    wander = np.stack([np.sin(2 * math.pi * k / pw + ph[2]),
                       0.5 * np.sin(2 * math.pi * k / (pw * 1.3) + ph[3]),
                       np.sin(2 * math.pi * k / (pw * 0.9) + ph[4])], axis=1)

    def build(span, amp):
        theta = th0 + span * np.sin(2 * math.pi * k / period + ph[0])
        cam_y = c[1] - height + 0.05 * np.sin(2 * math.pi * k / (period * 0.7) + ph[1])
        pos = np.stack([c[0] + radius * np.cos(theta), cam_y,
                        c[2] + radius * np.sin(theta)], axis=1)
        targets = c[None, :] + radius * amp * wander + np.array([0.0, 0.25, 0.0])
        return np.stack([look_at(pos[i], targets[i]) for i in range(n_frames)])

    span, amp = max_span, 0.02
    if n_frames < 2:
        return build(span, amp)
    for _ in range(4):
        m = motion_stats(build(span, amp))
        if m["trans_m"] > 0:
            span = min(span * trans_per_frame / m["trans_m"], math.radians(60.0))
        m = motion_stats(build(span, amp))
        if m["rot_deg"] > 0:
            amp = min(max(amp * rot_per_frame_deg / m["rot_deg"], 0.0), 0.5)
    return build(span, amp)


def motion_stats(poses: np.ndarray) -> dict:
    """Mean translation (m) and rotation (deg) between consecutive poses."""
    if len(poses) < 2:
        return {"trans_m": 0.0, "rot_deg": 0.0}
    t = np.linalg.norm(np.diff(poses[:, :3, 3], axis=0), axis=1)
    rots = []
    for a, b in zip(poses[:-1], poses[1:]):
        R = a[:3, :3].T @ b[:3, :3]
        rots.append(math.degrees(math.acos(max(-1.0, min(1.0, (np.trace(R) - 1) / 2)))))
    return {"trans_m": float(np.mean(t)), "rot_deg": float(np.mean(rots))}


def _fade(t):
    return t * t * t * (t * (t * 6 - 15) + 10)


_GRAD = np.array([[1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0],
                  [1, 0, 1], [-1, 0, 1], [1, 0, -1], [-1, 0, -1],
                  [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1],
                  [1, 1, 0], [0, -1, 1], [-1, 1, 0], [0, -1, -1]], dtype=np.float64)


def perlin3(p: np.ndarray, perm: np.ndarray) -> np.ndarray:
    """Improved Perlin gradient noise (Perlin 2002) at points p (n, 3);
    values roughly in [-1, 1]."""
    pi = np.floor(p).astype(np.int64)
    pf = p - pi
    pi &= 255
    u, v, w = _fade(pf[:, 0]), _fade(pf[:, 1]), _fade(pf[:, 2])

    def g(ix, iy, iz, fx, fy, fz):
        h = perm[perm[perm[ix] + iy] + iz] & 15
        gv = _GRAD[h]
        return gv[:, 0] * fx + gv[:, 1] * fy + gv[:, 2] * fz

    X, Y, Z = pi[:, 0], pi[:, 1], pi[:, 2]
    x, y, z = pf[:, 0], pf[:, 1], pf[:, 2]
    n000 = g(X, Y, Z, x, y, z)
    n100 = g(X + 1, Y, Z, x - 1, y, z)
    n010 = g(X, Y + 1, Z, x, y - 1, z)
    n110 = g(X + 1, Y + 1, Z, x - 1, y - 1, z)
    n001 = g(X, Y, Z + 1, x, y, z - 1)
    n101 = g(X + 1, Y, Z + 1, x - 1, y, z - 1)
    n011 = g(X, Y + 1, Z + 1, x, y - 1, z - 1)
    n111 = g(X + 1, Y + 1, Z + 1, x - 1, y - 1, z - 1)
    nx00 = n000 + u * (n100 - n000)
    nx10 = n010 + u * (n110 - n010)
    nx01 = n001 + u * (n101 - n001)
    nx11 = n011 + u * (n111 - n011)
    nxy0 = nx00 + v * (nx10 - nx00)
    nxy1 = nx01 + v * (nx11 - nx01)
    return nxy0 + w * (nxy1 - nxy0)


def render(scene: Scene, pose: np.ndarray, rows: int, cols: int, fx: float,
           fy: float, cx: float, cy: float, rng: np.random.Generator | None,
           depth_scaler: float = 1000.0, max_range: float = 4.0,
           min_range: float = 0.1, with_rgb: bool = False):
    """Ray-cast one frame.  Returns (depth uint16 (rows, cols), rgb uint8
    (rows, cols, 3) or None).  rng None = noise-free depth."""
    u, v = np.meshgrid(np.arange(cols, dtype=np.float64),
                       np.arange(rows, dtype=np.float64))
    dcam = np.stack([(u - cx) / fx, (v - cy) / fy, np.ones_like(u)], -1).reshape(-1, 3)
    R, o = pose[:3, :3], pose[:3, 3]
    d = dcam @ R.T  # world direction with camera z component 1 => t = z-depth
    n = d.shape[0]
    tbest = np.full(n, np.inf)
    prim = np.full(n, -1, dtype=np.int64)
    # floor
    with np.errstate(divide="ignore", invalid="ignore"):
        t = (scene.floor_y - o[1]) / d[:, 1]
    hit = o[None, :] + t[:, None] * d
    ok = (t > 0) & (hit[:, 0] >= scene.floor_lo[0]) & (hit[:, 0] <= scene.floor_hi[0]) \
        & (hit[:, 2] >= scene.floor_lo[1]) & (hit[:, 2] <= scene.floor_hi[1])
    upd = ok & (t < tbest)
    tbest[upd], prim[upd] = t[upd], 0
    # boxes (slab method)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / d
    for bi, b in enumerate(scene.boxes):
        t1 = (b.lo[None, :] - o[None, :]) * inv
        t2 = (b.hi[None, :] - o[None, :]) * inv
        tmin = np.nanmax(np.minimum(t1, t2), axis=1)
        tmax = np.nanmin(np.maximum(t1, t2), axis=1)
        if b.inside:
            t = tmax
            ok = (tmax > 0) & (tmax >= tmin)
        else:
            t = tmin
            ok = (tmin > 0) & (tmax >= tmin)
        upd = ok & (t < tbest)
        tbest[upd], prim[upd] = t[upd], 1 + bi
    # spheres
    for si, s in enumerate(scene.spheres):
        oc = o - s.center
        a = np.einsum("ij,ij->i", d, d)
        bq = 2.0 * (d @ oc)
        cq = float(oc @ oc) - s.radius ** 2
        disc = bq * bq - 4 * a * cq
        ok = disc >= 0
        sq = np.sqrt(np.where(ok, disc, 0.0))
        t = (-bq - sq) / (2 * a)
        ok &= t > 0
        upd = ok & (t < tbest)
        tbest[upd], prim[upd] = t[upd], 1 + len(scene.boxes) + si
    valid = np.isfinite(tbest) & (tbest >= min_range) & (tbest <= max_range)
    z = np.where(valid, tbest, 0.0)
    if rng is not None:
        sigma = 0.0012 + 0.0019 * (z - 0.4) ** 2
        noise = rng.standard_normal(n)
        z = np.where(valid, z + sigma * noise, 0.0)
    raw = np.where(valid, np.rint(z * depth_scaler), 0.0)
    raw = np.clip(raw, 0, 65535).astype(np.uint16).reshape(rows, cols)
    rgb = None
    if with_rgb:
        hit = o[None, :] + np.where(np.isfinite(tbest), tbest, 0.0)[:, None] * d
        cols_tab = [scene.floor_color] + [b.color for b in scene.boxes] + \
                   [s.color for s in scene.spheres]
        base = np.stack(cols_tab)[np.maximum(prim, 0)]
        tex = perlin3(hit * 6.0, scene.perm)
        tex2 = perlin3(hit * 23.0 + 17.0, scene.perm)
        shade = np.clip(0.65 + 0.35 * tex + 0.15 * tex2, 0.0, 1.2)
        col = np.clip(base * shade[:, None], 0.0, 1.0) * 255.0
        col[prim < 0] = 0.0
        rgb = np.rint(col).astype(np.uint8).reshape(rows, cols, 3)
    return raw, rgb


@dataclasses.dataclass
class Sequence:
    depth: np.ndarray      # (n, rows, cols) uint16
    rgb: np.ndarray | None  # (n, rows, cols, 3) uint8
    poses: np.ndarray      # (n, 4, 4) float64 ground truth, camera-to-world
    sensor: dict           # rows, cols, fx, fy, cx, cy, depth_scaler
    seed: int
    motion: dict


def make_sequence(seed: int, n_frames: int, rows: int, cols: int, fx: float,
                  fy: float, cx: float, cy: float, trans_per_frame: float,
                  rot_per_frame_deg: float, with_rgb: bool = False,
                  kind: str = "cube", noise: bool = True,
                  depth_scaler: float = 1000.0, max_range: float = 4.0,
                  radius: float = 1.6) -> Sequence:
    scene = make_scene(seed, kind)
    poses = trajectory(scene, n_frames, seed, trans_per_frame,
                       rot_per_frame_deg, radius=radius)
    rng = np.random.default_rng(seed + 104729) if noise else None
    depth = np.zeros((n_frames, rows, cols), np.uint16)
    rgb = np.zeros((n_frames, rows, cols, 3), np.uint8) if with_rgb else None
    for i in range(n_frames):
        d, c = render(scene, poses[i], rows, cols, fx, fy, cx, cy, rng,
                      depth_scaler=depth_scaler, max_range=max_range,
                      with_rgb=with_rgb)
        depth[i] = d
        if with_rgb:
            rgb[i] = c
    sensor = dict(rows=rows, cols=cols, fx=fx, fy=fy, cx=cx, cy=cy,
                  depth_scaler=depth_scaler)
    return Sequence(depth, rgb, poses, sensor, seed, motion_stats(poses))
