"""ctypes binding of the CPU oracle (test infrastructure only).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the
checker; the product (dynamap_b200) never imports it.  Build the library with
`make -C oracle` (or __graft_entry__.build()).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from dynamap_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libdynoracle.so")

C_NEW, C_BUCKET_FULL, C_HEAP, C_DDA, C_VIS, C_REHASH, C_RC, C_UNIQUE = range(8)

_lib = None
P = C.POINTER
_vp = C.c_void_p


def build() -> None:
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        sig = {
            "dyo_set_threads": (None, [C.c_int]),
            "dyo_get_threads": (C.c_int, []),
            "dyo_hash": (C.c_int32, [C.c_int32] * 5),
            "dyo_level_sensor": (None, [P(abi.Sensor), C.c_int32, P(abi.Sensor)]),
            "dyo_dda_blocks": (C.c_int32, [P(C.c_float), P(C.c_float), C.c_float, C.c_float,
                                           C.c_int32, P(C.c_int32), C.c_int32]),
            "dyo_merge_voxel": (None, [P(C.c_uint8), P(C.c_float), C.c_float, P(C.c_uint8),
                                       C.c_int32, C.c_int32]),
            "dyo_depth_from_raw": (None, [_vp, C.c_int64, C.c_float, _vp]),
            "dyo_bilateral": (None, [_vp, _vp, C.c_int32, C.c_int32, P(abi.BilateralParams)]),
            "dyo_downsample_depth": (None, [_vp, C.c_int32, C.c_int32, _vp]),
            "dyo_intensity": (None, [_vp, C.c_int64, _vp]),
            "dyo_downsample_intensity": (None, [_vp, C.c_int32, C.c_int32, _vp]),
            "dyo_maps": (None, [_vp, P(abi.Sensor), _vp, _vp]),
            "dyo_icp_normal_equations": (None, [_vp] * 6 + [P(abi.Sensor), P(abi.GnParams),
                                                           P(C.c_float), P(C.c_double)]),
            "dyo_icp_normal_equations_refsum": (C.c_int64, [_vp] * 6 + [
                P(abi.Sensor), P(abi.GnParams), P(C.c_float), P(C.c_float), P(C.c_float)]),
            "dyo_gn_solve_refsum": (None, [_vp] * 4 + [P(abi.Sensor), P(abi.GnParams),
                                                       P(C.c_double)]),
            "dyo_inverse4": (None, [P(C.c_float), P(C.c_float)]),
            "dyo_se3_exp": (None, [P(C.c_double), P(C.c_double)]),
            "dyo_ldlt_solve6": (C.c_int, [P(C.c_double), P(C.c_double), P(C.c_double)]),
            "dyo_volume_create": (_vp, [P(abi.TsdfParams), C.c_int32]),
            "dyo_volume_destroy": (None, [_vp]),
            "dyo_volume_allocate": (None, [_vp, _vp, P(abi.Sensor), P(C.c_float), P(C.c_int64)]),
            "dyo_volume_integrate": (None, [_vp, _vp, _vp, P(abi.Sensor), P(C.c_float), P(C.c_int64)]),
            "dyo_volume_raycast": (None, [_vp, P(C.c_float), P(abi.Sensor), _vp, _vp, P(C.c_int64)]),
            "dyo_volume_num_blocks": (C.c_int64, [_vp]),
            "dyo_mesh_vertices": (C.c_int64, [_vp, P(C.c_float), P(C.c_float), _vp, C.c_int64]),
            "dyo_mesh_triangles": (C.c_int64, [_vp, P(C.c_float), P(C.c_float), _vp, C.c_int64]),
            "dyo_volume_download": (C.c_int64, [_vp, _vp, _vp, _vp, C.c_int64]),
            "dyo_volume_upload": (C.c_int64, [_vp, _vp, _vp, _vp, C.c_int64]),
            "dyo_session_create": (_vp, [P(abi.TsdfParams), P(abi.GnParams),
                                         P(abi.BilateralParams), P(abi.Sensor), C.c_int32]),
            "dyo_session_destroy": (None, [_vp]),
            "dyo_session_set_pose": (None, [_vp, P(C.c_float)]),
            "dyo_session_get_pose": (None, [_vp, P(C.c_float)]),
            "dyo_session_get_pose_f64": (None, [_vp, P(C.c_double)]),
            "dyo_session_frame": (None, [_vp, _vp, _vp, P(C.c_float), P(abi.FrameStats)]),
            "dyo_session_integrate_with_pose": (None, [_vp, _vp, _vp, P(C.c_float)]),
            "dyo_session_volume": (_vp, [_vp]),
            "dyo_session_image": (C.c_int, [_vp, C.c_int32, C.c_int32, _vp, C.c_int64]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_vp)


def fptr(a: np.ndarray):
    return a.ctypes.data_as(P(C.c_float))


def dda_blocks(start, point, trunc: float, block_size: float, cap: int = 100000):
    """Visited block coordinates (k, 3) and whether the ray finished."""
    st = (C.c_float * 3)(*[float(x) for x in start])
    pt = (C.c_float * 3)(*[float(x) for x in point])
    mx = 4096
    out = np.empty((mx, 3), np.int32)
    n = lib().dyo_dda_blocks(st, pt, trunc, block_size, cap,
                             out.ctypes.data_as(P(C.c_int32)), mx)
    k = abs(n)
    return out[:min(k, mx)].copy(), n >= 0


def merge_voxel(rgbw, sdf: float, new_sdf: float, new_rgb, new_w: int, max_w: int):
    a = (C.c_uint8 * 4)(*rgbw)
    sd = C.c_float(sdf)
    nc = (C.c_uint8 * 3)(*new_rgb)
    lib().dyo_merge_voxel(a, C.byref(sd), new_sdf, nc, new_w, max_w)
    return list(a), sd.value


def set_threads(n: int) -> None:
    lib().dyo_set_threads(int(n))


def level_sensor(s: abi.Sensor, scale: int) -> abi.Sensor:
    o = abi.Sensor()
    lib().dyo_level_sensor(C.byref(s), scale, C.byref(o))
    return o


def depth_from_raw(raw: np.ndarray, scaler: float) -> np.ndarray:
    raw = np.ascontiguousarray(raw, np.uint16)
    out = np.empty(raw.shape, np.float32)
    lib().dyo_depth_from_raw(ptr(raw), raw.size, scaler, ptr(out))
    return out


def bilateral(d: np.ndarray, p: abi.BilateralParams) -> np.ndarray:
    d = np.ascontiguousarray(d, np.float32)
    out = np.empty_like(d)
    lib().dyo_bilateral(ptr(d), ptr(out), d.shape[0], d.shape[1], C.byref(p))
    return out


def downsample_depth(d: np.ndarray) -> np.ndarray:
    d = np.ascontiguousarray(d, np.float32)
    out = np.empty((d.shape[0] // 2, d.shape[1] // 2), np.float32)
    lib().dyo_downsample_depth(ptr(d), d.shape[0], d.shape[1], ptr(out))
    return out


def intensity(rgb: np.ndarray) -> np.ndarray:
    rgb = np.ascontiguousarray(rgb, np.uint8)
    out = np.empty(rgb.shape[:2], np.float32)
    lib().dyo_intensity(ptr(rgb), out.size, ptr(out))
    return out


def downsample_intensity(i: np.ndarray) -> np.ndarray:
    i = np.ascontiguousarray(i, np.float32)
    out = np.empty((i.shape[0] // 2, i.shape[1] // 2), np.float32)
    lib().dyo_downsample_intensity(ptr(i), i.shape[0], i.shape[1], ptr(out))
    return out


def maps(d: np.ndarray, s: abi.Sensor):
    d = np.ascontiguousarray(d, np.float32)
    v = np.empty(d.shape + (4,), np.float32)
    n = np.empty(d.shape + (4,), np.float32)
    lib().dyo_maps(ptr(d), C.byref(s), ptr(v), ptr(n))
    return v, n


def icp_normal_equations(sd, sn, si, td, tn, ti, s, g, T) -> np.ndarray:
    out = np.zeros(29, np.float64)
    T = np.ascontiguousarray(T, np.float32).reshape(16)
    args = [np.ascontiguousarray(a, np.float32) if a is not None else None
            for a in (sd, sn, si, td, tn, ti)]
    lib().dyo_icp_normal_equations(*[ptr(a) for a in args], C.byref(s), C.byref(g),
                                   fptr(T), out.ctypes.data_as(P(C.c_double)))
    return out


def icp_normal_equations_refsum(sd, sn, si, td, tn, ti, s, g, T):
    """(A float32 [36], acc_b float32 [6], pixel count) summed as the
    reference's buildNLSKernel sums them on one thread."""
    A = np.zeros(36, np.float32)
    b = np.zeros(6, np.float32)
    T = np.ascontiguousarray(T, np.float32).reshape(16)
    args = [np.ascontiguousarray(a, np.float32) if a is not None else None
            for a in (sd, sn, si, td, tn, ti)]
    n = lib().dyo_icp_normal_equations_refsum(*[ptr(a) for a in args], C.byref(s), C.byref(g),
                                              fptr(T), fptr(A), fptr(b))
    return A, b, int(n)


def gn_solve_refsum(sd, sn, td, tn, s, g) -> np.ndarray:
    """xi of gnSolver::solve's loop on full-resolution images, the normal
    equations summed as the reference sums them."""
    inc = np.zeros(6, np.float64)
    args = [np.ascontiguousarray(a, np.float32) for a in (sd, sn, td, tn)]
    lib().dyo_gn_solve_refsum(*[ptr(a) for a in args], C.byref(s), C.byref(g),
                              inc.ctypes.data_as(P(C.c_double)))
    return inc


def inverse4(m: np.ndarray) -> np.ndarray:
    m = np.ascontiguousarray(m, np.float32).reshape(16)
    out = np.empty(16, np.float32)
    lib().dyo_inverse4(fptr(m), fptr(out))
    return out.reshape(4, 4)


def se3_exp(xi) -> np.ndarray:
    xi = np.ascontiguousarray(xi, np.float64)
    out = np.empty(16, np.float64)
    lib().dyo_se3_exp(xi.ctypes.data_as(P(C.c_double)), out.ctypes.data_as(P(C.c_double)))
    return out.reshape(4, 4)


class Volume:
    """Oracle TSDF volume (fp64=True: the FP64 oracle)."""

    def __init__(self, tsdf: abi.TsdfParams, fp64: bool = False, handle=None, owner=None):
        self.fp64 = fp64
        self.tsdf = tsdf
        self._owner = owner
        self.h = handle if handle is not None else lib().dyo_volume_create(C.byref(tsdf), int(fp64))
        self._own = handle is None

    def __del__(self):
        if getattr(self, "_own", False) and self.h:
            lib().dyo_volume_destroy(self.h)
            self.h = None

    def allocate(self, depth, sensor, pose) -> np.ndarray:
        c = np.zeros(8, np.int64)
        d = np.ascontiguousarray(depth, np.float32)
        P16 = np.ascontiguousarray(pose, np.float32).reshape(16)
        lib().dyo_volume_allocate(self.h, ptr(d), C.byref(sensor), fptr(P16),
                                  c.ctypes.data_as(P(C.c_int64)))
        return c

    def integrate(self, depth, rgb, sensor, pose) -> np.ndarray:
        c = np.zeros(8, np.int64)
        d = np.ascontiguousarray(depth, np.float32)
        r = None if rgb is None else np.ascontiguousarray(rgb, np.uint8)
        P16 = np.ascontiguousarray(pose, np.float32).reshape(16)
        lib().dyo_volume_integrate(self.h, ptr(d), ptr(r), C.byref(sensor), fptr(P16),
                                   c.ctypes.data_as(P(C.c_int64)))
        return c

    def raycast(self, pose, sensor, rgb: bool = False):
        c = np.zeros(8, np.int64)
        n = sensor.rows * sensor.cols
        d = np.empty((sensor.rows, sensor.cols), np.float32)
        r = np.empty((sensor.rows, sensor.cols, 3), np.uint8) if rgb else None
        P16 = np.ascontiguousarray(pose, np.float32).reshape(16)
        lib().dyo_volume_raycast(self.h, fptr(P16), C.byref(sensor), ptr(d), ptr(r),
                                 c.ctypes.data_as(P(C.c_int64)))
        return d, r, c

    def mesh_vertices(self, lo, hi) -> np.ndarray:
        """[n, 6] {x, y, z, r, g, b} of the vertices MeshExtractor's
        triangles use over the box [lo, hi]."""
        lo_c = (C.c_float * 3)(*[float(x) for x in lo])
        hi_c = (C.c_float * 3)(*[float(x) for x in hi])
        n = lib().dyo_mesh_vertices(self.h, lo_c, hi_c, None, 0)
        out = np.zeros((max(n, 0), 6), np.float32)
        if n > 0:
            lib().dyo_mesh_vertices(self.h, lo_c, hi_c, ptr(out), n)
        return out

    def mesh_triangles(self, lo, hi) -> np.ndarray:
        """[n, 3, 6] triangles of the same cells with this project's
        marching-cubes table."""
        lo_c = (C.c_float * 3)(*[float(x) for x in lo])
        hi_c = (C.c_float * 3)(*[float(x) for x in hi])
        n = lib().dyo_mesh_triangles(self.h, lo_c, hi_c, None, 0)
        out = np.zeros((max(n, 0), 3, 6), np.float32)
        if n > 0:
            lib().dyo_mesh_triangles(self.h, lo_c, hi_c, ptr(out), n)
        return out

    def num_blocks(self) -> int:
        return int(lib().dyo_volume_num_blocks(self.h))

    def upload(self, coords, rgbw, sdf) -> int:
        """Blocks [n, 3] with voxels rgbw [n, 512, 4] u8 and sdf [n, 512]
        (FP32 volumes); returns the blocks placed."""
        coords = np.ascontiguousarray(coords, np.int32)
        rgbw = np.ascontiguousarray(rgbw, np.uint8)
        sdf = np.ascontiguousarray(sdf, np.float32)
        n = len(coords)
        assert rgbw.shape == (n, 512, 4) and sdf.shape == (n, 512)
        return int(lib().dyo_volume_upload(self.h, ptr(coords), ptr(rgbw), ptr(sdf), n))

    def download(self):
        n = self.num_blocks()
        coords = np.empty((n, 3), np.int32)
        rgbw = np.empty((n, 512, 4), np.uint8)
        sdf = np.empty((n, 512), np.float64 if self.fp64 else np.float32)
        lib().dyo_volume_download(self.h, ptr(coords), ptr(rgbw), ptr(sdf), n)
        return coords, rgbw, sdf


class Session:
    """Oracle per-frame pipeline (builder::buildModelLS with the fixes)."""

    def __init__(self, tsdf, gn, bil, sensor, fp64: bool = False):
        self.sensor = sensor
        self.fp64 = fp64
        self.h = lib().dyo_session_create(C.byref(tsdf), C.byref(gn), C.byref(bil),
                                          C.byref(sensor), int(fp64))
        self.volume = Volume(tsdf, fp64, handle=lib().dyo_session_volume(self.h), owner=self)

    def __del__(self):
        if getattr(self, "h", None):
            lib().dyo_session_destroy(self.h)
            self.h = None

    def set_pose(self, pose) -> None:
        P16 = np.ascontiguousarray(pose, np.float32).reshape(16)
        lib().dyo_session_set_pose(self.h, fptr(P16))

    def pose(self) -> np.ndarray:
        out = np.empty(16, np.float64)
        lib().dyo_session_get_pose_f64(self.h, out.ctypes.data_as(P(C.c_double)))
        return out.reshape(4, 4)

    def frame(self, depth, rgb=None):
        d = np.ascontiguousarray(depth, np.uint16)
        r = None if rgb is None else np.ascontiguousarray(rgb, np.uint8)
        pose = np.empty(16, np.float32)
        st = abi.FrameStats()
        lib().dyo_session_frame(self.h, ptr(d), ptr(r), fptr(pose), C.byref(st))
        return pose.reshape(4, 4), st

    def integrate_with_pose(self, depth, rgb, pose) -> None:
        d = np.ascontiguousarray(depth, np.uint16)
        r = None if rgb is None else np.ascontiguousarray(rgb, np.uint8)
        P16 = np.ascontiguousarray(pose, np.float32).reshape(16)
        lib().dyo_session_integrate_with_pose(self.h, ptr(d), ptr(r), fptr(P16))

    def image(self, which: int, level: int, shape, dtype) -> np.ndarray:
        out = np.empty(shape, dtype)
        ok = lib().dyo_session_image(self.h, which, level, ptr(out), out.nbytes)
        if not ok:
            raise ValueError("bad image request")
        return out
