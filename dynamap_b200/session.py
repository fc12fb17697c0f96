"""Python wrapper of a libdynamap_b200 session (the reference's builder,
include/builder/builder.h:49-117), over the C ABI.

    t, g, b, s = configs.structs(configs.preset("cfg1"))
    with Session(t, g, b, s) as m:
        m.set_pose(pose0)
        for depth in frames:
            pose, stats = m.process(depth)        # buildModelLS
        coords, voxels = m.download_blocks()

Batch steps a fixed set of sessions together (one launch per stage for all
of them, one CUDA graph per frame):

    with Batch([m0, m1, m2]) as b:
        poses, stats, status = b.process([d0, d1, d2])

Server admits sessions under an HBM budget and steps whichever have a frame
waiting (continuous batching):

    with Server(budget_bytes=150 << 30) as sv:
        slot = sv.admit(t, g, b, s, pose0=pose0)
        sv.push(slot, depth)
        sv.step()
        pose, stats = sv.result(slot)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi

_vp = C.c_void_p


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_vp)


def _download_blocks(lib, h):
    n = C.c_int64()
    abi.check("dyn_num_blocks", lib.dyn_num_blocks(h, C.byref(n)))
    n = n.value
    coords = np.empty((n, 3), np.int32)
    vox = np.empty((n, 512, 2), np.uint32)  # {rgbw, sdf bits} per voxel
    got = C.c_int64()
    abi.check("dyn_download_blocks", lib.dyn_download_blocks(
        h, _ptr(coords), _ptr(vox), n, C.byref(got)))
    rgbw = vox[..., 0].copy().view(np.uint8).reshape(n, 512, 4)
    sdf = vox[..., 1].copy().view(np.float32)
    return coords, rgbw, sdf


def _removed(lib, h, fn, args, out: bool):
    """dyn_evict_blocks / dyn_delete_blocks on session handle h: the removed
    blocks as _download_blocks returns them (out), else their count.

    With 'out' the host buffers are sized for every allocated block, since
    the removal itself decides how many go: 4 KiB + 12 B per allocated block
    (8 GiB for a full pool of 2^21 blocks), whatever the number removed.
    Callers that only need the count pass out=False, which allocates
    nothing."""
    n = C.c_int64()
    abi.check("dyn_num_blocks", lib.dyn_num_blocks(h, C.byref(n)))
    n = n.value
    coords = np.empty((n, 3), np.int32) if out else None
    vox = np.empty((n, 512, 2), np.uint32) if out else None
    k = C.c_int64()
    abi.check(fn, getattr(lib, fn)(h, *args, _ptr(coords), _ptr(vox), n if out else 0,
                                   C.byref(k)))
    if not out:
        return k.value
    m = min(k.value, n)
    rgbw = vox[:m, :, 0].copy().view(np.uint8).reshape(m, 512, 4)
    return coords[:m], rgbw, vox[:m, :, 1].copy().view(np.float32)


def _f16(pose) -> C.Array:
    p = np.ascontiguousarray(pose, np.float32).reshape(16)
    return (C.c_float * 16)(*p.tolist())


class Session:
    def __init__(self, tsdf, gn, bil, sensor, precision: int = abi.PRECISION_FP32,
                 device: int = 0):
        self.lib = abi.load()
        self.sensor = sensor
        self.tsdf = tsdf
        self.h = _vp()
        abi.check("dyn_session_create",
                  self.lib.dyn_session_create(C.byref(tsdf), C.byref(gn), C.byref(bil),
                                              C.byref(sensor), precision, device,
                                              C.byref(self.h)))

    def close(self) -> None:
        if self.h:
            self.lib.dyn_session_destroy(self.h)
            self.h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- pose
    def set_pose(self, pose) -> None:
        abi.check("dyn_session_set_pose", self.lib.dyn_session_set_pose(self.h, _f16(pose)))

    def pose(self) -> np.ndarray:
        out = (C.c_float * 16)()
        abi.check("dyn_session_get_pose", self.lib.dyn_session_get_pose(self.h, out))
        return np.array(out, np.float32).reshape(4, 4)

    # ---- frames
    def submit(self, depth: np.ndarray, rgb: np.ndarray | None = None, pose_hint=None) -> None:
        """One frame (dyn_frame_submit).  Up to two frames may be in flight:
        submit frame k+1 before reading frame k's result and its copy to the
        device overlaps frame k's work; results come back in order."""
        d = np.ascontiguousarray(depth, np.uint16)
        r = None if rgb is None else np.ascontiguousarray(rgb, np.uint8)
        # page-locked inputs are read by the copy after the call returns:
        # keep the last two frames' arrays alive
        self._keep = (getattr(self, "_keep", (None,))[-1], (d, r))
        if pose_hint is None:
            abi.check("dyn_frame_submit", self.lib.dyn_frame_submit(self.h, _ptr(d), _ptr(r)))
        else:
            abi.check("dyn_frame_submit_hint", self.lib.dyn_frame_submit_hint(
                self.h, _ptr(d), _ptr(r), _f16(pose_hint)))

    def submit_device(self, depth_ptr: int, rgb_ptr: int | None = None) -> None:
        abi.check("dyn_frame_submit_device",
                  self.lib.dyn_frame_submit_device(self.h, depth_ptr, rgb_ptr))

    def result(self, strict: bool = True):
        pose = (C.c_float * 16)()
        st = abi.FrameStats()
        r = self.lib.dyn_frame_result(self.h, pose, C.byref(st))
        if strict or r not in (abi.DYN_ERR_HASH_FULL, abi.DYN_ERR_HEAP_EXHAUSTED):
            abi.check("dyn_frame_result", r)
        return np.array(pose, np.float32).reshape(4, 4), st

    def process(self, depth, rgb=None, strict: bool = True, pose_hint=None):
        self.submit(depth, rgb, pose_hint)
        return self.result(strict)

    def integrate_with_pose(self, depth, rgb, pose) -> None:
        d = np.ascontiguousarray(depth, np.uint16)
        r = None if rgb is None else np.ascontiguousarray(rgb, np.uint8)
        abi.check("dyn_integrate_with_pose",
                  self.lib.dyn_integrate_with_pose(self.h, _ptr(d), _ptr(r), _f16(pose)))

    def raycast(self, pose, sensor=None, rgb: bool = False):
        s = sensor if sensor is not None else self.sensor
        d = np.empty((s.rows, s.cols), np.float32)
        c = np.empty((s.rows, s.cols, 3), np.uint8) if rgb else None
        abi.check("dyn_raycast", self.lib.dyn_raycast(
            self.h, _f16(pose), C.byref(s) if sensor is not None else None, _ptr(d), _ptr(c)))
        return d, c

    def raycast_maps(self, pose, sensor=None, rgb: bool = False):
        """(depth, vertex4, normal4, rgb) of the model seen from 'pose'."""
        s = sensor if sensor is not None else self.sensor
        d = np.empty((s.rows, s.cols), np.float32)
        v = np.empty((s.rows, s.cols, 4), np.float32)
        n = np.empty((s.rows, s.cols, 4), np.float32)
        c = np.empty((s.rows, s.cols, 3), np.uint8) if rgb else None
        abi.check("dyn_raycast_maps", self.lib.dyn_raycast_maps(
            self.h, _f16(pose), C.byref(s) if sensor is not None else None, _ptr(d), _ptr(v),
            _ptr(n), _ptr(c)))
        return d, v, n, c

    # ---- map access
    def num_blocks(self) -> int:
        n = C.c_int64()
        abi.check("dyn_num_blocks", self.lib.dyn_num_blocks(self.h, C.byref(n)))
        return n.value

    def download_blocks(self):
        """(coords (n,3) int32, rgbw (n,512,4) uint8, sdf (n,512) float32)."""
        return _download_blocks(self.lib, self.h)

    def _removed(self, fn, args, out: bool):
        return _removed(self.lib, self.h, fn, args, out)

    def evict_blocks(self, max_age: int, out: bool = True):
        """Remove the blocks the allocation has not touched in the last
        max_age + 1 frames; with 'out', returns them as download_blocks
        does (heap order), else their count."""
        return self._removed("dyn_evict_blocks", (int(max_age),), out)

    def delete_blocks(self, coords, out: bool = True):
        """Remove the blocks at the given block coordinates [m, 3]."""
        c = np.ascontiguousarray(coords, np.int32).reshape(-1, 3)
        return self._removed("dyn_delete_blocks", (_ptr(c), len(c)), out)

    def upload_blocks(self, coords, rgbw, sdf) -> np.ndarray:
        """Put blocks (as download_blocks returns them) into the volume;
        returns [placed, already present, bucket full, heap exhausted]."""
        c = np.ascontiguousarray(coords, np.int32).reshape(-1, 3)
        n = len(c)
        vox = np.empty((n, 512, 2), np.uint32)
        vox[..., 0] = np.ascontiguousarray(rgbw, np.uint8).reshape(n, 512, 4).view(np.uint32)[..., 0]
        vox[..., 1] = np.ascontiguousarray(sdf, np.float32).reshape(n, 512).view(np.uint32)
        counts = np.zeros(4, np.int64)
        abi.check("dyn_upload_blocks", self.lib.dyn_upload_blocks(
            self.h, _ptr(c), _ptr(vox), n, counts.ctypes.data_as(C.POINTER(C.c_int64))))
        return counts

    def extract_mesh(self, lower, upper, capacity: int | None = None) -> np.ndarray:
        """Triangles [n, 3, 6] ({x, y, z, r, g, b} per vertex, colour 0..1)
        of the model over the box between lower and upper
        (tsdfVolume::ExtractMesh); with no capacity, counted first."""
        lo = (C.c_float * 3)(*[float(x) for x in lower])
        hi = (C.c_float * 3)(*[float(x) for x in upper])
        n = C.c_int64()
        if capacity is None:
            abi.check("dyn_extract_mesh",
                      self.lib.dyn_extract_mesh(self.h, lo, hi, None, 0, C.byref(n)))
            capacity = n.value
        out = np.zeros((capacity, 3, 6), np.float32)
        abi.check("dyn_extract_mesh",
                  self.lib.dyn_extract_mesh(self.h, lo, hi, _ptr(out), capacity, C.byref(n)))
        return out[:min(n.value, capacity)]

    def image(self, which: int, level: int, shape, dtype) -> np.ndarray:
        out = np.empty(shape, dtype)
        abi.check("dyn_debug_image",
                  self.lib.dyn_debug_image(self.h, which, level, _ptr(out), out.nbytes))
        return out


class Batch:
    """dyn_batch over existing sessions (which stay owned by the caller)."""

    def __init__(self, sessions):
        self.lib = abi.load()
        self.sessions = list(sessions)
        self.n = len(self.sessions)
        arr = (_vp * self.n)(*[s.h for s in self.sessions])
        self.h = _vp()
        abi.check("dyn_batch_create", self.lib.dyn_batch_create(arr, self.n, C.byref(self.h)))

    def close(self) -> None:
        if self.h:
            self.lib.dyn_batch_destroy(self.h)
            self.h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, depths, rgbs=None) -> None:
        d = [np.ascontiguousarray(x, np.uint16) for x in depths]
        r = None if rgbs is None else [
            None if x is None else np.ascontiguousarray(x, np.uint8) for x in rgbs]
        self._keep = (d, r)
        dp = (_vp * self.n)(*[x.ctypes.data for x in d])
        rp = None if r is None else (_vp * self.n)(*[None if x is None else x.ctypes.data
                                                    for x in r])
        abi.check("dyn_batch_submit", self.lib.dyn_batch_submit(self.h, dp, rp))

    def submit_device(self, depth_ptrs, rgb_ptrs=None) -> None:
        dp = (_vp * self.n)(*depth_ptrs)
        rp = None if rgb_ptrs is None else (_vp * self.n)(*rgb_ptrs)
        abi.check("dyn_batch_submit_device", self.lib.dyn_batch_submit_device(self.h, dp, rp))

    def result(self, strict: bool = True):
        """(poses (n,4,4) float32, [FrameStats], [status])."""
        poses = (C.c_float * (16 * self.n))()
        stats = (abi.FrameStats * self.n)()
        status = (C.c_int * self.n)()
        r = self.lib.dyn_batch_result(self.h, poses, stats, status)
        if strict or r not in (abi.DYN_ERR_HASH_FULL, abi.DYN_ERR_HEAP_EXHAUSTED):
            abi.check("dyn_batch_result", r)
        return (np.array(poses, np.float32).reshape(self.n, 4, 4), list(stats),
                list(status))

    def process(self, depths, rgbs=None, strict: bool = True):
        self.submit(depths, rgbs)
        return self.result(strict)

    def stream(self) -> int:
        p = _vp()
        abi.check("dyn_batch_stream", self.lib.dyn_batch_stream(self.h, C.byref(p)))
        return p.value or 0

    def profile(self, enable: bool) -> None:
        abi.check("dyn_batch_profile", self.lib.dyn_batch_profile(self.h, int(enable)))

    def stage_times(self, reset: bool = True):
        ms = (C.c_double * len(abi.STAGES))()
        n = C.c_int64()
        abi.check("dyn_batch_stage_times",
                  self.lib.dyn_batch_stage_times(self.h, ms, C.byref(n), int(reset)))
        return list(ms), n.value

    def autotune(self, frames_per_candidate: int = 3) -> None:
        abi.check("dyn_batch_autotune", self.lib.dyn_batch_autotune(self.h, frames_per_candidate))

    def tuning(self):
        """(done, integration CTAs, raycast tile: 0 16x16, 1 32x8, 2 8x8)."""
        d, c, t = C.c_int32(), C.c_int32(), C.c_int32()
        abi.check("dyn_batch_tuning",
                  self.lib.dyn_batch_tuning(self.h, C.byref(d), C.byref(c), C.byref(t)))
        return bool(d.value), c.value, t.value

    def kernels_per_frame(self) -> int:
        n = C.c_int32()
        abi.check("dyn_batch_kernels_per_frame",
                  self.lib.dyn_batch_kernels_per_frame(self.h, C.byref(n)))
        return n.value


class Server:
    """dyn_server: sessions admitted by HBM budget, stepped together."""

    def __init__(self, budget_bytes: int = 0, max_sessions: int = 0, device: int = 0):
        self.lib = abi.load()
        p = abi.ServerParams(budget_bytes, max_sessions, device)
        self.h = _vp()
        abi.check("dyn_server_create", self.lib.dyn_server_create(C.byref(p), C.byref(self.h)))
        self.sensors = {}

    def close(self) -> None:
        if self.h:
            self.lib.dyn_server_destroy(self.h)
            self.h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def admit(self, tsdf, gn, bil, sensor, precision: int = abi.PRECISION_FP32, pose0=None):
        """Slot index, or None when the budget (or the slot table) is full."""
        slot = C.c_int32(-1)
        r = self.lib.dyn_server_admit(self.h, C.byref(tsdf), C.byref(gn), C.byref(bil),
                                      C.byref(sensor), precision,
                                      None if pose0 is None else _f16(pose0), C.byref(slot))
        if r == abi.DYN_ERR_BUDGET_EXCEEDED:
            return None
        abi.check("dyn_server_admit", r)
        self.sensors[slot.value] = sensor
        return slot.value

    def release(self, slot: int) -> None:
        abi.check("dyn_server_release", self.lib.dyn_server_release(self.h, slot))
        self.sensors.pop(slot, None)

    def push(self, slot: int, depth, rgb=None) -> bool:
        """False when the slot's previous frame has not been stepped yet."""
        d = np.ascontiguousarray(depth, np.uint16)
        c = None if rgb is None else np.ascontiguousarray(rgb, np.uint8)
        r = self.lib.dyn_server_push(self.h, slot, _ptr(d), _ptr(c))
        if r == abi.DYN_ERR_NOT_READY:
            return False
        abi.check("dyn_server_push", r)
        return True

    def step(self) -> int:
        n = C.c_int32()
        abi.check("dyn_server_step", self.lib.dyn_server_step(self.h, C.byref(n)))
        return n.value

    def ready(self, slot: int) -> bool:
        r = C.c_int32()
        abi.check("dyn_server_poll", self.lib.dyn_server_poll(self.h, slot, C.byref(r)))
        return bool(r.value)

    def result(self, slot: int, strict: bool = True):
        pose = (C.c_float * 16)()
        st = abi.FrameStats()
        r = self.lib.dyn_server_result(self.h, slot, pose, C.byref(st))
        if strict or r not in (abi.DYN_ERR_HASH_FULL, abi.DYN_ERR_HEAP_EXHAUSTED):
            abi.check("dyn_server_result", r)
        return np.array(pose, np.float32).reshape(4, 4), st

    def sync(self) -> None:
        abi.check("dyn_server_sync", self.lib.dyn_server_sync(self.h))

    def session_handle(self, slot: int):
        p = _vp()
        abi.check("dyn_server_session", self.lib.dyn_server_session(self.h, slot, C.byref(p)))
        return p

    def usage(self) -> dict:
        u = abi.ServerUsage()
        abi.check("dyn_server_info", self.lib.dyn_server_info(self.h, C.byref(u)))
        return {k: getattr(u, k) for k, _ in u._fields_}

    def download_blocks(self, slot: int):
        """The slot's map, as Session.download_blocks."""
        return _download_blocks(self.lib, self.session_handle(slot))

    def evict_blocks(self, slot: int, max_age: int, out: bool = True):
        """Between steps: the slot's blocks not touched in its last
        max_age + 1 frames removed, as Session.evict_blocks."""
        self.sync()
        return _removed(self.lib, self.session_handle(slot), "dyn_evict_blocks",
                        (int(max_age),), out)
