"""ctypes mirror of include/dynamap.h and the loader of libdynamap_b200.so.

The structs below are field-for-field copies of the C declarations; the
loader raises if the shared library is missing -- there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdynamap_b200.so")

DYN_OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "out of device memory",
          3: "memory budget exceeded", 4: "hash bucket full",
          5: "voxel block heap exhausted", 6: "icp diverged", 7: "timeout",
          8: "cuda error", 9: "not ready", 10: "no cuda device"}
DYN_ERR_BUDGET_EXCEEDED = 3
DYN_ERR_HASH_FULL = 4
DYN_ERR_HEAP_EXHAUSTED = 5
DYN_ERR_TIMEOUT = 7
DYN_ERR_NOT_READY = 9
DYN_ERR_NO_DEVICE = 10
STAGES = ["ingest", "bilateral", "source_maps", "icp", "allocate", "visible", "integrate",
          "raycast", "target_maps", "frame"]
PRECISION_FP32 = 0
PRECISION_MIXED = 1
PRECISION_MIXED_BAND = 2


class Sensor(C.Structure):
    """rgbdSensor (include/image/sensor/rgbdSensor.h:13-19)."""
    _fields_ = [("rows", C.c_uint32), ("cols", C.c_uint32), ("fx", C.c_float),
                ("fy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
                ("depth_scaler", C.c_float)]


class TsdfParams(C.Structure):
    """tsdf::tsdfProperties (include/geometry/tsdf/tsdf.h:19-35)."""
    _fields_ = [("voxel_size", C.c_float), ("num_buckets", C.c_int32),
                ("bucket_size", C.c_int32), ("num_blocks", C.c_int32),
                ("block_size", C.c_int32), ("max_sdf_weight", C.c_int32),
                ("truncation_distance", C.c_float), ("max_sensor_depth", C.c_float),
                ("min_sensor_depth", C.c_float)]


class GnParams(C.Structure):
    """solver::Properties (include/solver/gnSolver/gnSolver.h:47-55) + the
    values the reference hard-codes."""
    _fields_ = [("lvl_iteration_num", C.c_int32 * 3), ("lvl_scale", C.c_int32 * 3),
                ("max_iteration", C.c_int32), ("min_increment", C.c_float),
                ("max_increment", C.c_float), ("regularization", C.c_float),
                ("huber_constant", C.c_float), ("color_weight", C.c_float),
                ("icp_min_depth", C.c_float), ("icp_max_depth", C.c_float),
                ("normal_cos_thresh", C.c_float), ("mode", C.c_int32),
                ("compose_left", C.c_int32)]


class BilateralParams(C.Structure):
    """gaussianKernal (include/image/kernel2D/kernel2D.h:20-43)."""
    _fields_ = [("diameter", C.c_int32), ("sigma_i", C.c_float),
                ("sigma_s", C.c_float), ("enabled", C.c_int32)]


class Voxel(C.Structure):
    """geometry::Voxel (include/geometry/geom_Types.h:72-76), 8 bytes."""
    _fields_ = [("r", C.c_uint8), ("g", C.c_uint8), ("b", C.c_uint8),
                ("weight", C.c_uint8), ("sdf", C.c_float)]


class FrameStats(C.Structure):
    _fields_ = [("frame_index", C.c_int32), ("icp_iterations", C.c_int32 * 3),
                ("icp_inliers", C.c_int32 * 3), ("icp_rms", C.c_float * 3),
                ("icp_reset", C.c_int32), ("blocks_total", C.c_int32),
                ("blocks_new", C.c_int32), ("blocks_visible", C.c_int32),
                ("unique_blocks_probed", C.c_int32), ("bucket_full", C.c_int32),
                ("heap_exhausted", C.c_int32), ("dda_overruns", C.c_int32),
                ("raycast_overruns", C.c_int32), ("pose_increment", C.c_double * 6)]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class ServerParams(C.Structure):
    _fields_ = [("budget_bytes", C.c_size_t), ("max_sessions", C.c_int32),
                ("device", C.c_int32)]


class ServerUsage(C.Structure):
    _fields_ = [("budget_bytes", C.c_size_t), ("used_bytes", C.c_size_t),
                ("capacity", C.c_int32), ("sessions", C.c_int32), ("steps", C.c_int64),
                ("steps_done", C.c_int64), ("frames", C.c_int64)]


P = C.POINTER
_vp = C.c_void_p

# name: (restype, argtypes)
SIGNATURES = {
    "dyn_abi_version": (C.c_int32, []),
    "dyn_status_string": (C.c_char_p, [C.c_int]),
    "dyn_default_params": (C.c_int, [P(TsdfParams), P(GnParams), P(BilateralParams), P(Sensor)]),
    "dyn_load_yaml": (C.c_int, [C.c_char_p, P(TsdfParams), P(GnParams), P(BilateralParams), P(Sensor)]),
    "dyn_session_bytes": (C.c_int, [P(TsdfParams), P(Sensor), C.c_int32, P(C.c_size_t)]),
    "dyn_session_create": (C.c_int, [P(TsdfParams), P(GnParams), P(BilateralParams), P(Sensor),
                                     C.c_int32, C.c_int32, P(_vp)]),
    "dyn_session_destroy": (C.c_int, [_vp]),
    "dyn_session_reset": (C.c_int, [_vp]),
    "dyn_session_get_pose": (C.c_int, [_vp, P(C.c_float)]),
    "dyn_session_set_pose": (C.c_int, [_vp, P(C.c_float)]),
    "dyn_frame_submit": (C.c_int, [_vp, _vp, _vp]),
    "dyn_frame_submit_device": (C.c_int, [_vp, _vp, _vp]),
    "dyn_frame_submit_hint": (C.c_int, [_vp, _vp, _vp, P(C.c_float)]),
    "dyn_raycast_maps": (C.c_int, [_vp, P(C.c_float), P(Sensor), _vp, _vp, _vp, _vp]),
    "dyn_frame_result": (C.c_int, [_vp, P(C.c_float), P(FrameStats)]),
    "dyn_integrate_with_pose": (C.c_int, [_vp, _vp, _vp, P(C.c_float)]),
    "dyn_raycast": (C.c_int, [_vp, P(C.c_float), P(Sensor), _vp, _vp]),
    "dyn_num_blocks": (C.c_int, [_vp, P(C.c_int64)]),
    "dyn_find_blocks": (C.c_int, [_vp, _vp, C.c_int64, _vp]),
    "dyn_barrier_selftest": (C.c_int, [C.c_int32, C.c_int32, C.c_int32]),
    "dyn_download_blocks": (C.c_int, [_vp, _vp, _vp, C.c_int64, P(C.c_int64)]),
    "dyn_extract_mesh": (C.c_int, [_vp, P(C.c_float), P(C.c_float), _vp, C.c_int64,
                                   P(C.c_int64)]),
    "dyn_evict_blocks": (C.c_int, [_vp, C.c_int32, _vp, _vp, C.c_int64, P(C.c_int64)]),
    "dyn_delete_blocks": (C.c_int, [_vp, _vp, C.c_int64, _vp, _vp, C.c_int64, P(C.c_int64)]),
    "dyn_upload_blocks": (C.c_int, [_vp, _vp, _vp, C.c_int64, P(C.c_int64)]),
    "dyn_debug_image": (C.c_int, [_vp, C.c_int32, C.c_int32, _vp, C.c_size_t]),
    "dyn_bilateral_filter": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, P(BilateralParams), _vp]),
    "dyn_depth_to_maps": (C.c_int, [_vp, P(Sensor), _vp, _vp, _vp]),
    "dyn_depth_to_maps_host": (C.c_int, [_vp, P(Sensor), _vp, _vp]),
    "dyn_icp_normal_equations": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, P(Sensor), P(GnParams),
                                           P(C.c_float), P(C.c_double), _vp]),
    "dyn_sessions_submit": (C.c_int, [P(_vp), C.c_int32, P(_vp), P(_vp)]),
    "dyn_session_stream": (C.c_int, [_vp, P(_vp)]),
    "dyn_session_profile": (C.c_int, [_vp, C.c_int32]),
    "dyn_session_stage_times": (C.c_int, [_vp, P(C.c_double), P(C.c_int64), C.c_int32]),
    "dyn_session_kernels_per_frame": (C.c_int, [_vp, P(C.c_int32)]),
    "dyn_frame_d2h_bytes": (C.c_size_t, []),
    "dyn_solver_solve": (C.c_int, [_vp, _vp, _vp, _vp, _vp, P(C.c_float), P(C.c_double),
                                   P(FrameStats)]),
    "dyn_icp_normal_equations_noalloc": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, P(Sensor),
                                                   P(GnParams), P(C.c_float), P(C.c_double),
                                                   _vp]),
    "dyn_batch_create": (C.c_int, [P(_vp), C.c_int32, P(_vp)]),
    "dyn_batch_destroy": (C.c_int, [_vp]),
    "dyn_batch_submit": (C.c_int, [_vp, P(_vp), P(_vp)]),
    "dyn_batch_submit_device": (C.c_int, [_vp, P(_vp), P(_vp)]),
    "dyn_batch_result": (C.c_int, [_vp, P(C.c_float), P(FrameStats), P(C.c_int)]),
    "dyn_batch_size": (C.c_int, [_vp, P(C.c_int32)]),
    "dyn_batch_stream": (C.c_int, [_vp, P(_vp)]),
    "dyn_batch_profile": (C.c_int, [_vp, C.c_int32]),
    "dyn_batch_stage_times": (C.c_int, [_vp, P(C.c_double), P(C.c_int64), C.c_int32]),
    "dyn_batch_kernels_per_frame": (C.c_int, [_vp, P(C.c_int32)]),
    "dyn_batch_autotune": (C.c_int, [_vp, C.c_int32]),
    "dyn_batch_tuning": (C.c_int, [_vp, P(C.c_int32), P(C.c_int32), P(C.c_int32)]),
    "dyn_server_create": (C.c_int, [P(ServerParams), P(_vp)]),
    "dyn_server_destroy": (C.c_int, [_vp]),
    "dyn_server_admit": (C.c_int, [_vp, P(TsdfParams), P(GnParams), P(BilateralParams),
                                   P(Sensor), C.c_int32, P(C.c_float), P(C.c_int32)]),
    "dyn_server_release": (C.c_int, [_vp, C.c_int32]),
    "dyn_server_push": (C.c_int, [_vp, C.c_int32, _vp, _vp]),
    "dyn_server_step": (C.c_int, [_vp, P(C.c_int32)]),
    "dyn_server_poll": (C.c_int, [_vp, C.c_int32, P(C.c_int32)]),
    "dyn_server_result": (C.c_int, [_vp, C.c_int32, P(C.c_float), P(FrameStats)]),
    "dyn_server_sync": (C.c_int, [_vp]),
    "dyn_server_session": (C.c_int, [_vp, C.c_int32, P(_vp)]),
    "dyn_server_info": (C.c_int, [_vp, P(ServerUsage)]),
}

_lib = None


class DynError(RuntimeError):
    def __init__(self, fn: str, status: int):
        super().__init__(f"{fn}: {STATUS.get(status, status)} ({status})")
        self.status = status


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the CUDA library; raises if it is missing (no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"libdynamap_b200.so not found at {path}: build it with "
            "`python -m dynamap_b200.build` (nvcc, sm_100a)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(fn: str, status: int) -> None:
    if status != DYN_OK:
        raise DynError(fn, status)


def defaults():
    """(tsdf, gn, bilateral, sensor) structs with the reference's defaults."""
    t, g, b, s = TsdfParams(), GnParams(), BilateralParams(), Sensor()
    check("dyn_default_params", load().dyn_default_params(C.byref(t), C.byref(g),
                                                          C.byref(b), C.byref(s)))
    return t, g, b, s


def make_params(sensor: dict, tsdf: dict, gn: dict, bilateral: dict | None = None):
    """Structs from plain dicts (keys are the struct field names).  Fields
    not given keep the reference defaults (config/*.yaml)."""
    t, g, b, s = TsdfParams(), GnParams(), BilateralParams(), Sensor()
    _fill_defaults(t, g, b, s)
    for k, v in sensor.items():
        setattr(s, k, v)
    for k, v in tsdf.items():
        setattr(t, k, v)
    for k, v in gn.items():
        if k in ("lvl_iteration_num", "lvl_scale"):
            getattr(g, k)[:] = list(v)
        else:
            setattr(g, k, v)
    for k, v in (bilateral or {}).items():
        setattr(b, k, v)
    return t, g, b, s


def _fill_defaults(t, g, b, s) -> None:
    """The defaults of dyn_default_params, without loading the library (the
    oracle and CPU-only tests use them too)."""
    import math
    t.voxel_size, t.num_buckets, t.bucket_size, t.num_blocks = 0.01, 2500, 10, 25000
    t.block_size, t.max_sdf_weight, t.truncation_distance = 8, 64, 0.05
    t.max_sensor_depth, t.min_sensor_depth = 5.0, 0.3
    g.lvl_iteration_num[:] = [0, 0, 20]
    g.lvl_scale[:] = [4, 2, 1]
    g.max_iteration, g.min_increment, g.max_increment = 20, 0.001, 0.3
    g.regularization, g.huber_constant, g.color_weight = 0.02, 0.3, 0.0
    g.icp_min_depth, g.icp_max_depth = 0.15, 2.0
    g.normal_cos_thresh = math.cos(math.pi / 10)
    g.mode, g.compose_left = 1, 0
    b.diameter, b.sigma_i, b.sigma_s, b.enabled = 8, 10.0, 1.0, 1
    s.fx, s.fy, s.cx, s.cy, s.depth_scaler, s.rows, s.cols = 525.0, 525.0, 319.5, 239.5, 5000.0, 480, 640
