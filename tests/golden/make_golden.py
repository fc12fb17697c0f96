"""Generate tests/golden/ref_rigid_small.npz from the REFERENCE's own code.

Runs the reference's rigid-path sources (tsdf.cu, hashTable.cu, heap.cu,
rgbdImage.cu, pyramid.cu, compiled for the CPU by oracle/ref_cpu/build_ref.sh
into oracle/_ref/libdynref.so) on a small seeded synthetic sequence and
stores inputs and outputs:

  - IntegrateScan (AllocateFromDepthKernel + IntegrateScanKernel) of three
    frames at their ground-truth poses: every allocated block's coordinate,
    heap index and voxels (colour, weight, sdf);
  - GenerateDepth / GenerateRgb at two poses and at a half-resolution
    virtual sensor;
  - the vertex map and vertex normals of rgbdImage;
  - pyramid::applyBilateralFilter on pixels whose window lies in the image;
  - HashTable::Hash of random block coordinates.

Kernels run serially (one host thread), so the reference's races do not
occur and its heap hands out indices 0, 1, 2, ... in pixel order.

Usage (needs the reference tree, present only where the fixtures are made):
    bash oracle/ref_cpu/build_ref.sh && python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from dynamap_b200 import abi, scene  # noqa: E402

LIB = os.path.join(ROOT, "oracle", "_ref", "libdynref.so")
OUT = os.path.join(HERE, "ref_rigid_small.npz")


def block_crc(rgbw: np.ndarray, sdf: np.ndarray) -> int:
    """CRC32 of one block's voxels: 512 x (r, g, b, w) bytes, then 512 sdf
    float32 bit patterns (little endian)."""
    import zlib
    return zlib.crc32(np.ascontiguousarray(sdf, "<f4").tobytes(),
                      zlib.crc32(np.ascontiguousarray(rgbw, np.uint8).tobytes()))


def params():
    sensor = abi.Sensor(rows=60, cols=80, fx=65.625, fy=65.625, cx=39.5, cy=29.5,
                        depth_scaler=1000.0)
    tsdf = abi.TsdfParams(voxel_size=0.008, num_buckets=1 << 12, bucket_size=10,
                          num_blocks=1 << 13, block_size=8, max_sdf_weight=64,
                          truncation_distance=0.032, max_sensor_depth=3.0,
                          min_sensor_depth=0.15)
    return sensor, tsdf


def main():
    L = C.CDLL(LIB)
    vp = C.c_void_p
    L.ref_volume_create.restype = vp
    L.ref_volume_create.argtypes = [C.POINTER(abi.TsdfParams)]
    L.ref_volume_integrate.argtypes = [vp, vp, vp, C.POINTER(abi.Sensor), C.POINTER(C.c_float)]
    L.ref_volume_generate.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(abi.Sensor), vp, vp]
    L.ref_volume_download.restype = C.c_int64
    L.ref_volume_download.argtypes = [vp, vp, vp, vp, C.c_int64]
    L.ref_hash.restype = C.c_int32
    L.ref_hash.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32]
    L.ref_normals.argtypes = [vp, C.POINTER(abi.Sensor), vp, vp]
    L.ref_bilateral_pixel.restype = C.c_float
    L.ref_bilateral_pixel.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_float, C.c_float]
    L.ref_set_threads(1)
    sensor, tsdf = params()
    seq = scene.make_sequence(7, 3, sensor.rows, sensor.cols, sensor.fx, sensor.fy, sensor.cx,
                              sensor.cy, 0.005, 0.5, with_rgb=True, kind="cube")
    p = lambda a: a.ctypes.data_as(vp)
    f16 = lambda m: (C.c_float * 16)(*np.asarray(m, np.float32).reshape(16).tolist())
    depth_f = (seq.depth.astype(np.float32) / np.float32(sensor.depth_scaler)).astype(np.float32)
    vol = L.ref_volume_create(C.byref(tsdf))
    for k in range(3):
        L.ref_volume_integrate(vol, p(np.ascontiguousarray(depth_f[k])),
                               p(np.ascontiguousarray(seq.rgb[k])), C.byref(sensor),
                               f16(seq.poses[k]))
    n = L.ref_volume_download(vol, None, None, None, 0)
    coords = np.zeros((n, 3), np.int32)
    rgbw = np.zeros((n, 512, 4), np.uint8)
    sdf = np.zeros((n, 512), np.float32)
    L.ref_volume_download(vol, p(coords), p(rgbw), p(sdf), n)
    # raycasts
    rays = {}
    for name, pose, s in (("ray_pose2", seq.poses[2], sensor), ("ray_pose0", seq.poses[0], sensor),
                          ("ray_half", seq.poses[1],
                           abi.Sensor(rows=30, cols=40, fx=32.8125, fy=32.8125, cx=19.75,
                                      cy=14.75, depth_scaler=1000.0))):
        d = np.zeros((s.rows, s.cols), np.float32)
        c = np.zeros((s.rows, s.cols, 3), np.uint8)
        L.ref_volume_generate(vol, f16(pose), C.byref(s), p(d), p(c))
        rays[name + "_depth"] = d
        rays[name + "_rgb"] = c
    # normals
    pts = np.zeros((sensor.rows, sensor.cols, 3), np.float32)
    nrm = np.zeros((sensor.rows, sensor.cols, 3), np.float32)
    L.ref_normals(p(np.ascontiguousarray(depth_f[0])), C.byref(sensor), p(pts), p(nrm))
    # bilateral on pixels whose 16x16 window (offsets -8..7) is inside
    r = 8
    bil = np.full((sensor.rows, sensor.cols), np.nan, np.float32)
    src = np.ascontiguousarray(depth_f[1])
    for x in range(r, sensor.rows - r + 1):
        for y in range(r, sensor.cols - r + 1):
            bil[x, y] = L.ref_bilateral_pixel(p(src), sensor.rows, sensor.cols, x, y, r, 10.0, 1.0)
    # hash
    rng = np.random.default_rng(11)
    hc = rng.integers(-5000, 5000, size=(256, 3)).astype(np.int32)
    hv = np.array([L.ref_hash(vol, int(a), int(b), int(c_)) for a, b, c_ in hc], np.int32)
    # every block: coordinate + CRC32 of its voxels; every 16th block (in
    # coordinate order): the voxels themselves
    order = np.lexsort((coords[:, 2], coords[:, 1], coords[:, 0]))
    coords, rgbw, sdf = coords[order], rgbw[order], sdf[order]
    crc = np.array([block_crc(rgbw[i], sdf[i]) for i in range(n)], np.uint32)
    sub = np.arange(0, n, 16)
    np.savez_compressed(
        OUT, depth=seq.depth, rgb=seq.rgb, poses=seq.poses.astype(np.float32),
        sensor=np.array([sensor.rows, sensor.cols, sensor.fx, sensor.fy, sensor.cx, sensor.cy,
                         sensor.depth_scaler], np.float64),
        tsdf=np.array([tsdf.voxel_size, tsdf.num_buckets, tsdf.bucket_size, tsdf.num_blocks,
                       tsdf.block_size, tsdf.max_sdf_weight, tsdf.truncation_distance,
                       tsdf.max_sensor_depth, tsdf.min_sensor_depth], np.float64),
        block_coords=coords, block_crc=crc, subset=sub, subset_rgbw=rgbw[sub],
        subset_sdf=sdf[sub], normals_points=pts,
        normals=nrm, bilateral=bil, bilateral_src_frame=np.int32(1), hash_coords=hc,
        hash_values=hv, **rays)
    print(f"wrote {OUT}: {n} blocks, {os.path.getsize(OUT) / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
