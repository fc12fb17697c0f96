"""Helpers of the mesh tests: the host build of the mesh extraction's
block walk (tests/cpp/mesh_host.cpp) and a canonical order of triangles."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def build_mesh_host(outdir):
    """The host walk as a function (coords, rgbw, sdf, vs, lo, hi) ->
    triangles [n, 3, 6] in the kernel's order, or None for an invalid box;
    None when there is no C++ compiler."""
    cxx = shutil.which("g++")
    if cxx is None:
        return None
    so = os.path.join(str(outdir), "libmesh_host.so")
    subprocess.run([cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-ffp-contract=off",
                    os.path.join(HERE, "cpp", "mesh_host.cpp"), "-o", so], check=True)
    f = C.CDLL(so).mesh_host_extract
    f.restype = C.c_int64
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_float,
                  C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_void_p, C.c_int64]

    def extract(coords, rgbw, sdf, vs, lo, hi):
        coords = np.ascontiguousarray(coords, np.int32)
        rgbw = np.ascontiguousarray(rgbw, np.uint8)
        sdf = np.ascontiguousarray(sdf, np.float32)
        lo_c = (C.c_float * 3)(*[float(x) for x in lo])
        hi_c = (C.c_float * 3)(*[float(x) for x in hi])
        args = (coords.ctypes.data, rgbw.ctypes.data, sdf.ctypes.data, len(coords), vs, lo_c, hi_c)
        n = f(*args, None, 0)
        if n < 0:
            return None
        out = np.zeros((n, 3, 6), np.float32)
        assert f(*args, out.ctypes.data, n) == n
        return out
    return extract


def canon(tris):
    """The triangles as a sorted multiset of 18 bit patterns each."""
    a = np.ascontiguousarray(tris, np.float32).reshape(len(tris), 18).view(np.uint32)
    return a[np.lexsort(a.T[::-1])]


def assert_same_mesh(a, b):
    assert a.shape == b.shape
    np.testing.assert_array_equal(canon(a), canon(b))


def sphere_volume(seed, vs=0.01, centre=(0.05, -0.1, 0.3), radius=0.23, trunc=0.04,
                  hole_frac=0.03, drop_frac=0.08):
    """Blocks of a noisy sphere SDF around centre (negative coordinates
    included) with unobserved voxels and missing blocks."""
    rng = np.random.default_rng(seed)
    c = np.asarray(centre)
    lo = np.floor((c - radius - trunc) / (8 * vs)).astype(int) - 1
    hi = np.ceil((c + radius + trunc) / (8 * vs)).astype(int) + 1
    bl = np.stack(np.meshgrid(*[np.arange(a, b) for a, b in zip(lo, hi)], indexing="ij"),
                  -1).reshape(-1, 3)
    centres = (bl * 8 + 3.5) * vs
    dist = np.abs(np.linalg.norm(centres - c, axis=1) - radius)
    bl = bl[dist < trunc + 8 * vs]
    bl = bl[rng.random(len(bl)) >= drop_frac]
    bl = bl[rng.permutation(len(bl))]
    loc = np.stack(np.meshgrid(np.arange(8), np.arange(8), np.arange(8), indexing="ij"),
                   -1).reshape(512, 3)  # x-major, as the voxel order
    g = bl[:, None, :] * 8 + loc[None]
    p = g * vs
    sdf = np.clip(np.linalg.norm(p - c, axis=2) - radius, -trunc, trunc)
    sdf = (sdf + rng.normal(0, 0.002, sdf.shape)).astype(np.float32)
    rgbw = rng.integers(0, 256, size=(len(bl), 512, 4)).astype(np.uint8)
    rgbw[..., 3] = rng.integers(1, 65, size=(len(bl), 512))
    rgbw[..., 3][rng.random((len(bl), 512)) < hole_frac] = 0
    return bl.astype(np.int32), rgbw, sdf
