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
