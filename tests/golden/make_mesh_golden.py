"""Generate tests/golden/ref_mesh_vertices.npz from the REFERENCE's own mesh
extraction (MeshExtractor::ExtractMesh, include/geometry/mesh/meshExtractor/
meshExtractor.cu:364-407 with mesh.cu, compiled for the CPU by
oracle/ref_cpu/build_ref.sh into oracle/_ref/libdynref.so).

The volume is the one ref_rigid_small.npz pins (its three frames integrated
at their poses by the reference); the mesh of a box through the observed
surfaces is extracted on one host thread.  Stored: the box, the triangle
count, the total area and the distinct vertices {x, y, z, r, g, b} of the
triangles (sorted by their bit patterns) -- the part of the mesh that does
not depend on the marching-cubes triangle table.

Usage (needs the reference tree, present only where the fixtures are made):
    bash oracle/ref_cpu/build_ref.sh && python tests/golden/make_mesh_golden.py
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from dynamap_b200 import abi  # noqa: E402
from make_golden import params  # noqa: E402

LIB = os.path.join(ROOT, "oracle", "_ref", "libdynref.so")
OUT = os.path.join(HERE, "ref_mesh_vertices.npz")
BOX = ((2.6, -0.25, 2.6), (3.4, 0.3, 3.4))


def main():
    L = C.CDLL(LIB)
    vp = C.c_void_p
    L.ref_volume_create.restype = vp
    L.ref_volume_create.argtypes = [C.POINTER(abi.TsdfParams)]
    L.ref_volume_integrate.argtypes = [vp, vp, vp, C.POINTER(abi.Sensor), C.POINTER(C.c_float)]
    L.ref_extract_mesh.restype = C.c_int64
    L.ref_extract_mesh.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float,
                                   vp, C.c_int64]
    L.ref_set_threads(1)
    sensor, tsdf = params()
    g = np.load(os.path.join(HERE, "ref_rigid_small.npz"))
    p = lambda a: a.ctypes.data_as(vp)
    f16 = lambda m: (C.c_float * 16)(*np.asarray(m, np.float32).reshape(16).tolist())
    vol = L.ref_volume_create(C.byref(tsdf))
    for k in range(3):
        d = (g["depth"][k].astype(np.float32) / np.float32(sensor.depth_scaler)).astype(np.float32)
        L.ref_volume_integrate(vol, p(np.ascontiguousarray(d)), p(np.ascontiguousarray(g["rgb"][k])),
                               C.byref(sensor), f16(g["poses"][k]))
    lo, hi = BOX
    cap = 1 << 20
    out = np.zeros((cap, 18), np.float32)
    n = L.ref_extract_mesh(vol, (C.c_float * 3)(*lo), (C.c_float * 3)(*hi), tsdf.voxel_size,
                           p(out), cap)
    assert 0 < n < cap
    verts = out[:n].reshape(-1, 6)
    uniq = np.unique(np.ascontiguousarray(verts).view(np.uint32), axis=0).view(np.float32)
    t = out[:n].reshape(-1, 3, 6)[:, :, :3].astype(np.float64)
    area = 0.5 * np.linalg.norm(np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]), axis=1).sum()
    np.savez_compressed(OUT, box=np.array(BOX, np.float32), triangles=np.int64(n),
                        area=np.float64(area), vertices=uniq)
    print(f"wrote {OUT}: {n} triangles, {len(uniq)} distinct vertices")


if __name__ == "__main__":
    main()
