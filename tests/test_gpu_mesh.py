"""Mesh extraction on the GPU (dyn_extract_mesh, dynamap_b200/csrc/mesh.cu)
on the volume the session built, read back: bit for bit and in the same
order as the host build of the same block walk (tests/cpp/mesh_host.cpp),
and the same triangle multiset as the oracle's dense cell walk
(MeshExtractor::ExtractMesh restated) on that volume; FP32 and mixed
voxels; counting, truncation, determinism, invalid boxes; the C++ drop-in
(builder::ExtractMesh, Mesh::SaveToFile)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from dynamap_b200 import abi, configs
from dynamap_b200.session import Session
from meshutil import assert_same_mesh, build_mesh_host

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def mesh_host(tmp_path_factory):
    f = build_mesh_host(tmp_path_factory.mktemp("mesh"))
    if f is None:
        pytest.skip("no C++ compiler")
    return f


def small_rgb():
    p = configs.preset("cfg2")
    p["tsdf"].update(num_blocks=1 << 16, num_buckets=1 << 16)
    p["sensor"].update(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5)
    return p


def centre_box(coords, vs, half=0.3, shift=0.37):
    """A box of +-half metres around the middle of the allocated blocks,
    off the voxel grid by 'shift' voxels."""
    c = np.median(coords, axis=0) * 8 * vs + shift * vs
    return (c - half).astype(np.float32), (c + half).astype(np.float32)


def built_session(precision, n=4, seed=31):
    p = small_rgb()
    seq = configs.sequence(p, seed=seed, n_frames=n)
    t, g, b, s = configs.structs(p)
    m = Session(t, g, b, s, precision=precision)
    for k in range(n):
        m.integrate_with_pose(seq.depth[k], seq.rgb[k], seq.poses[k].astype(np.float32))
    return m, t


@pytest.mark.parametrize("precision", [abi.PRECISION_FP32, abi.PRECISION_MIXED])
def test_mesh_matches_host_walk_and_oracle(gpu_lib, oracle, mesh_host, precision):
    m, t = built_session(precision)
    with m:
        coords, rgbw, sdf = m.download_blocks()
        lo, hi = centre_box(coords, t.voxel_size)
        got = m.extract_mesh(lo, hi)
    assert len(got) > 200
    # the same walk on the host, in the same order
    want = mesh_host(coords, rgbw, sdf, t.voxel_size, lo, hi)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    # the oracle's dense walk over the same voxels
    vol = oracle.Volume(t)
    assert vol.upload(coords, rgbw, sdf) == len(coords)
    assert_same_mesh(got, vol.mesh_triangles(lo, hi))


def test_count_capacity_determinism_and_invalid(gpu_lib):
    m, t = built_session(abi.PRECISION_FP32, n=3, seed=32)
    with m:
        coords, _, _ = m.download_blocks()
        lo, hi = centre_box(coords, t.voxel_size, half=0.25)
        full = m.extract_mesh(lo, hi)
        again = m.extract_mesh(lo, hi)
        np.testing.assert_array_equal(full.view(np.uint32), again.view(np.uint32))
        k = len(full) // 3
        part = m.extract_mesh(lo, hi, capacity=k)
        np.testing.assert_array_equal(part.view(np.uint32), full[:k].view(np.uint32))
        assert len(m.extract_mesh(lo, lo)) == 0  # no cells
        far = m.extract_mesh(lo + 100.0, hi + 100.0)  # cells, no blocks there
        assert len(far) == 0
        for bad in (([0, 0, float("nan")], [1, 1, 1]), ([0, 0, 0], [1e6, 1, 1])):
            with pytest.raises(abi.DynError):
                m.extract_mesh(*bad)


def test_cpp_builder_extract_mesh(gpu_lib, tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    p = configs.preset("cfg1")
    seq = configs.sequence(p, seed=33, n_frames=3)
    s = p["sensor"]
    frames = tmp_path / "frames.bin"
    with open(frames, "wb") as f:
        f.write(f"{s['rows']} {s['cols']} {s['fx']} {s['fy']} {s['cx']} {s['cy']} "
                f"{s['depth_scaler']} {len(seq.depth)}\n".encode())
        f.write(np.ascontiguousarray(seq.depth, np.uint16).tobytes())
        f.write(np.ascontiguousarray(seq.poses, np.float32).tobytes())
    exe = str(tmp_path / "mesh_example")
    libdir = os.path.join(ROOT, "dynamap_b200")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(HERE, "cpp", "mesh_example.cpp"), "-L", libdir,
                    "-ldynamap_b200", f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    # the same volume through the Python session (the C++ example's parameters)
    t, g, b, sen = configs.structs(p)
    t.num_buckets, t.num_blocks = 1 << 16, 1 << 15
    with Session(t, g, b, sen) as m:
        for k in range(len(seq.depth)):
            m.integrate_with_pose(seq.depth[k], None, seq.poses[k].astype(np.float32))
        coords, _, _ = m.download_blocks()
        lo, hi = centre_box(coords, t.voxel_size, half=0.3)
        want = m.extract_mesh(lo, hi)
    obj = tmp_path / "mesh.obj"
    r = subprocess.run([exe, str(frames), str(obj)] + ["%.9g" % x for x in (*lo, *hi)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    n = int(r.stdout.split()[1])
    assert n == len(want) > 100
    lines = obj.read_text().splitlines()
    v = np.array([[float(x) for x in ln.split()[1:]] for ln in lines if ln.startswith("v ")])
    f = [ln for ln in lines if ln.startswith("f ")]
    assert v.shape == (3 * n, 6) and len(f) == n and f[0] == "f 1 2 3"
    # the OBJ's vertices are the mesh's, printed with 6 significant digits
    a = np.sort(v.round(3), axis=0)
    w = np.sort(want.reshape(-1, 6).astype(np.float64).round(3), axis=0)
    assert np.mean(np.abs(a - w) <= 1.5e-3) > 0.999
