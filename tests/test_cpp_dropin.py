"""The C++ drop-in classes (include/builder/builder.h,
include/geometry/tsdf/tsdf.h, include/solver/gnSolver/gnSolver.h) compile
against the C ABI library and, on a GPU, track a sequence end to end."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_example.cpp")
LIBDIR = os.path.join(ROOT, "dynamap_b200")


def compile_example(out):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SRC,
                    "-L", LIBDIR, "-ldynamap_b200", f"-Wl,-rpath,{LIBDIR}", "-o", out],
                   check=True)


def test_dropin_headers_compile_and_link(tmp_path):
    compile_example(str(tmp_path / "dropin"))
    # every header is self-contained
    for h in ("builder/builder.h", "geometry/tsdf/tsdf.h", "solver/gnSolver/gnSolver.h",
              "image/sensor/rgbdImage.h", "dynamap/types.h", "dynamap/pose_io.h", "utils/dataSet.h",
              "geometry/mesh/mesh.h", "geometry/geom_Types.h", "dynamap.h"):
        src = tmp_path / "inc.cpp"
        src.write_text(f'#include "{h}"\nint main() {{ return 0; }}\n')
        subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                        str(src)], check=True)


@pytest.mark.gpu
def test_dropin_builder_tracks(tmp_path, gpu_lib):
    from dynamap_b200 import configs
    p = configs.preset("cfg1")
    seq = configs.sequence(p, seed=4, n_frames=10)
    s = p["sensor"]
    path = tmp_path / "frames.bin"
    with open(path, "wb") as f:
        f.write(f"{s['rows']} {s['cols']} {s['fx']} {s['fy']} {s['cx']} {s['cy']} "
                f"{s['depth_scaler']} {len(seq.depth)}\n".encode())
        f.write(np.ascontiguousarray(seq.depth, np.uint16).tobytes())
        f.write(np.ascontiguousarray(seq.poses, np.float32).tobytes())
    exe = str(tmp_path / "dropin")
    compile_example(exe)
    r = subprocess.run([exe, str(path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "trans_err" in r.stdout


def test_mesh_save_to_file_and_volume_calls_compile(tmp_path):
    """Mesh::SaveToFile writes the reference's OBJ layout (mesh.cu:39-64):
    'v x y z r g b' per vertex, then 'f i i+1 i+2' (1-based) per triangle;
    the volume's mesh and eviction calls compile with the caller's types."""
    exe = str(tmp_path / "mesh_io")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I",
                    os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "mesh_io_example.cpp"), "-L", LIBDIR,
                    "-ldynamap_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    tri = np.arange(2 * 18, dtype=np.float32) * 0.25 - 1.0
    obj = tmp_path / "m.obj"
    r = subprocess.run([exe, str(obj)], input=" ".join("%.9g" % v for v in tri),
                       capture_output=True, text=True, check=True)
    assert r.stdout.strip() == "2"
    lines = obj.read_text().splitlines()
    assert lines[6:] == ["f 1 2 3", "f 4 5 6"]
    v = np.array([[float(a) for a in ln.split()[1:]] for ln in lines[:6]], np.float32)
    assert all(ln.startswith("v ") for ln in lines[:6])
    np.testing.assert_allclose(v.reshape(-1), tri, rtol=1e-5, atol=1e-6)


IDIOM = os.path.join(ROOT, "tests", "cpp", "reference_idiom.cpp")


def compile_idiom(out, extra=()):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-Werror", "-I",
                    os.path.join(ROOT, "include"), *extra, IDIOM, "-L", LIBDIR, "-ldynamap_b200",
                    f"-Wl,-rpath,{LIBDIR}", "-lz", "-o", out], check=True)


def test_reference_idiom_compiles(tmp_path):
    """The reference's calls as its driver and builder write them
    (dynaMap.cpp:180-301, builder.cu:70-139): gnSolver::solve on rgbdImage
    frames and point clouds, tsdfVolume::init(const tsdfProperties&),
    rgbdImage's clouds, HashTable's calls, builder's clouds -- against
    include/ alone, and with CUDA's own vector types on the include path."""
    compile_idiom(str(tmp_path / "idiom"))
    cuda_inc = "/usr/local/cuda/include"
    if os.path.isdir(cuda_inc):
        compile_idiom(str(tmp_path / "idiom_cuda"), ("-I", cuda_inc))


@pytest.mark.gpu
def test_reference_idiom_runs(tmp_path, gpu_lib):
    from test_dataset import make_tum
    root = tmp_path / "seq"
    root.mkdir()
    seq, p = make_tum(root, n=8)
    s = p["sensor"]
    exe = str(tmp_path / "idiom")
    compile_idiom(exe)
    r = subprocess.run([exe, str(root)] + [str(s[k]) for k in ("rows", "cols", "fx", "fy", "cx",
                                                                 "cy", "depth_scaler")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "FAILED" not in r.stdout
