"""The C-ABI library loads without a GPU, exports every entry point that
include/dynamap.h declares, and its host-only calls behave."""
import ctypes as C
import os
import re

import pytest

from dynamap_b200 import abi
from oracle import refsrc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "dynamap.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dyn_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = abi.load()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(abi.SIGNATURES), "ctypes table and header disagree"


def test_abi_version_and_status_strings():
    lib = abi.load()
    assert lib.dyn_abi_version() == 1
    assert lib.dyn_status_string(0) == b"ok"
    assert lib.dyn_status_string(5) == b"voxel block heap exhausted"


def test_struct_layouts_match_header_sizes():
    # field-by-field mirrors: sizes follow the C layout
    assert C.sizeof(abi.Sensor) == 28
    assert C.sizeof(abi.TsdfParams) == 36
    assert C.sizeof(abi.GnParams) == 68
    assert C.sizeof(abi.BilateralParams) == 16
    assert C.sizeof(abi.Voxel) == 8  # geometry::Voxel is 8 bytes


def test_defaults_are_the_reference_config():
    t, g, b, s = abi.defaults()
    assert (t.voxel_size, t.num_buckets, t.bucket_size, t.num_blocks) == pytest.approx(
        (0.01, 2500, 10, 25000))
    assert (t.block_size, t.max_sdf_weight) == (8, 64)
    assert list(g.lvl_iteration_num) == [0, 0, 20] and list(g.lvl_scale) == [4, 2, 1]
    assert g.min_increment == pytest.approx(1e-3) and g.regularization == pytest.approx(0.02)
    assert (b.diameter, b.sigma_i, b.sigma_s) == (8, 10.0, 1.0)
    assert (s.rows, s.cols, s.fx, s.depth_scaler) == (480, 640, 525.0, 5000.0)
    # the python-side defaults (used without the library) agree
    t2, g2, b2, s2 = abi.TsdfParams(), abi.GnParams(), abi.BilateralParams(), abi.Sensor()
    abi._fill_defaults(t2, g2, b2, s2)
    for a, c in ((t, t2), (g, g2), (b, b2), (s, s2)):
        assert bytes(a) == bytes(c)


def test_yaml_parser(tmp_path):
    y = tmp_path / "p.yaml"
    y.write_text("# comment\ntsdfParams:\n  - voxelSize: 0.005\n  - numBuckets: 1048576\n"
                 "gnOptimParams:\n - lvlIterationNum[0]: 10\n - lvlIterationNum[1]: 5\n"
                 " - lvlIterationNum[2]: 4\n - lvlScale[0]: 8\n - colorWeight: 0.1\n"
                 "bilateralFParams:\n  - diameter: 5\n  - sigmaI: 0.03\n"
                 "cameraParams:\n - f.x: 262.5\n - c.y: 119.5\n - width: 320\n - height: 240\n")
    t, g, b, s = abi.defaults()
    lib = abi.load()
    abi.check("yaml", lib.dyn_load_yaml(str(y).encode(), C.byref(t), C.byref(g), C.byref(b),
                                        C.byref(s)))
    assert t.voxel_size == pytest.approx(0.005) and t.num_buckets == 1 << 20
    assert t.bucket_size == 10  # untouched keys keep their value
    assert list(g.lvl_iteration_num) == [10, 5, 4] and g.lvl_scale[0] == 8
    assert g.color_weight == pytest.approx(0.1)
    assert (b.diameter, b.sigma_i) == (5, pytest.approx(0.03))
    assert (s.fx, s.cy, s.cols, s.rows) == (262.5, 119.5, 320, 240)
    assert lib.dyn_load_yaml(b"/nonexistent.yaml", None, None, None, None) == 1


@pytest.mark.skipif(not os.path.isdir(os.path.join(refsrc.reference_root(), "config")),
                    reason="reference tree absent")
def test_yaml_parser_reads_reference_files():
    lib = abi.load()
    t, g, b, s = abi.TsdfParams(), abi.GnParams(), abi.BilateralParams(), abi.Sensor()
    for f in ("tsdfParams", "gnOptimParams", "bilateralFParams", "cameraParams"):
        path = os.path.join(refsrc.reference_root(), "config", f"{f}.yaml").encode()
        abi.check(f, lib.dyn_load_yaml(path, C.byref(t), C.byref(g), C.byref(b), C.byref(s)))
    d = abi.defaults()
    for a, c in zip((t, g, b, s), d):
        for name, _ in a._fields_:
            if name in ("color_weight", "icp_min_depth", "icp_max_depth", "normal_cos_thresh",
                        "mode", "compose_left", "max_iteration", "enabled"):
                continue
            va, vc = getattr(a, name), getattr(c, name)
            va = list(va) if hasattr(va, "__len__") else va
            vc = list(vc) if hasattr(vc, "__len__") else vc
            assert va == vc, name


def test_session_create_validates_before_touching_a_device():
    lib = abi.load()
    t, g, b, s = abi.defaults()
    h = C.c_void_p()
    bad = abi.TsdfParams.from_buffer_copy(t)
    bad.block_size = 16
    assert lib.dyn_session_create(C.byref(bad), C.byref(g), C.byref(b), C.byref(s), 0, 0,
                                  C.byref(h)) == 1
    bad_g = abi.GnParams.from_buffer_copy(g)
    bad_g.lvl_scale[0] = 3
    assert lib.dyn_session_create(C.byref(t), C.byref(bad_g), C.byref(b), C.byref(s), 0, 0,
                                  C.byref(h)) == 1
    assert lib.dyn_session_create(None, C.byref(g), C.byref(b), C.byref(s), 0, 0,
                                  C.byref(h)) == 1
    n = C.c_size_t()
    abi.check("bytes", lib.dyn_session_bytes(C.byref(t), C.byref(s), 0, C.byref(n)))
    assert n.value > 25000 * 512 * 8


def test_session_create_without_device_reports_it():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    lib = abi.load()
    t, g, b, s = abi.defaults()
    h = C.c_void_p()
    assert lib.dyn_session_create(C.byref(t), C.byref(g), C.byref(b), C.byref(s), 0, 0,
                                  C.byref(h)) == 10


def test_server_create_without_device_reports_it():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    lib = abi.load()
    h = C.c_void_p()
    assert lib.dyn_server_create(None, C.byref(h)) == 1
    p = abi.ServerParams(1 << 30, 8, 0)
    assert lib.dyn_server_create(C.byref(p), C.byref(h)) == 10
    assert lib.dyn_server_step(None, None) == 1
    assert lib.dyn_server_push(None, 0, None, None) == 1


def test_session_bytes_follow_the_voxel_form():
    lib = abi.load()
    t, g, b, s = abi.defaults()
    n32, n16 = C.c_size_t(), C.c_size_t()
    abi.check("bytes", lib.dyn_session_bytes(C.byref(t), C.byref(s), 0, C.byref(n32)))
    abi.check("bytes", lib.dyn_session_bytes(C.byref(t), C.byref(s), 1, C.byref(n16)))
    vox = t.num_blocks * 512
    # FP32 voxels are 8 bytes; the mixed bound counts 4 + 4 (colour kept)
    # plus the raycast's free-space summaries (5 bytes per block)
    assert n16.value - n32.value == 5 * t.num_blocks
    assert n32.value > vox * 8
    assert lib.dyn_session_bytes(C.byref(t), C.byref(s), 0, None) == 1


def test_extract_mesh_validates_before_touching_a_device():
    lib = abi.load()
    lo = (C.c_float * 3)(0.0, 0.0, 0.0)
    hi = (C.c_float * 3)(1.0, 1.0, 1.0)
    n = C.c_int64(-7)
    assert lib.dyn_extract_mesh(None, lo, hi, None, 0, C.byref(n)) == 1
    assert lib.dyn_extract_mesh(None, lo, hi, None, -1, C.byref(n)) == 1
    assert lib.dyn_extract_mesh(None, None, hi, None, 0, C.byref(n)) == 1


def test_eviction_entries_validate_before_touching_a_device():
    lib = abi.load()
    n = C.c_int64(-7)
    counts = (C.c_int64 * 4)()
    assert lib.dyn_evict_blocks(None, 3, None, None, 0, C.byref(n)) == 1
    assert lib.dyn_delete_blocks(None, None, 0, None, None, 0, C.byref(n)) == 1
    assert lib.dyn_upload_blocks(None, None, None, 0, counts) == 1
