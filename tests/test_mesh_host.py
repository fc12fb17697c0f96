"""The mesh extraction's block-driven walk (dynamap_b200/csrc/mesh.cu), built
for the host from the same mesh_cell.h arithmetic (tests/cpp/mesh_host.cpp),
against the oracle's dense cell walk (MeshExtractor::ExtractMesh restated,
pinned to the reference in test_golden_ref.py): the same triangles, bit for
bit, on the reference's volume and on synthetic fields with holes, missing
neighbour blocks, negative coordinates and unaligned boxes; invalid boxes
rejected.  The GPU kernel itself is compared with both in
test_gpu_mesh.py."""
import os

import numpy as np
import pytest

from dynamap_b200 import abi
from meshutil import assert_same_mesh as same_mesh, build_mesh_host, sphere_volume

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def mesh_host(tmp_path_factory):
    f = build_mesh_host(tmp_path_factory.mktemp("mesh"))
    if f is None:
        pytest.skip("no C++ compiler")
    return f


@pytest.fixture(scope="module")
def reference_volume(oracle):
    """The volume the reference's own mesh golden was extracted from: three
    frames of the pinned small sequence."""
    g = np.load(os.path.join(HERE, "golden", "ref_rigid_small.npz"))
    s, t = g["sensor"], g["tsdf"]
    sensor = abi.Sensor(rows=int(s[0]), cols=int(s[1]), fx=s[2], fy=s[3], cx=s[4], cy=s[5],
                        depth_scaler=s[6])
    tsdf = abi.TsdfParams(voxel_size=t[0], num_buckets=int(t[1]), bucket_size=int(t[2]),
                          num_blocks=int(t[3]), block_size=int(t[4]), max_sdf_weight=int(t[5]),
                          truncation_distance=t[6], max_sensor_depth=t[7], min_sensor_depth=t[8])
    vol = oracle.Volume(tsdf)
    for k in range(3):
        d = oracle.depth_from_raw(g["depth"][k], sensor.depth_scaler)
        vol.allocate(d, sensor, g["poses"][k])
        vol.integrate(d, g["rgb"][k], sensor, g["poses"][k])
    return vol, tsdf


def test_reference_volume(mesh_host, reference_volume):
    vol, tsdf = reference_volume
    coords, rgbw, sdf = vol.download()
    z = np.load(os.path.join(HERE, "golden", "ref_mesh_vertices.npz"))
    boxes = [z["box"],
             np.array([[2.513, -0.31, 2.487], [3.52, 0.42, 3.61]], np.float32),
             np.array([[3.4, 0.3, 3.4], [2.6, -0.25, 2.6]], np.float32)]  # corners swapped
    for lo, hi in boxes:
        want = vol.mesh_triangles(lo, hi)
        got = mesh_host(coords, rgbw, sdf, tsdf.voxel_size, lo, hi)
        assert len(want) > 1000
        same_mesh(got, want)
    assert len(mesh_host(coords, rgbw, sdf, tsdf.voxel_size, *z["box"])) == int(z["triangles"])


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_synthetic_fields(mesh_host, oracle, seed):
    vs = 0.01
    coords, rgbw, sdf = sphere_volume(seed, vs=vs)
    tsdf = abi.TsdfParams(voxel_size=vs, num_buckets=1 << 14, bucket_size=10,
                          num_blocks=len(coords) + 16, block_size=8, max_sdf_weight=64,
                          truncation_distance=0.04, max_sensor_depth=3.0, min_sensor_depth=0.1)
    vol = oracle.Volume(tsdf)
    assert vol.upload(coords, rgbw, sdf) == len(coords)
    rng = np.random.default_rng(100 + seed)
    boxes = [np.array([[-0.25, -0.4, 0.0], [0.35, 0.2, 0.6]], np.float32)]
    for _ in range(2):
        lo = np.array([-0.22, -0.36, 0.03]) + rng.uniform(-0.05, 0.05, 3)
        boxes.append(np.array([lo, lo + rng.uniform(0.1, 0.3, 3)], np.float32))
    total = 0
    for lo, hi in boxes:
        want = vol.mesh_triangles(lo, hi)
        got = mesh_host(coords, rgbw, sdf, vs, lo, hi)
        same_mesh(got, want)
        total += len(want)
    assert total > 2000


def test_boxes_without_cells_and_invalid(mesh_host):
    coords, rgbw, sdf = sphere_volume(5)
    assert len(mesh_host(coords, rgbw, sdf, 0.01, [0.1, 0.1, 0.1], [0.1, 0.5, 0.5])) == 0
    assert mesh_host(coords, rgbw, sdf, 0.01, [0, 0, float("nan")], [1, 1, 1]) is None
    assert mesh_host(coords, rgbw, sdf, 0.01, [0, 0, 0], [1e6, 1, 1]) is None
    assert mesh_host(coords, rgbw, sdf, 0.01, [0, 0, 0], [float("inf"), 1, 1]) is None
