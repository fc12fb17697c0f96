"""The mesh-extraction and eviction kernels themselves
(dynamap_b200/csrc/{mesh,evict}_kernels.cuh), run on the CPU under a
thread-block emulation (tests/cpp/cuda_emu.h: one user-space context per
CUDA thread, barriers for __syncthreads, a per-warp exchange for shuffles), in
the launch order of the library's entry points, on volumes built by the
library's own upload kernel in both voxel forms: the mesh equals the host
build of the same walk in content and order, and eviction leaves the same
volume and hands out the same blocks as the host build of the same steps.
This covers what the host builds do not: the two-pass mesh output with its
scans and offsets, the shared-memory tile (and, built with a smaller tile,
its fallback to the volume), the upload's counts, and the kernels'
indexing."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from meshutil import build_mesh_host, sphere_volume
from test_evict_host import Host, blocks, lib as evict_lib  # noqa: F401 (fixture)

HERE = os.path.dirname(os.path.abspath(__file__))
CUDA_INC = "/usr/local/cuda/include"


def build_emu(outdir, tile=None):
    cxx = shutil.which("g++")
    if cxx is None or not os.path.exists(os.path.join(CUDA_INC, "cuda_fp16.h")):
        pytest.skip("no C++ compiler or CUDA headers")
    so = str(outdir / "libkernels_emu.so")
    extra = [] if tile is None else [f"-DDYN_MESH_TILE={tile}"]
    subprocess.run([cxx, "-std=c++20", "-O1", "-fPIC", "-shared", "-ffp-contract=off",
                    "-I", CUDA_INC] + extra + [os.path.join(HERE, "cpp", "kernels_emu.cpp"),
                                               "-o", so], check=True)
    L = C.CDLL(so)
    vp, i64, i32, f32 = C.c_void_p, C.c_int64, C.c_int, C.c_float
    L.emu_volume.restype = vp
    L.emu_volume.argtypes = [f32, f32, i32, i32, i32, i32]
    L.emu_volume_free.argtypes = [vp]
    L.emu_nalloc.argtypes = [vp]
    L.emu_upload.argtypes = [vp, vp, vp, vp, i64, vp]
    L.emu_download.restype = i64
    L.emu_download.argtypes = [vp, vp, vp]
    L.emu_mesh.restype = i64
    L.emu_mesh.argtypes = [vp, C.POINTER(f32), C.POINTER(f32), vp, i64]
    L.emu_remove.restype = i64
    L.emu_remove.argtypes = [vp, i32, i32, i32, vp, i64, vp, vp, i64]
    L.emu_find.argtypes = [vp, i32, i32, i32]
    L.emu_summaries.argtypes = [vp, vp, vp]
    L.emu_set_free.argtypes = [vp, i32, i32]
    return L


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    return build_emu(tmp_path_factory.mktemp("emu"))


@pytest.fixture(scope="module")
def emu_small_tile(tmp_path_factory):
    """The kernels with a 9-voxel tile: the samples of the top layers of
    cells read the volume instead of shared memory."""
    return build_emu(tmp_path_factory.mktemp("emu9"), tile=9)


@pytest.fixture(scope="module")
def mesh_host(tmp_path_factory):
    f = build_mesh_host(tmp_path_factory.mktemp("mesh"))
    if f is None:
        pytest.skip("no C++ compiler")
    return f


class EmuVolume:
    def __init__(self, L, vs, trunc, nb, bsz, num_blocks, fp16):
        self.L = L
        self.num_blocks = num_blocks
        self.h = L.emu_volume(vs, trunc, nb, bsz, num_blocks, int(fp16))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.emu_volume_free(self.h)

    def upload(self, coords, vox8, stamps=None):
        coords = np.ascontiguousarray(coords, np.int32)
        vox8 = np.ascontiguousarray(vox8, np.uint8)
        st = None if stamps is None else np.ascontiguousarray(stamps, np.int32)
        c = np.zeros(4, np.int64)
        self.L.emu_upload(self.h, coords.ctypes.data, vox8.ctypes.data,
                          None if st is None else st.ctypes.data, len(coords), c.ctypes.data)
        return c

    def download(self):
        n = min(self.L.emu_nalloc(self.h), self.num_blocks)  # as dyn_num_blocks
        c = np.zeros((n, 3), np.int32)
        v = np.zeros((n, 512, 8), np.uint8)
        assert self.L.emu_download(self.h, c.ctypes.data, v.ctypes.data) == n
        return c, v

    def mesh(self, lo, hi, cap=200000):
        lo_c = (C.c_float * 3)(*[float(x) for x in lo])
        hi_c = (C.c_float * 3)(*[float(x) for x in hi])
        out = np.zeros((cap, 3, 6), np.float32)
        n = self.L.emu_mesh(self.h, lo_c, hi_c, out.ctypes.data, cap)
        assert 0 <= n <= cap
        return out[:n]

    def remove(self, mode, last=0, max_age=0, coords=None):
        n = self.L.emu_nalloc(self.h)
        d = np.ascontiguousarray(coords if coords is not None else np.zeros((0, 3)), np.int32)
        oc = np.zeros((n, 3), np.int32)
        ov = np.zeros((n, 512, 8), np.uint8)
        k = self.L.emu_remove(self.h, mode, last, max_age, d.ctypes.data, len(d),
                              oc.ctypes.data, ov.ctypes.data, n)
        assert k >= 0
        return k, oc[:k], ov[:k]


def vox8_of(rgbw, sdf):
    v = np.zeros(rgbw.shape[:2] + (8,), np.uint8)
    v[..., :4] = rgbw
    v[..., 4:] = np.ascontiguousarray(sdf, np.float32)[..., None].view(np.uint8)
    return v


def split8(v8):
    return v8[..., :4], np.ascontiguousarray(v8[..., 4:]).view(np.float32)[..., 0]


@pytest.mark.parametrize("fp16,tile", [(False, 11), (True, 11), (False, 9)])
def test_mesh_kernels_match_host_walk(emu, emu_small_tile, mesh_host, fp16, tile):
    emu = emu if tile == 11 else emu_small_tile
    vs = 0.01
    coords, rgbw, sdf = sphere_volume(7, vs=vs, radius=0.12)
    vol = EmuVolume(emu, vs, 0.04, 1 << 12, 10, len(coords) + 8, fp16)
    assert list(vol.upload(coords, vox8_of(rgbw, sdf))) == [len(coords), 0, 0, 0]
    hc, hv = vol.download()  # heap order; f16-rounded sdf in the mixed form
    h_rgbw, h_sdf = split8(hv)
    # one box, off the voxel grid (the reference-volume test below adds another)
    boxes = [np.array([[-0.123, -0.271, 0.134], [0.22, 0.07, 0.47]], np.float32)]
    for lo, hi in boxes:
        got = vol.mesh(lo, hi)
        want = mesh_host(hc, h_rgbw, h_sdf, vs, lo, hi)
        assert len(got) > 200
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("fp16", [False, True])
def test_evict_kernels_match_host_build(emu, evict_lib, fp16):  # noqa: F811
    coords, vox = blocks(11, 260)
    vox[..., 4:] = np.random.default_rng(12).uniform(-0.03, 0.03, (260, 512, 1)).astype(
        np.float32).view(np.uint8)  # sdf values of a TSDF
    vox[..., 3] = np.minimum(vox[..., 3], 200)
    stamps = np.random.default_rng(13).integers(1, 30, 260).astype(np.int32)
    vol = EmuVolume(emu, 0.01, 0.04, 257, 6, 300, fp16)
    counts = vol.upload(coords, vox, stamps)
    assert counts[0] + counts[2] == 260
    hc, hv = vol.download()
    st = dict(zip(map(tuple, coords.tolist()), stamps.tolist()))
    hst = np.array([st[tuple(c)] for c in hc.tolist()], np.int32)
    host = Host(evict_lib, 257, 6, 300)
    assert host.insert(hc, hv, hst)[0] == len(hc)
    # by age, then by coordinate (with repeats and absent ones)
    for step in range(2):
        if step == 0:
            k1, c1, v1 = vol.remove(0, last=29, max_age=9)
            k2, c2, v2 = host.remove(0, last=29, max_age=9)
        else:
            cur = vol.download()[0]
            dels = np.concatenate([cur[::3], cur[:4], [[500, 500, 500]]]).astype(np.int32)
            k1, c1, v1 = vol.remove(1, coords=dels)
            k2, c2, v2 = host.remove(1, coords=dels)
        assert k1 == k2 > 0
        np.testing.assert_array_equal(c1, c2)
        np.testing.assert_array_equal(v1, v2)
        e, h = vol.download(), host.download()
        np.testing.assert_array_equal(e[0], h[0])
        np.testing.assert_array_equal(e[1], h[1])
        assert host.check() == 0
        for c in c1[:50]:
            assert emu.emu_find(vol.h, *[int(x) for x in c]) == -1
        for i, c in enumerate(e[0][:50]):
            assert emu.emu_find(vol.h, *[int(x) for x in c]) == i
    # streamed back: the removed blocks return (new heap indices from the top)
    counts = vol.upload(c1, v1)
    assert list(counts) == [len(c1), 0, 0, 0]
    e = vol.download()
    assert len(e[0]) == len(h[0]) + len(c1)


def test_upload_counts_heap_exhausted_and_present(emu):
    coords, vox = blocks(21, 15)
    vox[..., 4:] = np.zeros((15, 512, 4), np.uint8)
    vol = EmuVolume(emu, 0.01, 0.04, 64, 4, 10, False)
    assert list(vol.upload(coords, vox)) == [10, 0, 0, 5]
    c, v = vol.download()
    assert len(c) == 10
    assert list(vol.upload(c[:3], v[:3])) == [0, 3, 0, 0]
    # a retry of the keys the heap could not hold reports the heap exhausted
    # again (their entries exist without a block), not "present"
    held = {tuple(x) for x in c.tolist()}
    miss = np.array([i for i, x in enumerate(coords.tolist()) if tuple(x) not in held])
    assert list(vol.upload(coords[miss], vox[miss])) == [0, 0, 0, 5]
    # keys whose block the heap could not hold are found as absent, and go at
    # the next removal; the freed space takes them afterwards
    placed = {tuple(x) for x in c.tolist()}
    for x in coords.tolist():
        assert (emu.emu_find(vol.h, *x) >= 0) == (tuple(x) in placed)
    k, _, _ = vol.remove(1, coords=c[:6])
    assert k == 6
    rest = [x for x in coords.tolist() if tuple(x) not in placed]
    assert list(vol.upload(np.array(rest, np.int32), vox[:len(rest)])) == [len(rest), 0, 0, 0]


def test_upload_places_a_repeated_key_once(emu):
    coords, vox = blocks(22, 3)
    vol = EmuVolume(emu, 0.01, 0.04, 64, 4, 10, False)
    twice = np.concatenate([coords, coords[:1]])
    assert list(vol.upload(twice, np.concatenate([vox, vox[:1]]))) == [3, 1, 0, 0]
    c, _ = vol.download()
    assert sorted(map(tuple, c.tolist())) == sorted(map(tuple, coords.tolist()))


def _nonsat_of(vox8, trunc, fp16):
    """Observed voxels that are not saturated, per block, as the volume
    stores them (FP32: sdf >= trunc (1 - 1e-6); mixed: f16 sdf/trunc == 1)."""
    w = vox8[..., 3]
    sdf = vox8[..., 4:].copy().view(np.float32)[..., 0]
    if fp16:
        h = (sdf / np.float32(trunc)).astype(np.float16)
        sat = h == np.float16(1.0)
    else:
        sat = sdf >= np.float32(trunc * (1.0 - 1e-6))
    return ((w != 0) & ~sat).sum(axis=1)


@pytest.mark.parametrize("fp16", [False, True])
def test_free_space_summaries_follow_upload_and_eviction(emu, fp16):
    """The raycast's free-space summaries (VolumeDev::nonsat / freecell):
    the upload counts each block's observed non-saturated voxels and clears
    the free-cell flags of the lower neighbours of a block that holds any;
    eviction moves both with the blocks and zeroes them above the new heap
    top."""
    trunc = 0.04
    coords = np.array([[x, y, z] for x in range(3) for y in range(3) for z in range(2)], np.int32)
    rng = np.random.default_rng(5)
    n = len(coords)
    vox = np.zeros((n, 512, 8), np.uint8)
    sdf = np.full((n, 512), np.float32(trunc), np.float32)
    w = rng.integers(0, 3, size=(n, 512)).astype(np.uint8)
    surf = rng.random(n) < 0.4  # blocks with some near-surface voxels
    for i in np.nonzero(surf)[0]:
        k = rng.choice(512, 20, replace=False)
        sdf[i, k] = rng.uniform(-trunc, trunc * 0.9, size=20).astype(np.float32)
        w[i, k] = 3
    vox[..., 3] = w
    vox[..., 4:] = sdf.view(np.uint8).reshape(n, 512, 4)
    vol = EmuVolume(emu, 0.01, trunc, 64, 8, 64, fp16)
    # every block's flag set first, as a frame might have left them
    assert list(vol.upload(coords[~surf], vox[~surf])) == [int((~surf).sum()), 0, 0, 0]
    m0 = int((~surf).sum())
    for p in range(m0):
        emu.emu_set_free(vol.h, p, 1)
    assert list(vol.upload(coords[surf], vox[surf])) == [int(surf.sum()), 0, 0, 0]

    def summaries():
        c, v = vol.download()
        ns = np.zeros(len(c), np.int32)
        fc = np.zeros(len(c), np.uint8)
        emu.emu_summaries(vol.h, ns.ctypes.data, fc.ctypes.data)
        return c, v, ns, fc

    c, v, ns, fc = summaries()
    np.testing.assert_array_equal(ns, _nonsat_of(v, trunc, fp16))
    busy = {tuple(x) for x, k in zip(c.tolist(), ns) if k}
    for x, f in zip(c.tolist(), fc):
        reads_busy = any((x[0] + (q & 1), x[1] + ((q >> 1) & 1), x[2] + ((q >> 2) & 1)) in busy
                         for q in range(8))
        if reads_busy:
            assert f == 0, x  # never free where a cell reads a non-saturated voxel
    assert fc.sum() > 0  # some flags survive (blocks with no busy upper neighbour)
    # evict a third: the survivors keep their summaries under their new index
    before = {tuple(x): (k, f) for x, k, f in zip(c.tolist(), ns, fc)}
    k, _, _ = vol.remove(1, coords=c[::3])
    assert k == len(c[::3])
    c2, v2, ns2, fc2 = summaries()
    for x, k_, f in zip(c2.tolist(), ns2, fc2):
        assert (k_, f) == before[tuple(x)]
    np.testing.assert_array_equal(ns2, _nonsat_of(v2, trunc, fp16))


def test_mesh_kernels_reproduce_the_reference_vertices(emu, oracle):
    """The mesh kernels on the volume the reference's own MeshExtractor
    golden was made from (tests/golden/make_mesh_golden.py): the distinct
    vertices of their triangles are the reference's, bit for bit, and the
    triangle count is the reference's."""
    g = np.load(os.path.join(HERE, "golden", "ref_rigid_small.npz"))
    z = np.load(os.path.join(HERE, "golden", "ref_mesh_vertices.npz"))
    from dynamap_b200 import abi
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
    coords, rgbw, sdf = vol.download()
    lo, hi = z["box"]
    # only the blocks the walk can read: its cells span lo .. lo + 2 |hi - lo|
    # (the reference's grid), their samples 1.5 voxels beyond
    vs = float(tsdf.voxel_size)
    a, b = lo - 2 * vs, lo + 2 * np.abs(hi - lo) + 2 * vs
    near = np.all((coords * 8 * vs < b) & ((coords + 1) * 8 * vs > a), axis=1)
    coords, rgbw, sdf = coords[near], rgbw[near], sdf[near]
    ev = EmuVolume(emu, float(tsdf.voxel_size), float(tsdf.truncation_distance),
                   int(tsdf.num_buckets), int(tsdf.bucket_size), int(tsdf.num_blocks), False)
    assert ev.upload(coords, vox8_of(rgbw, sdf))[0] == len(coords)
    tris = ev.mesh(lo, hi)
    assert len(tris) == int(z["triangles"])
    uniq = np.unique(np.ascontiguousarray(tris.reshape(-1, 6)).view(np.uint32), axis=0)
    np.testing.assert_array_equal(uniq, z["vertices"].view(np.uint32))
