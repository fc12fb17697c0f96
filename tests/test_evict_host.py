"""Block eviction (dynamap_b200/csrc/evict.cu), built for the host from the
same evict_ops.h steps (tests/cpp/evict_host.cpp), against what removing
blocks means (HashTable::DeleteBlock, hashTable.cu:112-134, applied to each
block): the survivors keep their voxels and are found by lookup, the
removed are gone and handed out with their voxels in heap order, the heap
stays dense with the tail cleared, buckets stay front-packed, and blocks
inserted afterwards (streamed back) take the freed space.  The GPU entry
points are compared with this in test_gpu_evict.py."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
P = C.POINTER


class Host:
    def __init__(self, lib, nb, bsz, num_blocks):
        self.lib = lib
        self.h = lib.evh_create(nb, bsz, num_blocks)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.evh_destroy(self.h)

    @property
    def nalloc(self):
        return self.lib.evh_nalloc(self.h)

    def insert(self, coords, vox, stamps):
        coords = np.ascontiguousarray(coords, np.int32)
        vox = np.ascontiguousarray(vox, np.uint8)
        stamps = np.ascontiguousarray(stamps, np.int32)
        c = np.zeros(4, np.int64)
        self.lib.evh_insert(self.h, coords.ctypes.data, vox.ctypes.data, stamps.ctypes.data,
                            len(coords), c.ctypes.data)
        return c

    def remove(self, mode, last=0, max_age=0, coords=None, cap=1 << 30):
        n = self.nalloc
        d = np.ascontiguousarray(coords if coords is not None else np.zeros((0, 3)), np.int32)
        oc = np.zeros((n, 3), np.int32)
        ov = np.zeros((n, 512, 8), np.uint8)
        k = self.lib.evh_remove(self.h, mode, last, max_age, d.ctypes.data, len(d),
                                oc.ctypes.data, ov.ctypes.data, min(cap, n))
        m = min(k, cap, n)
        return k, oc[:m], ov[:m]

    def download(self):
        n = self.nalloc
        c = np.zeros((n, 3), np.int32)
        v = np.zeros((n, 512, 8), np.uint8)
        self.lib.evh_download(self.h, c.ctypes.data, v.ctypes.data)
        return c, v

    def find(self, xyz):
        return self.lib.evh_find(self.h, *[int(a) for a in xyz])

    def check(self):
        return self.lib.evh_check(self.h)


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    so = str(tmp_path_factory.mktemp("evict") / "libevict_host.so")
    subprocess.run([cxx, "-std=c++17", "-O2", "-fPIC", "-shared",
                    os.path.join(HERE, "cpp", "evict_host.cpp"), "-o", so], check=True)
    L = C.CDLL(so)
    vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int
    L.evh_create.restype = vp
    L.evh_create.argtypes = [i32, i32, i32]
    L.evh_destroy.argtypes = [vp]
    L.evh_nalloc.argtypes = [vp]
    L.evh_insert.argtypes = [vp, vp, vp, vp, i64, vp]
    L.evh_remove.restype = i64
    L.evh_remove.argtypes = [vp, i32, i32, i32, vp, i64, vp, vp, i64]
    L.evh_download.restype = i64
    L.evh_download.argtypes = [vp, vp, vp]
    L.evh_find.argtypes = [vp, i32, i32, i32]
    L.evh_check.argtypes = [vp]
    return L


def blocks(seed, n, span=12):
    """n distinct block coordinates (negative ones included) with random
    voxels."""
    rng = np.random.default_rng(seed)
    pool = np.stack(np.meshgrid(*[np.arange(-span, span)] * 3, indexing="ij"), -1).reshape(-1, 3)
    coords = pool[rng.choice(len(pool), n, replace=False)].astype(np.int32)
    vox = rng.integers(0, 256, size=(n, 512, 8)).astype(np.uint8)
    vox[..., 3] |= 1  # observed
    return coords, vox


def as_map(coords, vox):
    return {tuple(c): v.tobytes() for c, v in zip(coords.tolist(), vox)}


def assert_state(h, want):
    """The host volume holds exactly the blocks of 'want' (coord -> voxels)."""
    assert h.check() == 0
    c, v = h.download()
    assert h.nalloc == len(want) == len(c)
    assert as_map(c, v) == want
    for xyz in list(want)[:200]:
        assert h.find(xyz) >= 0


@pytest.mark.parametrize("nb,bsz", [(4096, 10), (97, 4)])  # roomy / crowded buckets
def test_evict_by_age(lib, nb, bsz):
    coords, vox = blocks(1, 350)
    stamps = np.random.default_rng(2).integers(0, 40, len(coords)).astype(np.int32)
    h = Host(lib, nb, bsz, 400)
    counts = h.insert(coords, vox, stamps)
    placed = counts[0]
    assert counts[0] + counts[2] == len(coords)
    assert h.check() == 0
    c0, v0 = h.download()
    st = {tuple(c): s for c, s in zip(coords.tolist(), stamps)}
    last, age = 39, 12
    k, oc, ov = h.remove(0, last=last, max_age=age)
    gone = [i for i, c in enumerate(c0.tolist()) if last - st[tuple(c)] > age]
    assert 0 < k == len(gone) < placed
    # handed out in heap order, with their voxels
    np.testing.assert_array_equal(oc, c0[gone])
    np.testing.assert_array_equal(ov, v0[gone])
    keep = [i for i in range(len(c0)) if i not in set(gone)]
    assert_state(h, as_map(c0[keep], v0[keep]))
    for c in c0[gone][:100]:
        assert h.find(c) == -1
    # nothing more to evict at the same age; everything at a negative cut
    assert h.remove(0, last=last, max_age=age)[0] == 0
    k2, _, _ = h.remove(0, last=last + 1000, max_age=age)
    assert k2 == len(keep) and h.nalloc == 0
    assert_state(h, {})


def test_delete_and_stream_back(lib):
    coords, vox = blocks(3, 300)
    h = Host(lib, 1024, 6, 320)
    assert h.insert(coords, vox, np.zeros(len(coords), np.int32))[0] == 300
    rng = np.random.default_rng(4)
    sel = rng.choice(300, 90, replace=False)
    absent = np.array([[100, 100, 100], [-50, 7, 3]], np.int32)
    dels = np.concatenate([coords[sel], coords[sel[:10]], absent])  # duplicates, absent
    k, oc, ov = h.remove(1, coords=dels, cap=40)
    assert k == 90 and len(oc) == 40
    order = np.sort(sel)  # heap order = insertion order here
    np.testing.assert_array_equal(oc, coords[order[:40]])
    np.testing.assert_array_equal(ov, vox[order[:40]])
    rest = np.setdiff1d(np.arange(300), sel)
    assert_state(h, as_map(coords[rest], vox[rest]))
    # the removed blocks come back (new heap indices from the top)
    counts = h.insert(coords[sel], vox[sel], np.ones(90, np.int32))
    assert list(counts) == [90, 0, 0, 0]
    assert_state(h, as_map(coords, vox))
    # present keys are left as they are
    assert list(h.insert(coords[:5], vox[5:10], np.ones(5, np.int32))) == [0, 5, 0, 0]
    assert_state(h, as_map(coords, vox))


def test_heap_exhausted_entries_are_dropped(lib):
    coords, vox = blocks(5, 60)
    h = Host(lib, 512, 8, 50)
    counts = h.insert(coords, vox, np.arange(60, dtype=np.int32))
    assert counts[0] == 50 and counts[3] == 10  # keys without a block
    k, _, _ = h.remove(0, last=59, max_age=29)  # stamps 0..29 go
    assert k == 30 and h.nalloc == 20
    assert h.check() == 0
    # the ten keys that never got a block are gone from their buckets too
    for c in coords[50:]:
        assert h.find(c) == -1
    assert list(h.insert(coords[50:], vox[50:], np.zeros(10, np.int32))) == [10, 0, 0, 0]
    assert h.check() == 0 and h.nalloc == 30
