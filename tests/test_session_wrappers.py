"""The Python wrappers of the mesh and eviction entry points
(dynamap_b200/session.py) against a stand-in for the library that keeps a
map of blocks in numpy: arguments, pointers and array layouts as
include/dynamap.h declares them -- 8-byte voxels as {r, g, b, weight, sdf},
18 floats per triangle, counts -- without a GPU."""
import ctypes as C

import numpy as np

from dynamap_b200.session import Session


def arr(ptr, dtype, shape):
    """A numpy view of the memory behind a ctypes pointer argument."""
    addr = ptr.value if isinstance(ptr, C.c_void_p) else C.cast(ptr, C.c_void_p).value
    n = int(np.prod(shape)) * np.dtype(dtype).itemsize
    return np.frombuffer((C.c_char * n).from_address(addr), dtype).reshape(shape)


def setv(ref, v):
    ref._obj.value = v


class FakeLib:
    """Blocks as (coords [n,3] int32, voxels [n,512,8] uint8)."""

    def __init__(self, coords, vox8):
        self.coords = coords.copy()
        self.vox = vox8.copy()

    def dyn_num_blocks(self, h, n):
        setv(n, len(self.coords))
        return 0

    def _out(self, idx, coords_out, vox_out, cap, n_out):
        m = min(len(idx), cap)
        if coords_out is not None and m:
            arr(coords_out, np.int32, (m, 3))[:] = self.coords[idx[:m]]
        if vox_out is not None and m:
            arr(vox_out, np.uint8, (m, 512, 8))[:] = self.vox[idx[:m]]
        setv(n_out, len(idx))
        keep = np.setdiff1d(np.arange(len(self.coords)), idx)
        self.coords, self.vox = self.coords[keep], self.vox[keep]
        return 0

    def dyn_delete_blocks(self, h, coords, m, coords_out, vox_out, cap, n_out):
        want = {tuple(c) for c in arr(coords, np.int32, (m, 3)).tolist()}
        idx = np.array([i for i, c in enumerate(self.coords.tolist()) if tuple(c) in want], int)
        return self._out(idx, coords_out, vox_out, cap, n_out)

    def dyn_evict_blocks(self, h, max_age, coords_out, vox_out, cap, n_out):
        idx = np.arange(0, len(self.coords), 2)  # every other block
        return self._out(idx, coords_out, vox_out, cap, n_out)

    def dyn_upload_blocks(self, h, coords, vox, n, counts):
        self.coords = np.concatenate([self.coords, arr(coords, np.int32, (n, 3))])
        self.vox = np.concatenate([self.vox, arr(vox, np.uint8, (n, 512, 8))])
        c = arr(counts, np.int64, (4,))
        c[:] = [n, 0, 0, 0]
        return 0

    def dyn_download_blocks(self, h, coords_out, vox_out, cap, n_out):
        m = min(cap, len(self.coords))
        arr(coords_out, np.int32, (m, 3))[:] = self.coords[:m]
        arr(vox_out, np.uint8, (m, 512, 8))[:] = self.vox[:m]
        setv(n_out, len(self.coords))
        return 0

    def dyn_extract_mesh(self, h, lo, hi, out, cap, n_out):
        n = 7
        if out is not None and cap:
            t = arr(out, np.float32, (min(cap, n), 18))
            t[:] = np.arange(t.size, dtype=np.float32).reshape(t.shape) + lo[0] + hi[2]
        setv(n_out, n)
        return 0


def fake_session(coords, vox8):
    s = Session.__new__(Session)
    s.lib = FakeLib(coords, vox8)
    s.h = C.c_void_p(1)
    return s


def blocks(n, seed=0):
    rng = np.random.default_rng(seed)
    coords = rng.integers(-50, 50, (n, 3)).astype(np.int32)
    rgbw = rng.integers(0, 256, (n, 512, 4)).astype(np.uint8)
    sdf = rng.uniform(-0.05, 0.05, (n, 512)).astype(np.float32)
    vox8 = np.concatenate([rgbw, sdf[..., None].view(np.uint8)], axis=2)
    return coords, rgbw, sdf, vox8


def test_delete_upload_round_trip_layouts():
    coords, rgbw, sdf, vox8 = blocks(20)
    s = fake_session(coords, vox8)
    c, w, d = s.download_blocks()
    np.testing.assert_array_equal(w, rgbw)
    np.testing.assert_array_equal(d.view(np.uint32), sdf.view(np.uint32))
    out = s.delete_blocks(coords[[3, 7, 11]])
    np.testing.assert_array_equal(out[0], coords[[3, 7, 11]])
    np.testing.assert_array_equal(out[1], rgbw[[3, 7, 11]])
    np.testing.assert_array_equal(out[2].view(np.uint32), sdf[[3, 7, 11]].view(np.uint32))
    assert s.num_blocks() == 17
    assert list(s.upload_blocks(*out)) == [3, 0, 0, 0]
    c, w, d = s.download_blocks()
    np.testing.assert_array_equal(c[-3:], coords[[3, 7, 11]])
    np.testing.assert_array_equal(w[-3:], rgbw[[3, 7, 11]])
    np.testing.assert_array_equal(d[-3:].view(np.uint32), sdf[[3, 7, 11]].view(np.uint32))


def test_evict_counts_and_outputs():
    coords, rgbw, sdf, vox8 = blocks(9, seed=1)
    s = fake_session(coords, vox8)
    assert s.evict_blocks(5, out=False) == 5
    assert s.num_blocks() == 4
    out = s.evict_blocks(5)
    np.testing.assert_array_equal(out[0], coords[[1, 5]])
    np.testing.assert_array_equal(out[1], rgbw[[1, 5]])


def test_extract_mesh_layout():
    s = fake_session(*blocks(1)[::3])
    t = s.extract_mesh([1.0, 0, 0], [0, 0, 2.0])
    assert t.shape == (7, 3, 6) and t.dtype == np.float32
    np.testing.assert_array_equal(t.reshape(7, 18)[0, :3], [3.0, 4.0, 5.0])
    assert s.extract_mesh([1.0, 0, 0], [0, 0, 2.0], capacity=2).shape == (2, 3, 6)


def test_server_evict_syncs_then_evicts_the_slot():
    from dynamap_b200.session import Server
    coords, rgbw, sdf, vox8 = blocks(6, seed=2)
    fake = FakeLib(coords, vox8)
    calls = []
    fake.dyn_server_sync = lambda h: calls.append("sync") or 0

    def session(h, slot, out):
        calls.append(("session", slot))
        out._obj.value = 42
        return 0
    fake.dyn_server_session = session
    sv = Server.__new__(Server)
    sv.lib, sv.h = fake, C.c_void_p(1)
    out = sv.evict_blocks(3, max_age=10)
    assert calls == ["sync", ("session", 3)]
    np.testing.assert_array_equal(out[0], coords[[0, 2, 4]])
    np.testing.assert_array_equal(out[2].view(np.uint32), sdf[[0, 2, 4]].view(np.uint32))
