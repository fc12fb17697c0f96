"""dyn_icp_normal_equations_noalloc: the ICP normal equations for callers
that cannot allocate device memory (a host that reserves its GPU memory up
front and forbids cudaMalloc later, e.g. a real-time executor running the
tracker inside its control loop).  Its scratch is a fixed device array
inside the library, so it must give the same sums as the allocating entry
point dyn_icp_normal_equations -- within the tolerance of the parity tests
(1e-6 relative) -- on consecutive calls, since every call reuses (and must
re-initialise) that array.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from dynamap_b200 import abi, configs

pytestmark = pytest.mark.gpu


def _level_inputs(oracle, seq, s, b, scale, k_src, k_tgt):
    ls = oracle.level_sensor(s, scale)

    def level(depth):
        d = oracle.bilateral(oracle.depth_from_raw(depth, s.depth_scaler), b)
        while d.shape[0] > ls.rows:
            d = oracle.downsample_depth(d)
        return d

    sd, td = level(seq.depth[k_src]), level(seq.depth[k_tgt])
    _, sn = oracle.maps(sd, ls)
    _, tn = oracle.maps(td, ls)
    T = (np.linalg.inv(seq.poses[k_tgt]) @ seq.poses[k_src]).astype(np.float32)
    return ls, sd, sn, td, tn, T


def _call(lib, fn, dev, ls, g, T):
    out = (C.c_double * 29)()
    Tc = (C.c_float * 16)(*T.reshape(16).tolist())
    st = getattr(lib, fn)(dev[0].data_ptr(), dev[1].data_ptr(), None, dev[2].data_ptr(),
                          dev[3].data_ptr(), None, C.byref(ls), C.byref(g), Tc, out, None)
    abi.check(fn, st)
    return np.array(out)


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls(gpu_lib, oracle):
    import torch
    p = configs.preset("cfg1")
    seq = configs.sequence(p, seed=6, n_frames=3)
    t, g, b, s = configs.structs(p)
    cases = [_level_inputs(oracle, seq, s, b, 1, 1, 0),   # full resolution
             _level_inputs(oracle, seq, s, b, 4, 2, 1),   # coarse level, other frames
             _level_inputs(oracle, seq, s, b, 1, 1, 0)]   # the first again
    results = []
    for ls, sd, sn, td, tn, T in cases:
        dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (sd, sn, td, tn)]
        ref = _call(gpu_lib, "dyn_icp_normal_equations", dev, ls, g, T)
        got = _call(gpu_lib, "dyn_icp_normal_equations_noalloc", dev, ls, g, T)
        assert ref[28] > 100
        assert got[28] == ref[28]
        np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-9 * np.abs(ref).max())
        results.append(got)
    # the third call repeats the first: the shared array left no trace
    np.testing.assert_array_equal(results[0], results[2])


def test_noalloc_rejects_levels_beyond_its_capacity(gpu_lib):
    t, g, b, s = abi.defaults()
    big = abi.Sensor(rows=2048, cols=2048, fx=1000.0, fy=1000.0, cx=1023.5, cy=1023.5,
                     depth_scaler=1000.0)
    out = (C.c_double * 29)()
    Tc = (C.c_float * 16)(*np.eye(4, dtype=np.float32).reshape(16).tolist())
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    st = gpu_lib.dyn_icp_normal_equations_noalloc(dummy, dummy, None, dummy, dummy, None,
                                                  C.byref(big), C.byref(g), Tc, out, None)
    assert st == 1  # DYN_ERR_INVALID_ARG


def test_noalloc_checks_levels_as_the_allocating_entry_point_does(gpu_lib):
    """A 1 x 2,000,000 level fits the array but is not a sensor either entry
    point accepts (sides are limited to 8192): both reject it."""
    t, g, b, s = abi.defaults()
    thin = abi.Sensor(rows=1, cols=2_000_000, fx=500.0, fy=500.0, cx=0.0, cy=0.0,
                      depth_scaler=1000.0)
    out = (C.c_double * 29)()
    Tc = (C.c_float * 16)(*np.eye(4, dtype=np.float32).reshape(16).tolist())
    dummy = C.c_void_p(16)  # never dereferenced: the level check comes first
    for fn in ("dyn_icp_normal_equations", "dyn_icp_normal_equations_noalloc"):
        st = getattr(gpu_lib, fn)(dummy, dummy, None, dummy, dummy, None, C.byref(thin),
                                  C.byref(g), Tc, out, None)
        assert st == 1, fn  # DYN_ERR_INVALID_ARG
