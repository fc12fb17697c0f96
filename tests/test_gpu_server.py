"""dyn_server: admission by HBM budget and continuous batching.  Sessions
join and leave at different frames and share steps with changing partners;
each one's poses and map are bit-identical to the same session stepped
alone."""
import numpy as np
import pytest

from dynamap_b200 import abi, configs
from dynamap_b200.session import Server, Session

pytestmark = pytest.mark.gpu


def params():
    out = []
    p = configs.preset("cfg1")
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    out.append((p, abi.PRECISION_FP32, 0))      # joins at step 0
    p = configs.preset("cfg2")
    p["sensor"].update(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5)
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    out.append((p, abi.PRECISION_MIXED, 1))     # joins at step 1
    p = configs.preset("cfg1")
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    p["bilateral"].update(enabled=0)
    out.append((p, abi.PRECISION_MIXED, 3))     # joins at step 3
    p = configs.preset("cfg1")
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    out.append((p, abi.PRECISION_MIXED_BAND, 2))  # band allocation, joins at step 2
    return out


N = 5


@pytest.fixture(scope="module")
def streams():
    out = []
    for i, (p, prec, join) in enumerate(params()):
        seq = configs.sequence(p, seed=70 + i, n_frames=N)
        rgb = getattr(seq, "rgb", None)
        frames = [(seq.depth[k], None if rgb is None else rgb[k]) for k in range(N)]
        out.append((p, prec, join, seq.poses[0].astype(np.float32), frames))
    return out


def sorted_blocks(coords, rgbw, sdf):
    o = np.lexsort((coords[:, 2], coords[:, 1], coords[:, 0]))
    return coords[o], rgbw[o], sdf[o]


def test_results_same_alone_and_in_the_mix(gpu_lib, streams):
    alone = []
    for p, prec, join, pose0, frames in streams:
        t, g, b, s = configs.structs(p)
        with Session(t, g, b, s, precision=prec) as m:
            m.set_pose(pose0)
            poses = [m.process(d, c)[0] for d, c in frames]
            alone.append((poses, sorted_blocks(*m.download_blocks())))
    with Server(budget_bytes=8 << 30) as sv:
        slots = [None] * len(streams)
        done = [0] * len(streams)
        got = [[] for _ in streams]
        step = 0
        while any(d < N for d in done):
            for i, (p, prec, join, pose0, frames) in enumerate(streams):
                if slots[i] is None and step >= join:
                    t, g, b, s = configs.structs(p)
                    slots[i] = sv.admit(t, g, b, s, precision=prec, pose0=pose0)
                    assert slots[i] is not None
                # session 0 sits out step 2: partners change between steps
                if slots[i] is not None and done[i] < N and not (i == 0 and step == 2):
                    d, c = frames[done[i]]
                    assert sv.push(slots[i], d, c)
                    assert not sv.push(slots[i], d, c)  # one frame per slot per step
            n = sv.step()
            assert n > 0
            for i in range(len(streams)):
                if slots[i] is not None and done[i] < N and not (i == 0 and step == 2):
                    got[i].append(sv.result(slots[i])[0])
                    done[i] += 1
            step += 1
        for i in range(len(streams)):
            for k in range(N):
                assert np.array_equal(got[i][k], alone[i][0][k]), (i, k)
            gc, grgbw, gsdf = sorted_blocks(*sv.download_blocks(slots[i]))
            ac, argbw, asdf = alone[i][1]
            np.testing.assert_array_equal(gc, ac)
            np.testing.assert_array_equal(grgbw, argbw)
            np.testing.assert_array_equal(gsdf.view(np.uint32), asdf.view(np.uint32))
        assert sv.usage()["frames"] == len(streams) * N


def test_admission_by_budget(gpu_lib, streams):
    """The server reserves its budget once and carves sessions from it: a
    session is refused when its bytes do not fit, admitted after a release."""
    (p0, prec0), (p1, prec1) = streams[0][:2], streams[1][:2]
    need = []
    with Server(budget_bytes=4 << 30) as sv:
        for p, prec in ((p0, prec0), (p1, prec1)):
            slot = sv.admit(*configs.structs(p), precision=prec)
            need.append(sv.usage()["used_bytes"])
            sv.release(slot)
            assert sv.usage()["used_bytes"] == 0
    with Server(budget_bytes=need[0] + need[1] - 256) as sv:
        a = sv.admit(*configs.structs(p0), precision=prec0)
        assert a is not None
        assert sv.admit(*configs.structs(p1), precision=prec1) is None  # over budget
        u = sv.usage()
        assert u["sessions"] == 1 and u["used_bytes"] == need[0] <= u["budget_bytes"]
        sv.release(a)
        assert sv.usage()["used_bytes"] == 0
        b_ = sv.admit(*configs.structs(p1), precision=prec1)
        assert b_ is not None
        assert not sv.ready(b_)  # nothing stepped yet
        with pytest.raises(abi.DynError):
            sv.result(b_)
        # released space is reused: the first session fits again beside it
        # only if both fit
        assert sv.admit(*configs.structs(p0), precision=prec0) is None
