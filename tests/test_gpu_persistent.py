"""The persistent ICP: one cooperative launch per frame walks every pyramid
level and GN iteration, its blocks meeting at one bounded grid barrier per
iteration.  Its results equal the chained form's (one launch per iteration)
bit for bit -- both sum the same pixel tiles in the same order -- alone and
in a batch, and the barrier's failure paths end in a status, never a hang:
a wait that cannot complete times out after its bound, a grid that cannot
be resident is refused before it runs."""
import os
import subprocess
import sys

import numpy as np
import pytest

from dynamap_b200 import abi, configs

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# Runs in a child process: the chained form is chosen when the library
# loads (DYN_ICP_CHAINED), so each form gets a fresh process.
CHILD = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
from dynamap_b200 import abi, configs
from dynamap_b200.session import Session, Batch
out = sys.argv[2]
rows = []
for name, over, prec in (("cfg1", {}, abi.PRECISION_FP32),
                         ("cfg2", dict(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5),
                          abi.PRECISION_MIXED)):
    p = configs.preset(name)
    p["sensor"].update(over)
    p["tsdf"].update(num_blocks=1 << 15, num_buckets=1 << 16)
    seq = configs.sequence(p, seed=41, n_frames=6)
    t, g, b, s = configs.structs(p)
    with Session(t, g, b, s, precision=prec) as m:
        m.set_pose(seq.poses[0])
        for k in range(6):
            pose, st = m.process(seq.depth[k], None if seq.rgb is None else seq.rgb[k])
            rows.append(np.concatenate([pose.reshape(16), np.array(st.icp_iterations, np.float32)]))
# a batch of both kinds
mix = configs.session_mix(4, 5)
ss = []
seqs = []
for _, p, seed in mix:
    t, g, b, s = configs.structs(p)
    ss.append(Session(t, g, b, s))
    seqs.append(configs.sequence(p, seed=seed, n_frames=5))
for m, q in zip(ss, seqs):
    m.set_pose(q.poses[0])
with Batch(ss) as bt:
    for k in range(5):
        poses, stats, _ = bt.process([q.depth[k] for q in seqs])
        for j in range(len(ss)):
            rows.append(np.concatenate([poses[j].reshape(16),
                                        np.array(stats[j].icp_iterations, np.float32)]))
for m in ss:
    m.close()
np.save(out, np.array(rows, np.float32))
"""


def run_form(tmp_path, chained):
    out = str(tmp_path / f"poses_{int(chained)}.npy")
    env = dict(os.environ)
    if chained:
        env["DYN_ICP_CHAINED"] = "1"
    else:
        env.pop("DYN_ICP_CHAINED", None)
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, out], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return np.load(out)


def test_persistent_equals_chained(tmp_path, gpu_lib):
    a = run_form(tmp_path, chained=False)
    b = run_form(tmp_path, chained=True)
    assert a.shape == b.shape and len(a) > 20
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    assert (a[:, 16:] > 0).any()  # iterations ran


def test_barrier_completes_times_out_and_refuses(gpu_lib):
    assert gpu_lib.dyn_barrier_selftest(0, 64, 0) == abi.DYN_OK
    # a wait that nothing completes: the bound ends it, the device stays usable
    assert gpu_lib.dyn_barrier_selftest(0, 64, 1) == abi.DYN_ERR_TIMEOUT
    assert gpu_lib.dyn_barrier_selftest(0, 8, 0) == abi.DYN_OK
    # more blocks than can be resident at once: refused before it runs
    assert gpu_lib.dyn_barrier_selftest(0, 1 << 20, 0) == 1  # DYN_ERR_INVALID_ARG
    assert gpu_lib.dyn_barrier_selftest(0, 0, 0) == 1
