"""The streaming front end (include/nodeHandler/nodeHandler.h, the
counterpart of the reference's ROS node, nodeHandler.cpp:170): RGB-D
streams replayed from TUM-layout directories at 30 Hz and one fed through a
pipe go into one server; every frame is reported once, in each stream's
order, and each stream's poses and iteration counts equal the same frames
through a lone Session (the server fuses the streams' frames into shared
launches; a session's results do not depend on its batch)."""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from dynamap_b200 import abi, configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "stream_example.cpp")
LIBDIR = os.path.join(ROOT, "dynamap_b200")


def compile_stream(out):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    subprocess.run([cxx, "-std=c++17", "-O2", "-Wall", "-Werror", "-I",
                    os.path.join(ROOT, "include"), SRC, "-L", LIBDIR, "-ldynamap_b200",
                    f"-Wl,-rpath,{LIBDIR}", "-lz", "-pthread", "-o", out], check=True)


def test_front_end_compiles(tmp_path):
    compile_stream(str(tmp_path / "stream"))


def spec_line(source, p, precision, rate, pose0):
    s, t, g = p["sensor"], p["tsdf"], p["gn"]
    vals = [source, s["rows"], s["cols"], s["fx"], s["fy"], s["cx"], s["cy"], s["depth_scaler"],
            t["voxel_size"], int(np.log2(t["num_buckets"])), t["num_blocks"],
            t["truncation_distance"], t["max_sensor_depth"], g["color_weight"], precision, rate]
    vals += ["%.9g" % v for v in np.asarray(pose0, np.float32).reshape(16)]
    return " ".join(str(v) for v in vals)


def stream_preset(p, color_weight):
    """The parameters stream_example gives a stream (its fixed ICP schedule,
    bilateral filter and depth window)."""
    p = {k: (dict(v) if isinstance(v, dict) else v) for k, v in p.items()}
    p["tsdf"].update(bucket_size=10, block_size=8, max_sdf_weight=64, min_sensor_depth=0.15)
    p["gn"].update(lvl_iteration_num=[10, 5, 4], lvl_scale=[4, 2, 1], color_weight=color_weight,
                   icp_min_depth=0.15, icp_max_depth=p["tsdf"]["max_sensor_depth"], mode=1,
                   compose_left=0, huber_constant=0.3)
    p["bilateral"] = dict(diameter=8, sigma_i=10.0, sigma_s=1.0, enabled=1)
    return p


def pipe_frames(depth, stamps):
    out = bytearray()
    rows, cols = depth.shape[1:]
    for d, st in zip(depth, stamps):
        out += b"DYNF" + struct.pack("<IIIdQ", rows, cols, 0, st, 0)
        out += np.ascontiguousarray(d, np.uint16).tobytes()
    return bytes(out)


@pytest.mark.gpu
def test_streams_through_the_server_equal_lone_sessions(tmp_path, gpu_lib):
    from dynamap_b200.session import Session
    from test_dataset import make_tum
    n = 8
    dirs, seqs, presets, precs = [], [], [], []
    for k, (seed, prec) in enumerate(((31, abi.PRECISION_FP32), (32, abi.PRECISION_MIXED))):
        root = tmp_path / f"seq{k}"
        root.mkdir()
        seq, p = make_tum(root, n=n, seed=seed)
        p["tsdf"].update(num_buckets=1 << 18, num_blocks=1 << 16)
        dirs.append(str(root))
        seqs.append(seq)
        presets.append(stream_preset(p, 0.1))
        precs.append(prec)
    # the pipe stream: 320x240 depth only
    pp = configs.preset("cfg1")
    pp["tsdf"].update(num_buckets=1 << 18, num_blocks=1 << 16)
    pseq = configs.sequence(pp, seed=33, n_frames=n)
    pstamps = [100.0 + 0.0333 * k for k in range(n)]
    presets.append(stream_preset(pp, 0.0))
    precs.append(abi.PRECISION_FP32)
    spec = tmp_path / "spec.txt"
    lines = [spec_line(dirs[0], presets[0], precs[0], 30.0, seqs[0].poses[0]),
             spec_line(dirs[1], presets[1], precs[1], 30.0, seqs[1].poses[0]),
             spec_line("-", presets[2], precs[2], 0.0, pseq.poses[0])]
    spec.write_text("\n".join(lines) + "\n")
    exe = str(tmp_path / "stream")
    compile_stream(exe)
    out = tmp_path / "poses.txt"
    r = subprocess.run([exe, str(spec), str(out)], input=pipe_frames(pseq.depth, pstamps),
                       capture_output=True, timeout=300)
    assert r.returncode == 0, r.stdout.decode() + r.stderr.decode()
    rows = [ln.split() for ln in out.read_text().splitlines()]
    got = {}
    for row in rows:
        got.setdefault(int(row[0]), []).append(row)
    assert sorted(got) == [0, 1, 2] and all(len(v) == n for v in got.values())
    frames = [(seqs[0].depth, seqs[0].rgb, seqs[0].poses[0]),
              (seqs[1].depth, seqs[1].rgb, seqs[1].poses[0]),
              (pseq.depth, None, pseq.poses[0])]
    for sid in range(3):
        rs = got[sid]
        stamps = [float(x[1]) for x in rs]
        assert stamps == sorted(stamps)  # each stream in frame order
        assert all(int(x[2]) == 0 for x in rs)
        t, g, b, s = configs.structs(presets[sid])
        depth, rgb, pose0 = frames[sid]
        with Session(t, g, b, s, precision=precs[sid]) as m:
            m.set_pose(pose0)
            for k in range(n):
                pose, st = m.process(depth[k], None if rgb is None else rgb[k])
                want = np.array([float(v) for v in rs[k][6:22]], np.float32).reshape(4, 4)
                np.testing.assert_array_equal(want, pose, err_msg=f"stream {sid} frame {k}")
                assert [int(v) for v in rs[k][3:6]] == list(st.icp_iterations)
    # the pipe stream's stamps came through
    np.testing.assert_allclose(sorted(float(x[1]) for x in got[2]), pstamps, atol=1e-6)


def write_tum_order(root, seq, order, t0=1305031102.0):
    """A TUM-layout directory whose k-th frame is frame order[k] of seq."""
    import cv2
    from dynamap_b200 import trajectory
    os.makedirs(root / "depth")
    os.makedirs(root / "rgb")
    rows, gt = [], []
    for k, i in enumerate(order):
        td = t0 + 0.0333 * k
        dn, rn = "depth/%.6f.png" % td, "rgb/%.6f.png" % (td + 0.004)
        assert cv2.imwrite(str(root / dn), seq.depth[i].astype(np.uint16))
        assert cv2.imwrite(str(root / rn), np.ascontiguousarray(seq.rgb[i][:, :, ::-1]))
        rows.append((td, dn, td + 0.004, rn))
        gt.append(trajectory.tum_line(td + 0.002, seq.poses[i]))
    (root / "association.txt").write_text("".join("%.6f %s %.6f %s\n" % r for r in rows))
    (root / "groundtruth.txt").write_text("\n".join(gt) + "\n")


@pytest.mark.gpu
def test_eviction_keeps_a_small_pool_from_filling(tmp_path, gpu_lib):
    """A 160x120 RGB stream that moves 3 cm / 2 deg per frame for 12 frames
    and comes back: its map (about 57,000 blocks with free-space carving)
    outgrows a 52,000-block pool on the way out, while one frame touches
    about 41,000 blocks and two frames in a row at most about 43,600.
    Without a policy frames report the heap exhausted; with eviction (above
    85 % of the pool, blocks untouched for more than 1 frame) every frame
    succeeds, blocks go to the host and come back when the camera returns,
    and the trajectory stays within 5 mm of a session whose pool holds
    everything."""
    from dynamap_b200.session import Session
    p = configs.preset("cfg2")
    p["sensor"].update(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5)
    p["seq"].update(trans=0.03, rot=2.0)
    p["tsdf"].update(num_buckets=1 << 18, num_blocks=52000)
    seq = configs.sequence(p, seed=31, n_frames=12)
    order = list(range(12)) + list(range(10, -1, -1))
    root = tmp_path / "seq"
    root.mkdir()
    write_tum_order(root, seq, order)
    pp = stream_preset(p, 0.1)
    spec = tmp_path / "spec.txt"
    spec.write_text(spec_line(str(root), pp, abi.PRECISION_FP32, 0.0, seq.poses[0]) + "\n")
    exe = str(tmp_path / "stream")
    compile_stream(exe)
    runs = {}
    for name, extra in (("plain", []), ("evict", ["--evict", "0.85", "1", "0.1"])):
        out = tmp_path / f"{name}.txt"
        r = subprocess.run([exe, str(spec), str(out)] + extra, capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        runs[name] = ([ln.split() for ln in out.read_text().splitlines()], r.stdout)
    plain_status = [int(x[2]) for x in runs["plain"][0]]
    assert abi.DYN_ERR_HEAP_EXHAUSTED in plain_status
    rows, stdout = runs["evict"]
    assert len(rows) == len(order) and all(int(x[2]) == 0 for x in rows), \
        " ".join(x[2] for x in rows) + " | " + stdout
    c = [ln.split() for ln in stdout.splitlines() if ln.startswith("counts")][0]
    evictions, evicted, uploaded = int(c[2]), int(c[3]), int(c[4])
    assert evictions > 0 and evicted > 0 and uploaded > 0, c
    # the same frames through a session whose pool holds the whole map
    big = dict(pp)
    big["tsdf"] = dict(pp["tsdf"], num_blocks=1 << 17)
    t, g, b, s = configs.structs(big)
    with Session(t, g, b, s) as m:
        m.set_pose(seq.poses[0])
        ref = [m.process(seq.depth[i], seq.rgb[i])[0] for i in order]
    got = [np.array([float(v) for v in x[6:22]], np.float32).reshape(4, 4) for x in rows]
    diff = max(float(np.linalg.norm(a[:3, 3] - r_[:3, 3])) for a, r_ in zip(got, ref))
    assert diff < 5e-3, diff


@pytest.mark.gpu
def test_streams_beyond_the_budget_take_turns(tmp_path, gpu_lib):
    """Two 160x120 RGB streams under a budget that holds one session, with
    parking on: stream A replays frames 0-7 of its sequence, then stream B
    its 8 frames, then A frames 8-15.  B starts parked; its first frame
    parks A (A's blocks to host memory, its slot released) and admits B;
    A's return parks B and resumes A with its blocks uploaded back.  Every
    frame succeeds; A's frames before the first park equal a run whose
    budget holds both streams bit for bit; A's first frame after the resume
    holds at least the blocks it had before it was parked; and A's poses
    after the resume (the first of its frames integrated at its last pose
    without tracking) stay within 3 cm of the run that never parks."""
    from dynamap_b200.session import Server
    p = configs.preset("cfg2")
    p["sensor"].update(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5)
    p["tsdf"].update(num_buckets=1 << 16, num_blocks=1 << 15)
    seq_a = configs.sequence(p, seed=41, n_frames=16)
    seq_b = configs.sequence(p, seed=42, n_frames=8)
    write_tum_order(tmp_path / "a1", seq_a, range(8))
    write_tum_order(tmp_path / "a2", seq_a, range(8, 16), t0=1305031102.0 + 0.0333 * 8)
    write_tum_order(tmp_path / "b", seq_b, range(8), t0=1305031202.0)
    pp = stream_preset(p, 0.1)
    with Server(budget_bytes=4 << 30) as sv:
        slot = sv.admit(*configs.structs(pp), precision=abi.PRECISION_FP32)
        need = sv.usage()["used_bytes"]
        sv.release(slot)
    budget = int(need * 1.01) + (1 << 20)  # one session (and the visible list), not two
    spec = tmp_path / "spec.txt"
    spec.write_text(
        spec_line(f"{tmp_path / 'a1'},{tmp_path / 'a2'}", pp, abi.PRECISION_FP32, 0.0,
                  seq_a.poses[0]) + "\n" +
        spec_line(str(tmp_path / "b"), pp, abi.PRECISION_FP32, 0.0, seq_b.poses[0]) + "\n")
    exe = str(tmp_path / "stream")
    compile_stream(exe)
    runs = {}
    for name, extra in (("park", ["--park", str(budget), "--sequential"]),
                        ("roomy", ["--park", str(8 << 30), "--sequential"])):
        out = tmp_path / f"{name}.txt"
        r = subprocess.run([exe, str(spec), str(out)] + extra, capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        rows = [ln.split() for ln in out.read_text().splitlines()]
        counts = {int(c[1]): [int(v) for v in c[2:]] for c in
                  (ln.split() for ln in r.stdout.splitlines() if ln.startswith("counts"))}
        runs[name] = (rows, counts)
    rows, counts = runs["park"]
    assert len(rows) == 24 and all(int(x[2]) == 0 for x in rows), [x[2] for x in rows]
    a = [x for x in rows if x[0] == "0"]
    b = [x for x in rows if x[0] == "1"]
    assert len(a) == 16 and len(b) == 8
    # counts: evictions evicted uploaded stored parks resumes restored
    assert counts[0][4] == 1 and counts[0][5] == 1 and counts[0][6] > 0, counts
    assert counts[1][4] == 1 and counts[1][5] == 1, counts
    assert runs["roomy"][1][0][4] == 0 and runs["roomy"][1][1][4] == 0, runs["roomy"][1]
    assert int(a[8][22]) >= int(a[7][22]), (a[7][22], a[8][22])
    ref = [x for x in runs["roomy"][0] if x[0] == "0"]
    pose = lambda x: np.array([float(v) for v in x[6:22]], np.float32).reshape(4, 4)
    for k in range(8):
        np.testing.assert_array_equal(pose(a[k]), pose(ref[k]), err_msg=f"frame {k}")
    diff = max(float(np.linalg.norm(pose(a[k])[:3, 3] - pose(ref[k])[:3, 3]))
               for k in range(8, 16))
    assert diff < 0.03, diff


def test_parking_policy_against_a_stand_in_server(tmp_path):
    """The front end's parking and eviction policies without a GPU: the C
    ABI's serving calls answered by tests/cpp/fake_server.cpp (built, like
    the driver, with AddressSanitizer and UBSan where the compiler has
    them); tests/cpp/park_fake.cpp runs two streams taking turns under a
    budget for one session (frames, poses, restored blocks, park / resume /
    admission counts) and a stream whose map outgrows its pool (eviction
    counts: every evicted block stored or uploaded back)."""
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    lib = tmp_path / "libfakedyn.so"
    exe = tmp_path / "park_fake"
    inc = os.path.join(ROOT, "include")
    san = ["-O1", "-g", "-fsanitize=address,undefined"]
    probe = subprocess.run([cxx, "-x", "c++", "-", "-o", str(tmp_path / "probe")] + san,
                           input="int main(){return 0;}", text=True, capture_output=True)
    if probe.returncode != 0:
        san = ["-O2"]
    subprocess.run([cxx, "-std=c++17", "-Wall", "-Werror", "-fPIC", "-shared", "-I", inc] + san +
                   [os.path.join(ROOT, "tests", "cpp", "fake_server.cpp"), "-o", str(lib)],
                   check=True)
    subprocess.run([cxx, "-std=c++17", "-Wall", "-Werror", "-I", inc] + san +
                   [os.path.join(ROOT, "tests", "cpp", "park_fake.cpp"), "-L", str(tmp_path),
                    "-lfakedyn", f"-Wl,-rpath,{tmp_path}", "-pthread", "-o", str(exe)],
                   check=True)
    for _ in range(3):
        r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr
