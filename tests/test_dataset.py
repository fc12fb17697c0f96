"""TUM-layout RGB-D ingest (dynamap_b200.dataset, the reference's
utils::dataSet): 16-bit depth and RGB read back exactly, time order, both
association column orders, folder listing without an association file,
ground truth matched by time stamp, frame selection; the C++ drop-in
(include/utils/dataSet.h) decodes the same pixels and poses, and its PNG
reader every filter type; on a GPU, a session (Python) and the builder
(C++) track the sequence from the files and log the trajectory."""
import os

import numpy as np
import pytest

from dynamap_b200 import configs, dataset, trajectory

cv2 = pytest.importorskip("cv2")


def make_tum(root, n=6, seed=21, association="depth-first"):
    p = configs.preset("cfg2")
    p["sensor"].update(rows=120, cols=160, fx=131.25, fy=131.25, cx=79.5, cy=59.5)
    seq = configs.sequence(p, seed=seed, n_frames=n)
    os.makedirs(root / "depth")
    os.makedirs(root / "rgb")
    t0 = 1305031102.0
    rows = []
    for k in range(n):
        td, tr = t0 + 0.0333 * k, t0 + 0.0333 * k + 0.004
        dn, rn = "depth/%.6f.png" % td, "rgb/%.6f.png" % tr
        assert cv2.imwrite(str(root / dn), seq.depth[k].astype(np.uint16))
        assert cv2.imwrite(str(root / rn), np.ascontiguousarray(seq.rgb[k][:, :, ::-1]))
        rows.append((td, dn, tr, rn))
    if association == "depth-first":
        (root / "association.txt").write_text(
            "# depth rgb\n" + "".join("%.6f %s %.6f %s\n" % r for r in rows))
    elif association == "rgb-first":
        (root / "association.txt").write_text(
            "".join("%.6f %s %.6f %s\n" % (r[2], r[3], r[0], r[1]) for r in rows))
    # ground truth at slightly different stamps, one extra line
    (root / "groundtruth.txt").write_text(
        "# timestamp tx ty tz qx qy qz qw\n" +
        "".join(trajectory.tum_line(t0 + 0.0333 * k + 0.002, seq.poses[k]) + "\n"
                for k in range(n)) +
        trajectory.tum_line(t0 + 99.0, np.eye(4)) + "\n")
    return seq, p


@pytest.mark.parametrize("association", ["depth-first", "rgb-first", "none"])
def test_frames_read_back(tmp_path, association):
    seq, _ = make_tum(tmp_path, association=association)
    ds = dataset.TumDataset(str(tmp_path))
    assert len(ds) == len(seq.depth)
    stamps = [fr.stamp for fr in ds]
    assert stamps == sorted(stamps)
    for k, fr in enumerate(ds):
        assert fr.depth.dtype == np.uint16
        np.testing.assert_array_equal(fr.depth, seq.depth[k])
        np.testing.assert_array_equal(fr.rgb, seq.rgb[k])
        assert fr.gt_pose is not None
        np.testing.assert_allclose(fr.gt_pose, seq.poses[k], atol=4e-4)


def test_selection_and_missing_gt(tmp_path):
    seq, _ = make_tum(tmp_path, n=7)
    ds = dataset.TumDataset(str(tmp_path), first=1, last=6, skip=2)
    assert [fr.index for fr in ds] == [0, 1, 2]
    np.testing.assert_array_equal(ds[1].depth, seq.depth[3])
    os.remove(tmp_path / "groundtruth.txt")
    assert dataset.TumDataset(str(tmp_path))[0].gt_pose is None


def test_missing_folder(tmp_path):
    with pytest.raises(FileNotFoundError):
        dataset.TumDataset(str(tmp_path))


@pytest.mark.gpu
def test_session_tracks_from_files(tmp_path, gpu_lib):
    from dynamap_b200.session import Session
    seq, p = make_tum(tmp_path, n=8)
    t, g, b, s = configs.structs(p)
    log = tmp_path / "est.txt"
    with Session(t, g, b, s) as m:
        st, est = dataset.run_session(m, dataset.TumDataset(str(tmp_path)), str(log))
    gst, gt = trajectory.read_tum(str(log))
    assert len(gst) == len(seq.depth)
    np.testing.assert_allclose(gst, np.round(st, 4), atol=1e-9)
    e = trajectory.ate(est, seq.poses, aligned=False)
    assert e["rmse"] < 0.02


# --- the C++ drop-in (include/utils/dataSet.h) -------------------------------

@pytest.fixture(scope="module")
def cpp_reader(tmp_path_factory):
    import shutil
    import subprocess
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "dynamap_b200")
    exe = str(tmp_path_factory.mktemp("cpp") / "dataset_example")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "dataset_example.cpp"), "-L", libdir,
                    "-ldynamap_b200", f"-Wl,-rpath,{libdir}", "-lz", "-o", exe], check=True)
    return exe


def _png_bytes(img, bits, filters):
    """A PNG file of img (rows x cols [x channels]) written with the given
    filter type per row, so every filter the format has is exercised."""
    import struct
    import zlib
    a = np.asarray(img)
    ch = 1 if a.ndim == 2 else a.shape[2]
    color = {1: 0, 3: 2, 4: 6}[ch]
    rows, cols = a.shape[:2]
    raw = (a.astype(">u2") if bits == 16 else a.astype(np.uint8)).tobytes()
    stride = cols * ch * bits // 8
    bpp = ch * bits // 8
    out = bytearray()
    prev = np.zeros(stride, np.int32)
    for r in range(rows):
        cur = np.frombuffer(raw[r * stride:(r + 1) * stride], np.uint8).astype(np.int32)
        left = np.concatenate([np.zeros(bpp, np.int32), cur[:-bpp]])
        ul = np.concatenate([np.zeros(bpp, np.int32), prev[:-bpp]])
        ft = filters[r % len(filters)]
        if ft == 0:
            pred = np.zeros_like(cur)
        elif ft == 1:
            pred = left
        elif ft == 2:
            pred = prev
        elif ft == 3:
            pred = (left + prev) // 2
        else:
            p = left + prev - ul
            pa, pb, pc = np.abs(p - left), np.abs(p - prev), np.abs(p - ul)
            pred = np.where((pa <= pb) & (pa <= pc), left, np.where(pb <= pc, prev, ul))
        out.append(ft)
        out += ((cur - pred) & 0xFF).astype(np.uint8).tobytes()
        prev = cur

    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d))
    return (b"\x89PNG\r\n\x1a\n" +
            chunk(b"IHDR", struct.pack(">IIBBBBB", cols, rows, bits, color, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(bytes(out), 6)) + chunk(b"IEND", b""))


@pytest.mark.parametrize("kind", ["gray16", "gray8", "rgb8", "rgba8"])
def test_cpp_png_every_filter(tmp_path, kind, cpp_reader):
    import subprocess
    exe = cpp_reader
    rng = np.random.default_rng(3)
    shape = {"gray16": (37, 23), "gray8": (37, 23), "rgb8": (37, 23, 3),
             "rgba8": (37, 23, 4)}[kind]
    bits = 16 if kind == "gray16" else 8
    img = rng.integers(0, 1 << bits, size=shape).astype(np.uint16 if bits == 16 else np.uint8)
    img[5:15] = img[4]  # runs, where Up and Paeth predict exactly
    src = tmp_path / ("%s.png" % kind)
    src.write_bytes(_png_bytes(img, bits, [0, 1, 2, 3, 4, 4, 3, 2, 1]))
    # the encoder itself is checked by OpenCV
    np.testing.assert_array_equal(
        cv2.imread(str(src), cv2.IMREAD_UNCHANGED),
        img if img.ndim == 2 else img[:, :, [2, 1, 0, 3][:img.shape[2]]])
    out = tmp_path / "out.bin"
    subprocess.run([exe, "--png", str(src), str(out)], check=True)
    b = out.read_bytes()
    hdr = np.frombuffer(b[:16], np.int32)
    ch = 1 if img.ndim == 2 else img.shape[2]
    assert list(hdr) == [shape[0], shape[1], ch, bits]
    got = np.frombuffer(b[16:], ">u2" if bits == 16 else np.uint8).reshape(shape)
    np.testing.assert_array_equal(got, img)


def test_cpp_png_rejects_what_it_cannot_read(tmp_path, cpp_reader):
    import subprocess
    exe = cpp_reader
    bad = tmp_path / "bad.png"
    bad.write_bytes(b"not a png at all")
    r = subprocess.run([exe, "--png", str(bad), str(tmp_path / "o")], capture_output=True)
    assert r.returncode != 0
    pal = tmp_path / "pal.png"  # 16-bit RGB is outside what TUM recordings use
    pal.write_bytes(_png_bytes(np.zeros((4, 4, 3), np.uint16), 16, [0]))
    r = subprocess.run([exe, "--png", str(pal), str(tmp_path / "o")], capture_output=True)
    assert r.returncode != 0 and b"unsupported" in r.stderr


@pytest.mark.parametrize("association", ["depth-first", "rgb-first", "none"])
def test_cpp_dataset_matches_python_reader(tmp_path, association, cpp_reader):
    import subprocess
    exe = cpp_reader
    root = tmp_path / "seq"
    root.mkdir()
    seq, _ = make_tum(root, association=association)
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([exe, str(root), str(out)], capture_output=True, text=True, check=True)
    lines = r.stdout.splitlines()
    py = list(dataset.TumDataset(str(root)))
    assert len(lines) == len(py) == len(seq.depth)
    for k, (ln, fr) in enumerate(zip(lines, py)):
        v = ln.split()
        assert float(v[0]) == pytest.approx(fr.stamp, abs=1e-6)
        rows, cols = int(v[1]), int(v[2])
        assert (rows, cols) == fr.depth.shape
        d = np.fromfile(out / ("depth_%d.bin" % k), np.uint16).reshape(rows, cols)
        c = np.fromfile(out / ("rgb_%d.bin" % k), np.uint8).reshape(rows, cols, 3)
        np.testing.assert_array_equal(d, seq.depth[k])
        np.testing.assert_array_equal(c, seq.rgb[k])
        assert v[3] == "1"
        pose = np.array([float(x) for x in v[4:]], np.float32).reshape(4, 4)
        np.testing.assert_array_equal(pose, fr.gt_pose)


@pytest.mark.gpu
def test_cpp_builder_tracks_from_files(tmp_path, cpp_reader, gpu_lib):
    """builder::buildModelLS(dataSet&) over the files, the reference driver's
    loop, logging with builder::writePoseToTxt."""
    import subprocess
    root = tmp_path / "seq"
    root.mkdir()
    seq, p = make_tum(root, n=8)
    s = p["sensor"]
    log = tmp_path / "est.txt"
    r = subprocess.run([cpp_reader, "--track", str(root), str(log)] +
                       [str(s[k]) for k in ("rows", "cols", "fx", "fy", "cx", "cy",
                                            "depth_scaler")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    st, est = trajectory.read_tum(str(log))
    want = [fr.stamp for fr in dataset.TumDataset(str(root))]
    np.testing.assert_allclose(st, np.round(want, 4), atol=1e-9)
    e = trajectory.ate(est, seq.poses, aligned=False)
    assert e["rmse"] < 0.02


def test_prefixed_layout_python_and_cpp(tmp_path, cpp_reader):
    """Another layout (the reference's depthPrefix / rgbPrefix, e.g.
    depth_N.png / color_N.png with frame numbers): both readers list the
    frames in numeric order (not name order) and read them alike."""
    import subprocess
    root = tmp_path / "seq"
    (root / "depth").mkdir(parents=True)
    (root / "rgb").mkdir()
    rng = np.random.default_rng(9)
    n = 12
    depth = rng.integers(0, 4000, (n, 24, 32)).astype(np.uint16)
    rgb = rng.integers(0, 256, (n, 24, 32, 3)).astype(np.uint8)
    for k in range(n):  # numbers whose name order is not their order
        num = [3, 10, 1, 25, 7, 100, 2, 50, 8, 9, 11, 4][k]
        cv2.imwrite(str(root / "depth" / f"depth_{num}.png"), depth[k])
        cv2.imwrite(str(root / "rgb" / f"color_{num}.png"), rgb[k][:, :, ::-1])
        (root / "rgb" / f"other_{num}.txt").write_text("not a frame")
    order = np.argsort([3, 10, 1, 25, 7, 100, 2, 50, 8, 9, 11, 4], kind="stable")
    ds = dataset.TumDataset(str(root), depth_prefix="depth_", rgb_prefix="color_")
    assert [fr.stamp for fr in ds] == sorted([3, 10, 1, 25, 7, 100, 2, 50, 8, 9, 11, 4])
    for fr, k in zip(ds, order):
        np.testing.assert_array_equal(fr.depth, depth[k])
        np.testing.assert_array_equal(fr.rgb, rgb[k])
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([cpp_reader, str(root), str(out), "depth_", "color_"], capture_output=True,
                       text=True, check=True)
    lines = r.stdout.splitlines()
    assert [float(ln.split()[0]) for ln in lines] == [fr.stamp for fr in ds]
    for i, k in enumerate(order):
        d = np.fromfile(out / f"depth_{i}.bin", np.uint16).reshape(24, 32)
        c = np.fromfile(out / f"rgb_{i}.bin", np.uint8).reshape(24, 32, 3)
        np.testing.assert_array_equal(d, depth[k])
        np.testing.assert_array_equal(c, rgb[k])
