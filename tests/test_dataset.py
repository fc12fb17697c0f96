"""TUM-layout RGB-D ingest (dynamap_b200.dataset, the reference's
utils::dataSet): 16-bit depth and RGB read back exactly, time order, both
association column orders, folder listing without an association file,
ground truth matched by time stamp, frame selection; on a GPU, a session
tracks the sequence from the files and logs its trajectory."""
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
