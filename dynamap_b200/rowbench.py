"""Timing of the calls around the per-frame path: mesh extraction
(dyn_extract_mesh) and block eviction / streaming (dyn_delete_blocks,
dyn_evict_blocks, dyn_upload_blocks), on a map built by tracking a
synthetic sequence of a preset (cfg2 by default: 640x480 RGB-D, 5 mm
voxels).  Each call is synchronous, so it is timed on the host around the
call: what a caller waits for, device work and copies included.

  python -m dynamap_b200.rowbench --row mesh  [--config cfg2] [--frames 60] [--reps 5]
  python -m dynamap_b200.rowbench --row evict [--config cfg2] [--frames 60] [--reps 5]

One JSON line per row."""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import abi, configs


def build_map(config: str, frames: int, seed: int, precision: int):
    from .session import Session
    p = configs.preset(config)
    seq = configs.sequence(p, seed=seed, n_frames=frames)
    t, g, b, s = configs.structs(p)
    m = Session(t, g, b, s, precision=precision)
    m.set_pose(seq.poses[0].astype(np.float32))
    for k in range(frames):
        m.process(seq.depth[k], seq.rgb[k] if seq.rgb is not None else None, strict=False)
    return m, t, p


def timed(fn, reps: int):
    fn()  # warm-up (first-call allocations)
    ms = []
    for _ in range(reps):
        t0 = time.perf_counter()
        out = fn()
        ms.append((time.perf_counter() - t0) * 1e3)
    return float(np.median(ms)), out


def row_mesh(args, m, t, p):
    coords = m.download_blocks()[0]
    vs = t.voxel_size
    lo = coords.min(axis=0) * 8 * vs - vs
    hi = (coords.max(axis=0) + 1) * 8 * vs + vs
    ms_count, _ = timed(lambda: m.extract_mesh(lo, hi, capacity=0), args.reps)
    ms_full, tri = timed(lambda: m.extract_mesh(lo, hi), args.reps)
    return {"row": "mesh", "workload": f"{args.config}: map of {args.frames} tracked frames, "
            f"box over all allocated blocks", "blocks": int(len(coords)),
            "triangles": int(len(tri)), "ms_count_only": ms_count,
            "ms_extract": ms_full, "triangles_per_s": len(tri) / (ms_full * 1e-3),
            "blocks_per_s": len(coords) / (ms_count * 1e-3)}


def row_evict(args, m, t, p):
    coords, rgbw, sdf = m.download_blocks()
    n = len(coords)
    sel = coords[np.random.default_rng(args.seed).choice(n, n // 4, replace=False)]
    ms_del, ms_up = [], []
    for _ in range(args.reps + 1):
        t0 = time.perf_counter()
        out = m.delete_blocks(sel)
        t1 = time.perf_counter()
        counts = m.upload_blocks(*out)
        t2 = time.perf_counter()
        assert counts[0] == len(sel)
        ms_del.append((t1 - t0) * 1e3)
        ms_up.append((t2 - t1) * 1e3)
    t0 = time.perf_counter()
    aged = m.evict_blocks(args.max_age, out=False)
    ms_age = (time.perf_counter() - t0) * 1e3
    d, u = float(np.median(ms_del[1:])), float(np.median(ms_up[1:]))
    return {"row": "evict", "workload": f"{args.config}: map of {args.frames} tracked frames, "
            f"a quarter of its blocks deleted (streamed out) and uploaded back",
            "blocks": int(n), "moved_blocks": int(len(sel)), "ms_delete_stream_out": d,
            "ms_upload": u, "blocks_per_s_delete": len(sel) / (d * 1e-3),
            "blocks_per_s_upload": len(sel) / (u * 1e-3),
            "evict_by_age": {"max_age": args.max_age, "removed": int(aged), "ms": ms_age}}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--row", choices=["mesh", "evict"], required=True)
    ap.add_argument("--config", default="cfg2")
    ap.add_argument("--frames", type=int, default=60)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--max-age", type=int, default=20)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "mixed"])
    args = ap.parse_args(argv)
    prec = abi.PRECISION_FP32 if args.precision == "fp32" else abi.PRECISION_MIXED
    m, t, p = build_map(args.config, args.frames, args.seed, prec)
    with m:
        line = (row_mesh if args.row == "mesh" else row_evict)(args, m, t, p)
    line["precision"] = args.precision
    print(json.dumps(line))


if __name__ == "__main__":
    main()
