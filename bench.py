#!/usr/bin/env python
"""Benchmark of the rigid mapping path (one frame = one step).

Workload (default): the 640x480 depth + RGB configuration -- 5 mm voxels,
2^20 hash buckets, 3-level geometric + photometric (weight 0.1) ICP, FP32
TSDF -- on a seeded synthetic sequence (analytic scene, 1 cm / 1 deg per
frame).  Each step tracks one frame against the model, integrates it and
raycasts the next target.

Passes (each on a fresh session replaying the same frames; W warm-up frames
then K timed frames):
  A  device throughput: frames resident in HBM, submitted back to back;
     CUDA events on the session's stream around the K frames -> value.
  B  latency + stages: per-frame submit/result; per-stage CUDA events
     captured inside the frame graph -> p50/p99 and the roofline of the
     dominant kernel.
  C  end to end: frames in pinned host memory through dyn_frame_submit
     (H2D inside) and dyn_frame_result (D2H of pose + counters) -> e2e.
--impl reference times the CPU implementation instead (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "agg frames/s + p50/p99 frame latency vs plain FP32 path; ATE/SDF err vs FP64"
# --precision: the drop-in FP32 form, the mixed form, the mixed form with
# band allocation (values of dyn_precision)
PRECISIONS = {"fp32": 0, "mixed": 1, "band": 2}


def _render_chunk(args):
    from dynamap_b200 import configs, scene
    name, seed, n_frames, idx = args
    p = configs.preset(name) if isinstance(name, str) else name
    s, q = p["sensor"], p["seq"]
    sc = scene.make_scene(seed, q["kind"])
    poses = scene.trajectory(sc, n_frames, seed, q["trans"], q["rot"])
    import numpy as np
    out_d, out_c = [], []
    for i in idx:
        rng = np.random.default_rng(seed * 1000003 + i)
        d, c = scene.render(sc, poses[i], s["rows"], s["cols"], s["fx"], s["fy"], s["cx"],
                            s["cy"], rng, depth_scaler=s["depth_scaler"], with_rgb=q["rgb"],
                            max_range=q.get("max_range", 4.0))
        out_d.append(d)
        out_c.append(c)
    return idx, out_d, out_c, poses


def make_frames(name, seed: int, n_frames: int, workers: int):
    """Render the sequence with a spawn process pool (started before CUDA)."""
    return make_many([(name, seed)], n_frames, workers)[0]


def make_many(jobs, n_frames: int, workers: int):
    """Render several sequences [(preset name or dict, seed)] in one spawn
    process pool; returns [(depth, rgb, poses)]."""
    import concurrent.futures as cf
    import multiprocessing as mp
    import numpy as np
    chunks = [list(range(i, min(i + 8, n_frames))) for i in range(0, n_frames, 8)]
    work = [(j, (name, seed, n_frames, c)) for j, (name, seed) in enumerate(jobs) for c in chunks]
    depth = [[None] * n_frames for _ in jobs]
    rgb = [[None] * n_frames for _ in jobs]
    poses = [None] * len(jobs)
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        for (j, _), (idx, ds, cs, ps) in zip(work, ex.map(_render_chunk, [w for _, w in work])):
            poses[j] = ps
            for i, d, c in zip(idx, ds, cs):
                depth[j][i], rgb[j][i] = d, c
    out = []
    for j in range(len(jobs)):
        out.append((np.stack(depth[j]), np.stack(rgb[j]) if rgb[j][0] is not None else None,
                    poses[j]))
    return out


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during a timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(stage: str, st_avg: dict, P: int, bsz: int, levels_iters, rgb: bool,
                      Sv: int = 8):
    """Bytes a kernel must move per launch (the per-unit figures of the
    design's measurement section), from the run's own counters.  Sv = voxel
    bytes: 8 for the FP32 form, 4 for the mixed form (8 when it keeps
    colour)."""
    if stage == "integrate":
        return st_avg["blocks_visible"] * (16 + 2 * 512 * Sv) + 4 * P + (3 * P if rgb else 0)
    if stage == "raycast":
        return st_avg["blocks_visible"] * 512 * Sv + 4 * P + 32 * P + (3 * P if rgb else 0)
    if stage == "allocate":
        return 4 * P + st_avg["unique_blocks_probed"] * 16 * bsz + 16 * st_avg["blocks_new"]
    if stage == "icp":
        tot = 0
        for Pl, I in levels_iters:
            tot += I * Pl * (32 + 32 + (6 if rgb else 0))
        return tot
    if stage == "bilateral":
        return 2 * P + 4 * P
    if stage == "source_maps" or stage == "target_maps":
        return sum(4 * (P >> (2 * l)) + 16 * (P >> (2 * l)) for l in range(3))
    return None


def read_profile_traffic(kernel: str, st_avg: dict):
    """dram bytes per launch of 'kernel' from an ncu capture summarised in
    profiles/<kernel>_kernel.md ('traffic_bytes_per_launch: N' measured at
    'traffic_units: <counter> U'), scaled to this run's units (the traffic
    grows with the counter: visible blocks for raycast/integrate)."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_kernel.md")
    if not os.path.exists(path):
        return None
    traffic, unit, units = None, None, None
    for ln in open(path):
        ln = ln.strip()
        try:
            if ln.startswith("traffic_bytes_per_launch:"):
                traffic = float(ln.split(":", 1)[1].split()[0])
            elif ln.startswith("traffic_units:"):
                unit, units = ln.split(":", 1)[1].split()[:2]
                units = float(units)
        except (ValueError, IndexError):
            return None
    if traffic is None:
        return None
    if unit and units and unit in st_avg and st_avg[unit] > 0:
        traffic *= st_avg[unit] / units
    return traffic


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(name, depth, rgb, poses, seconds: float = 15.0):
    """The oracle (FP32 restatement, OpenMP on all host threads) on the
    first frames of the same sequence until ~seconds of CPU work."""
    from dynamap_b200 import configs
    from oracle import pyoracle as po
    p = configs.preset(name)
    t, g, b, s = configs.structs(p)
    cores = os.cpu_count() or 1
    po.set_threads(cores)
    S = po.Session(t, g, b, s)
    S.set_pose(poses[0])
    n, t0 = 0, time.perf_counter()
    while n < len(depth):
        S.frame(depth[n], None if rgb is None else rgb[n])
        n += 1
        if time.perf_counter() - t0 > seconds and n >= 2:
            break
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "frames/s", "cores": cores, "kind": "port",
            "sample": f"first {n} frames of the timed sequence ({s.cols}x{s.rows}), "
                      f"oracle FP32 restatement with OpenMP, {dt:.1f} s"}


def accuracy_vs_fp64(p, depth, rgb, poses, n: int, local: int):
    """The forms against the FP64 oracle on the first n frames of the
    sequence.  Tracking: RMS of the per-frame camera-position difference
    from the FP64 oracle's own trajectory (mm).  SDF: every form and the
    oracle integrate the same frames at the ground-truth poses; over the
    voxels observed in both maps, |sdf - sdf64| / truncation (mean, p99,
    max) -- the arithmetic alone, without the tracking differences."""
    import numpy as np
    from dynamap_b200 import abi, configs
    from dynamap_b200.session import Session
    from oracle import pyoracle as po
    t, g, b, s = configs.structs(p)
    po.set_threads(os.cpu_count() or 1)
    c = lambda k: None if rgb is None else rgb[k]
    O = po.Session(t, g, b, s, fp64=True)
    O.set_pose(poses[0])
    ref_poses = []
    for k in range(n):
        O.frame(depth[k], c(k))
        ref_poses.append(O.pose())
    G = po.Session(t, g, b, s, fp64=True)
    for k in range(n):
        G.integrate_with_pose(depth[k], c(k), poses[k])
    oc, orgbw, osdf = G.volume.download()
    index = {tuple(x): i for i, x in enumerate(oc)}
    out = {"frames": n, "oracle": "FP64 restatement (oracle/dynoracle.cpp, double throughout)"}
    for name, prec in (("fp32", abi.PRECISION_FP32), ("mixed", abi.PRECISION_MIXED),
                       ("band", abi.PRECISION_MIXED_BAND)):
        with Session(t, g, b, s, precision=prec, device=local) as m:
            m.set_pose(poses[0])
            track = [m.process(depth[k], c(k), strict=False)[0] for k in range(n)]
        with Session(t, g, b, s, precision=prec, device=local) as m:
            for k in range(n):
                m.integrate_with_pose(depth[k], c(k), poses[k].astype(np.float32))
            gc, grgbw, gsdf = m.download_blocks()
        ate = float(np.sqrt(np.mean([np.sum((a[:3, 3] - r[:3, 3]) ** 2)
                                     for a, r in zip(track, ref_poses)])))
        rows = [(i, index[tuple(x)]) for i, x in enumerate(gc) if tuple(x) in index]
        gi = np.array([r[0] for r in rows], np.int64)
        oi = np.array([r[1] for r in rows], np.int64)
        both = (grgbw[gi, :, 3] > 0) & (orgbw[oi, :, 3] > 0)
        err = np.abs(gsdf[gi].astype(np.float64) - osdf[oi])[both] / t.truncation_distance
        q = (lambda f: float(np.quantile(err, f))) if err.size else (lambda f: None)
        out[name] = {"ate_vs_fp64_mm": 1e3 * ate,
                     "sdf_err_over_trunc": {"mean": float(err.mean()) if err.size else None,
                                            "p99": q(0.99), "max": q(1.0),
                                            "voxels": int(err.size)}}
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    depth, rgb, poses = make_frames(args.config, args.seed, args.warmup + args.steps,
                                    max(1, (os.cpu_count() or 2) - 1))
    from dynamap_b200 import configs
    from oracle import pyoracle as po
    p = configs.preset(args.config)
    t, g, b, s = configs.structs(p)
    cores = os.cpu_count() or 1
    po.set_threads(cores)
    S = po.Session(t, g, b, s)
    S.set_pose(poses[0])
    budget = args.ref_seconds
    # every warm-up frame the run asks for (a frame takes a few seconds)
    for k in range(args.warmup):
        S.frame(depth[k], None if rgb is None else rgb[k])
    n, t0 = 0, time.perf_counter()
    k = args.warmup
    while n < args.steps and k < len(depth):
        S.frame(depth[k], None if rgb is None else rgb[k])
        n += 1
        k += 1
        if time.perf_counter() - t0 > budget:
            break
    dt = time.perf_counter() - t0
    v = n / dt
    line = {"metric": METRIC, "value": v, "unit": "frames/s", "n_gpus": args.gpus,
            "steps": n, "warmup": args.warmup, "ms_per_step": 1e3 * dt / max(n, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": config_block(args, p),
            "cpu_baseline": {"value": v, "unit": "frames/s", "cores": cores, "kind": "port",
                             "sample": f"{n} consecutive frames of the workload after "
                                       f"{args.warmup} warm-up frames (bounded to "
                                       f"~{budget:.0f} s), oracle FP32 restatement, OpenMP"},
            "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_block(args, p):
    s, t = p["sensor"], p["tsdf"]
    return {"workload": f"{args.config}: {s['cols']}x{s['rows']} uint16 depth"
                        f"{' + RGB' if p['seq']['rgb'] else ''}, {t['voxel_size']*1e3:g} mm voxels, "
                        f"2^{int(math.log2(t['num_buckets']))} buckets x {t['bucket_size']}, "
                        f"ICP iters {p['gn']['lvl_iteration_num']} at scales {p['gn']['lvl_scale']}, "
                        f"photometric weight {p['gn']['color_weight']}, "
                        f"{ {'fp32': 'FP32', 'mixed': 'f16/u16 mixed-precision', 'band': 'f16/u16 mixed-precision band-allocated'}[args.precision]} TSDF, "
                        "frame-to-model",
            "sessions_per_gpu": 1, "precision": args.precision, "seed": args.seed,
            "l2": "inputs larger than L2: the TSDF working set (voxel pool "
                  f"{t['num_blocks'] * 4096 / 2**30:.1f} GiB, hash "
                  f"{t['num_buckets'] * t['bucket_size'] * 16 / 2**20:.0f} MiB) exceeds the 126 MB L2"}


_T0 = time.perf_counter()


def note(what: str) -> None:
    """Progress of the run on stderr (the JSON line stays alone on stdout)."""
    print(f"[bench {time.perf_counter() - _T0:7.1f} s] {what}", file=sys.stderr, flush=True)


def run_ours(args):
    import numpy as np

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    nframes = args.warmup + args.steps
    workers = max(1, min(32, ((os.cpu_count() or 2) - 1) // max(world, 1)))
    depth, rgb, poses = make_frames(args.config, args.seed + rank, nframes, workers)
    note("frames rendered")

    import torch
    from dynamap_b200 import abi, configs
    from dynamap_b200.replicas import Ranks
    from dynamap_b200.session import Session
    torch.cuda.set_device(local)
    ranks = Ranks()  # replicas: one independent session per GPU
    p = configs.preset(args.config)
    if args.max_blocks:
        p["tsdf"]["num_blocks"] = min(p["tsdf"]["num_blocks"], args.max_blocks)
    t, g, b, s = configs.structs(p)
    lib = abi.load()
    prec = PRECISIONS[args.precision]
    P = s.rows * s.cols
    has_rgb = rgb is not None
    d_dev = torch.from_numpy(depth).cuda()
    c_dev = torch.from_numpy(rgb).cuda() if has_rgb else None
    fbytes_d, fbytes_c = P * 2, P * 3

    def fptr(tensor, i, nb):
        return tensor.data_ptr() + i * nb

    def barrier():
        torch.cuda.synchronize()
        ranks.barrier()

    max_over_ranks = ranks.max

    import ctypes as C

    def session_stream(m):
        ptr = C.c_void_p()
        abi.check("stream", lib.dyn_session_stream(m.h, C.byref(ptr)))
        return torch.cuda.ExternalStream(ptr.value, device=torch.device("cuda", local))

    note("pass A: device throughput")
    # ---- pass A: device throughput --------------------------------------
    with Session(t, g, b, s, precision=prec, device=local) as m:
        m.set_pose(poses[0])
        stream = session_stream(m)
        for i in range(args.warmup):
            m.submit_device(fptr(d_dev, i, fbytes_d), fptr(c_dev, i, fbytes_c) if has_rgb else None)
            m.result()
        kpf = C.c_int32()
        abi.check("kpf", lib.dyn_session_kernels_per_frame(m.h, C.byref(kpf)))
        barrier()
        clk = ClockSampler(local)
        clk.start()
        time.sleep(0.3)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for i in range(args.warmup, nframes):
            m.submit_device(fptr(d_dev, i, fbytes_d), fptr(c_dev, i, fbytes_c) if has_rgb else None)
        e1.record(stream)
        m.result(strict=False)
        torch.cuda.synchronize()
        elapsed_a = e0.elapsed_time(e1) / 1e3
        clocks = clk.stop()
        final_pose_a = m.pose()
    elapsed_a = max_over_ranks(elapsed_a)
    barrier()

    # ---- the other forms on the same frames (pass A only), for the line's
    # plain-vs-precision comparison
    forms = {}
    if prec == abi.PRECISION_FP32 and args.forms:
        for name, fp in (("mixed", abi.PRECISION_MIXED), ("band", abi.PRECISION_MIXED_BAND)):
            with Session(t, g, b, s, precision=fp, device=local) as m:
                m.set_pose(poses[0])
                st_f = session_stream(m)
                for i in range(args.warmup):
                    m.submit_device(fptr(d_dev, i, fbytes_d),
                                    fptr(c_dev, i, fbytes_c) if has_rgb else None)
                    m.result(strict=False)
                torch.cuda.synchronize()
                f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                f0.record(st_f)
                for i in range(args.warmup, nframes):
                    m.submit_device(fptr(d_dev, i, fbytes_d),
                                    fptr(c_dev, i, fbytes_c) if has_rgb else None)
                f1.record(st_f)
                m.result(strict=False)
                torch.cuda.synchronize()
                el = max_over_ranks(f0.elapsed_time(f1) / 1e3)
                forms[name] = {"value": world * args.steps / el, "unit": "frames/s",
                               "vs_fp32": elapsed_a / el}
        barrier()

    note("pass B: latency and stages")
    # ---- pass B: per-frame latency and stage times ------------------------
    lat_dev, lat_host, stats = [], [], []
    with Session(t, g, b, s, precision=prec, device=local) as m:
        m.set_pose(poses[0])
        abi.check("profile", lib.dyn_session_profile(m.h, 1))
        for i in range(args.warmup):
            m.submit_device(fptr(d_dev, i, fbytes_d), fptr(c_dev, i, fbytes_c) if has_rgb else None)
            m.result()
        ms = (C.c_double * abi.STAGES.__len__())()
        nfr = C.c_int64()
        abi.check("stages", lib.dyn_session_stage_times(m.h, ms, C.byref(nfr), 1))
        barrier()
        track = []
        for i in range(args.warmup, nframes):
            h0 = time.perf_counter()
            m.submit_device(fptr(d_dev, i, fbytes_d), fptr(c_dev, i, fbytes_c) if has_rgb else None)
            pose, st = m.result(strict=False)
            lat_host.append(time.perf_counter() - h0)
            stats.append(st.as_dict())
            track.append(pose.astype(np.float64))
        abi.check("stages", lib.dyn_session_stage_times(m.h, ms, C.byref(nfr), 0))
        stage_ms = {abi.STAGES[k]: ms[k] / max(nfr.value, 1) for k in range(len(abi.STAGES))}
    barrier()

    note("pass C: end to end")
    # ---- pass C: end to end through the host API ---------------------------
    pin_d = torch.from_numpy(depth).pin_memory()
    pin_c = torch.from_numpy(rgb).pin_memory() if has_rgb else None
    d_np = pin_d.numpy()
    c_np = pin_c.numpy() if has_rgb else None
    with Session(t, g, b, s, precision=prec, device=local) as m:
        m.set_pose(poses[0])
        stream = session_stream(m)
        for i in range(args.warmup):
            m.process(d_np[i], c_np[i] if has_rgb else None, strict=False)
        barrier()
        torch.cuda.synchronize()
        h0 = time.perf_counter()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        # two frames in flight: frame k+1 is submitted (its copy overlapping
        # frame k's work) before frame k's result is read
        m.submit(d_np[args.warmup], c_np[args.warmup] if has_rgb else None)
        for i in range(args.warmup + 1, nframes):
            m.submit(d_np[i], c_np[i] if has_rgb else None)
            m.result(strict=False)
        m.result(strict=False)
        e1.record(stream)
        torch.cuda.synchronize()
        elapsed_c_host = time.perf_counter() - h0
    elapsed_c = max_over_ranks(elapsed_c_host)

    # ---- the north star's forms in the same run: the batched configuration
    # (mixed and band against the plain FP32 per-frame path) and a
    # shortened serving run
    batched = serving = None
    if args.batched and prec == abi.PRECISION_FP32:
        note("batched block")
        del d_dev, c_dev, pin_d, pin_c
        torch.cuda.empty_cache()
        batched = measure_batched(args, ranks, local, args.sessions, args.steps, args.warmup,
                                  ["mixed", "band"], e2e=True)
    if args.serving and prec == abi.PRECISION_FP32:
        note("serving block")
        serving = measure_serving(args, ranks, local, args.embed_serve_seconds, "band")

    if rank != 0:
        ranks.close()
        return

    K = args.steps
    value = world * K / elapsed_a
    lat = sorted(x * 1e3 for x in lat_host)
    p50 = lat[len(lat) // 2]
    p99 = lat[min(len(lat) - 1, int(math.ceil(0.99 * len(lat))) - 1)]
    st_avg = {k: float(np.mean([d[k] for d in stats])) for k in
              ("blocks_visible", "unique_blocks_probed", "blocks_new", "blocks_total")}
    iters = np.mean([d["icp_iterations"] for d in stats], axis=0)
    lv = [(P >> (2 * {1: 0, 2: 1, 4: 2, 8: 3}[p["gn"]["lvl_scale"][k]]), iters[k]) for k in range(3)]
    kernel_stages = [k for k in abi.STAGES if k != "frame"]
    dom = max(kernel_stages, key=lambda k: stage_ms[k])
    Sv = 8 if (prec == abi.PRECISION_FP32 or g.color_weight != 0.0) else 4
    alg = algorithmic_bytes(dom, st_avg, P, t.bucket_size, lv, has_rgb, Sv)
    hbm, peak_kind = peaks()
    roof = None
    if alg is not None and stage_ms[dom] > 0:
        ach = alg / (stage_ms[dom] / 1e3) / 1e9
        traffic = read_profile_traffic(dom if prec == abi.PRECISION_FP32 else dom + "_mixed", st_avg)
        roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": ach / hbm, "peak_source": f"{peak_kind} hbm_gbs",
                "algorithmic_bytes_per_launch": alg, "launch_ms": stage_ms[dom],
                "traffic": traffic,
                "traffic_source": (None if traffic is None else
                                   "derived: dram__bytes_read.sum + dram__bytes_write.sum per "
                                   "launch from the ncu capture summarised in profiles/"
                                   f"{dom if prec == abi.PRECISION_FP32 else dom + '_mixed'}"
                                   "_kernel.md, scaled by this run's visible blocks; not "
                                   "measured in this run")}
    # tracking accuracy against the ground truth
    gt = poses[args.warmup:nframes]
    ate = float(np.sqrt(np.mean([np.sum((a[:3, 3] - b_[:3, 3]) ** 2) for a, b_ in zip(track, gt)])))
    note("cpu baseline and FP64 accuracy")
    cpu = cpu_baseline(args.config, depth, rgb, poses, seconds=args.cpu_seconds) \
        if not args.no_cpu else None
    acc = accuracy_vs_fp64(p, depth, rgb, poses, args.fp64_frames, local) \
        if (args.fp64_frames > 0 and rank == 0) else None
    line = {
        "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": 1e3 * elapsed_a / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded analytic scene (floor, box, 3 spheres), ray-cast depth with "
                "sigma(z)=0.0012+0.0019(z-0.4)^2 noise, Perlin albedo RGB",
        "config": config_block(args, p),
        "latency_ms": {"p50": p50, "p99": p99, "what": "host submit->result per frame, pass B"},
        "stages_ms": stage_ms,
        "e2e": {"value": world * K / elapsed_c, "unit": "frames/s",
                "h2d_bytes_per_step": fbytes_d + (fbytes_c if has_rgb else 0),
                "d2h_bytes_per_step": int(lib.dyn_frame_d2h_bytes())},
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": int(kpf.value) * K,
        "kernels_per_frame": int(kpf.value),
        "ate_gt_mm": ate * 1e3,
        "accuracy_vs_fp64": acc,
        "precision_forms": forms or None,
        "batched": batched,
        "serving": serving,
        "map": {"blocks_total": st_avg["blocks_total"], "visible_per_frame": st_avg["blocks_visible"],
                "load_factor": st_avg["blocks_total"] / (t.num_buckets * t.bucket_size)},
    }
    print(json.dumps(line), flush=True)
    ranks.close()


TUNE_FRAMES = 3  # autotuner frames per candidate shape (the first not timed)


def measure_batched(args, ranks, local, n_sessions, steps, warmup, precisions,
                    e2e=True, streams=False, stage_split=False):
    """The batched configuration: n_sessions independent sessions of mixed
    resolution (160x120 / 320x240 / 640x480 at 1:2:1), one frame of every
    session per step, for each precision in 'precisions' as one fused launch
    per stage (dyn_batch, one CUDA graph per frame), beside the plain FP32
    per-frame path on the same GPU: the same sessions driven one frame at a
    time, each waited for before the next (the reference's per-frame loop).
    Each fused batch runs the project's autotuner (dyn_batch_autotune) over
    its warm-up frames: integration grid x raycast tile, then the ICP form
    (persistent grid, half grid, chained kernels), all result-neutral; the
    timed frames use the shape it kept.
    Returns the per-form figures: aggregate frames/s (device-resident
    frames; end to end from pinned host memory with 'e2e'), the speed-up
    over the plain path, and each session's trajectory against the plain
    path's (ATE against the ground truth, and the difference)."""
    import ctypes as C

    import numpy as np
    import torch
    from dynamap_b200 import abi, configs
    from dynamap_b200.session import Batch, Session
    world, rank = ranks.world, ranks.rank
    # the autotuner's candidates (9 launch shapes, then 2 more ICP forms)
    # take TUNE_FRAMES frames each, then the kept shape's graph is captured
    warmup = max(warmup, 11 * TUNE_FRAMES + 2)
    nframes = warmup + steps
    mix = configs.session_mix(n_sessions, nframes, base_seed=100 + 1000 * rank)
    workers = max(1, min(32, ((os.cpu_count() or 2) - 1) // max(world, 1)))
    frames = make_many([(p, seed) for _, p, seed in mix], nframes, workers)
    lib = abi.load()
    structs = [configs.structs(p) for _, p, _ in mix]
    dev_frames = [torch.from_numpy(d).cuda() for d, _, _ in frames]
    nbytes = [d.shape[1] * d.shape[2] * 2 for d, _, _ in frames]
    pinned = [torch.from_numpy(d).pin_memory().numpy() for d, _, _ in frames] if e2e else None
    gt = [poses[warmup:nframes] for _, _, poses in frames]
    n = len(mix)
    # every step's device input pointers, computed before any timed loop
    ptrs = [[dev_frames[j].data_ptr() + k * nbytes[j] for j in range(n)]
            for k in range(nframes)]

    def barrier():
        torch.cuda.synchronize()
        ranks.barrier()

    def timed(fn):
        barrier()
        ts = torch.cuda.Stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ts)
        fn()
        torch.cuda.synchronize()
        e1.record(ts)
        torch.cuda.synchronize()
        return ranks.max(e0.elapsed_time(e1) / 1e3)

    def open_sessions(precision):
        ss = [Session(*st, precision=precision, device=local) for st in structs]
        for m, (_, _, poses) in zip(ss, frames):
            m.set_pose(poses[0])
        return ss

    def ate_mm(track, j):
        return 1e3 * float(np.sqrt(np.mean([np.sum((a[:3, 3] - b_[:3, 3]) ** 2)
                                            for a, b_ in zip(track, gt[j])])))

    # plain per-frame path: FP32, one frame at a time, waited for
    ss = open_sessions(abi.PRECISION_FP32)
    lat = []
    for k in range(warmup):
        for j, m in enumerate(ss):
            m.submit_device(ptrs[k][j])
            m.result(strict=False)
    plain_track = [[] for _ in range(n)]

    def plain():
        for k in range(warmup, nframes):
            for j, m in enumerate(ss):
                h0 = time.perf_counter()
                m.submit_device(ptrs[k][j])
                pose, _ = m.result(strict=False)
                lat.append(time.perf_counter() - h0)
                plain_track[j].append(pose)
    t_plain = timed(plain)
    plain_track = [[a.astype(np.float64) for a in tr] for tr in plain_track]
    for m in ss:
        m.close()
    total = world * n * steps
    lat.sort()
    plain_ate = [ate_mm(plain_track[j], j) for j in range(n)]
    kinds = {}
    for k_, _, _ in mix:
        kinds[k_] = kinds.get(k_, 0) + 1
    out = {"sessions": n, "mix": kinds, "steps": steps, "warmup": warmup,
           "plain": {"fps": total / t_plain, "precision": "fp32",
                     "latency_ms": {"p50": 1e3 * lat[len(lat) // 2],
                                    "p99": 1e3 * lat[min(len(lat) - 1, int(0.99 * len(lat)))]},
                     "ate_gt_mm_mean": float(np.mean(plain_ate))},
           "forms": {}}
    for pname in precisions:
        prec = PRECISIONS[pname]
        ss = open_sessions(prec)
        bt = Batch(ss)
        bt.autotune(TUNE_FRAMES)
        for k in range(warmup):
            bt.submit_device(ptrs[k])
            bt.result(strict=False)
        tuned, tune_ctas, tune_tile = bt.tuning()
        steps_out = []

        def fused_device():
            for k in range(warmup, nframes):
                bt.submit_device(ptrs[k])
                steps_out.append(bt.result(strict=False)[0])
        clk = ClockSampler(local)
        clk.start()
        t_dev = timed(fused_device)
        clocks = clk.stop()
        launches = bt.kernels_per_frame() * steps
        form = {"fps": total / t_dev, "ms_per_step": 1e3 * t_dev / steps,
                "speedup_vs_plain": t_plain / t_dev, "gpu_launches": launches,
                "clocks": clocks,
                "autotuned": {"done": tuned, "integrate_ctas": tune_ctas,
                              "ray_tile": ["16x16", "32x8", "8x8"][tune_tile],
                              "frames_per_candidate": TUNE_FRAMES}}
        if stage_split:
            bt.profile(True)
            for k in range(warmup, min(nframes, warmup + 20)):
                bt.submit_device(ptrs[k])
                bt.result(strict=False)
            ms, nprof = bt.stage_times()
            form["stage_ms_per_step"] = {abi.STAGES[i]: ms[i] / max(nprof, 1)
                                         for i in range(len(abi.STAGES))}
        bt.close()
        for m in ss:
            m.close()
        track = [[st[j].astype(np.float64) for st in steps_out] for j in range(n)]
        ate = [ate_mm(track[j], j) for j in range(n)]
        dpos = [1e3 * max(float(np.linalg.norm(a[:3, 3] - b_[:3, 3]))
                          for a, b_ in zip(track[j], plain_track[j])) for j in range(n)]
        form["ate_gt_mm_mean"] = float(np.mean(ate))
        form["ate_delta_vs_plain_mm"] = {
            "max": float(np.max(np.abs(np.array(ate) - np.array(plain_ate)))),
            "mean": float(np.mean(np.abs(np.array(ate) - np.array(plain_ate))))}
        form["max_position_diff_vs_plain_mm"] = float(np.max(dpos))
        if e2e:
            ss = open_sessions(prec)
            bt = Batch(ss)
            bt.autotune(TUNE_FRAMES)
            for k in range(warmup):
                bt.submit([pinned[j][k] for j in range(n)])
                bt.result(strict=False)

            def fused_e2e():
                for k in range(warmup, nframes):
                    bt.submit([pinned[j][k] for j in range(n)])
                    bt.result(strict=False)
            t_e2e = timed(fused_e2e)
            bt.close()
            for m in ss:
                m.close()
            form["e2e"] = {"value": total / t_e2e, "unit": "frames/s",
                           "h2d_bytes_per_step": int(sum(nbytes)),
                           "d2h_bytes_per_step": int(n * lib.dyn_frame_d2h_bytes())}
        if streams:
            ss = open_sessions(prec)
            handles = (C.c_void_p * n)(*[m.h.value for m in ss])
            for k in range(warmup):
                ptrs = (C.c_void_p * n)(*[pinned[j][k].ctypes.data for j in range(n)])
                abi.check("sessions_submit", lib.dyn_sessions_submit(handles, n, ptrs, None))
                for m in ss:
                    m.result(strict=False)

            def streams_e2e():
                for k in range(warmup, nframes):
                    ptrs = (C.c_void_p * n)(*[pinned[j][k].ctypes.data for j in range(n)])
                    abi.check("sessions_submit", lib.dyn_sessions_submit(handles, n, ptrs, None))
                    for m in ss:
                        m.result(strict=False)
            form["streams_e2e_fps"] = total / timed(streams_e2e)
            for m in ss:
                m.close()
        out["forms"][pname] = form
    del dev_frames
    torch.cuda.empty_cache()
    return out


def run_batched(args):
    """--config cfg3: the batched configuration alone (--precision's form)."""
    import torch
    from dynamap_b200.replicas import Ranks
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ranks = Ranks()  # each GPU runs its own session mix: weak scaling
    r = measure_batched(args, ranks, local, args.sessions, args.steps, args.warmup,
                        [args.precision], e2e=True, streams=True, stage_split=True)
    if ranks.rank != 0:
        ranks.close()
        return
    f = r["forms"][args.precision]
    n, K = r["sessions"], args.steps
    line = {
        "metric": METRIC, "value": f["fps"], "unit": "frames/s", "n_gpus": ranks.world,
        "steps": K, "warmup": args.warmup, "ms_per_step": f["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded analytic scenes, one per session",
        "config": {"workload": f"cfg3: {n} sessions per GPU, resolutions "
                               f"160x120/320x240/640x480 1:2:1 ({r['mix']}), voxels 10/8/5 mm, "
                               "2^18-2^20 buckets, one frame of every session per step, "
                               f"{args.precision}, one fused launch per stage for all "
                               "sessions (dyn_batch), one CUDA graph per frame; plain = "
                               "FP32 sessions one frame at a time",
                   "sessions_per_gpu": n, "precision": args.precision,
                   "l2": "per-step inputs and volumes exceed L2"},
        "plain_fps": r["plain"]["fps"],
        "speedup_vs_plain": f["speedup_vs_plain"],
        "plain_latency_ms": r["plain"]["latency_ms"],
        "ate_delta_vs_plain_mm": f["ate_delta_vs_plain_mm"],
        "step_ms": {"frame_of_all_sessions": f["ms_per_step"]},
        "stage_ms_per_step": f.get("stage_ms_per_step"),
        "streams_e2e_fps": f.get("streams_e2e_fps"),
        "autotuned": f.get("autotuned"),
        "gpu_launches": f["gpu_launches"],
        "clocks": f["clocks"],
        "e2e": f["e2e"],
    }
    print(json.dumps(line), flush=True)
    ranks.close()


def run_large(args):
    """Large-scene stress: one 1280x720 RGB-D session in the 8 x 8 x 3 m room
    (4 mm voxels, 2^23 buckets) stepped in one batch with eight 640x480
    sessions, all in the mixed form with band allocation (--precision).
    value = aggregate frames/s of the batch; the HBM fractions of the
    integration and raycast stages come from the batch's stage times and
    the per-session algorithmic bytes; the large session's hash load factor
    is reported."""
    import numpy as np
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    nframes = args.warmup + args.steps
    from dynamap_b200 import configs
    big = configs.preset("cfg5")
    small = configs.preset("cfg2")
    jobs = [(big, 5000 + rank)] + [(small, 5100 + 10 * rank + i) for i in range(8)]
    workers = max(1, min(32, ((os.cpu_count() or 2) - 1) // max(world, 1)))
    frames = make_many(jobs, nframes, workers)
    import torch
    from dynamap_b200 import abi
    from dynamap_b200.replicas import Ranks
    from dynamap_b200.session import Batch, Session
    torch.cuda.set_device(local)
    ranks = Ranks()
    prec = PRECISIONS[args.precision]
    structs = [configs.structs(p) for p, _ in jobs]
    dev_d = [torch.from_numpy(d).cuda() for d, _, _ in frames]
    dev_c = [torch.from_numpy(c).cuda() for _, c, _ in frames]
    nb_d = [d.shape[1] * d.shape[2] * 2 for d, _, _ in frames]
    nb_c = [3 * d.shape[1] * d.shape[2] for d, _, _ in frames]
    ss = [Session(*st, precision=prec, device=local) for st in structs]
    for m, (_, _, poses) in zip(ss, frames):
        m.set_pose(poses[0])
    n = len(ss)
    bt = Batch(ss)

    def step(k):
        bt.submit_device([dev_d[j].data_ptr() + k * nb_d[j] for j in range(n)],
                         [dev_c[j].data_ptr() + k * nb_c[j] for j in range(n)])
        return bt.result(strict=False)

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    ranks.barrier()
    clk = ClockSampler(local)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ts = torch.cuda.Stream()
    e0.record(ts)
    vis = np.zeros(n)
    stats = None
    exhausted = np.zeros(n, np.int64)  # frames that found the block pool full
    for k in range(args.warmup, nframes):
        _, stats, _ = step(k)
        vis += np.array([st.blocks_visible for st in stats], np.float64)
        exhausted += np.array([st.heap_exhausted > 0 for st in stats], np.int64)
    torch.cuda.synchronize()
    e1.record(ts)
    torch.cuda.synchronize()
    clocks = clk.stop()
    elapsed = ranks.max(e0.elapsed_time(e1) / 1e3)
    # stage split (profiled frames after the timed ones)
    bt.profile(True)
    for k in range(max(args.warmup, nframes - 10), nframes):
        step(k)
    ms, nprof = bt.stage_times()
    stage_ms = {abi.STAGES[i]: ms[i] / max(nprof, 1) for i in range(len(abi.STAGES))}
    bt.close()
    big_blocks = stats[0].blocks_total
    t0s = structs[0][0]
    for m in ss:
        m.close()
    if rank != 0:
        ranks.close()
        return
    K = args.steps
    vis /= K
    hbm = peaks()[0]
    P = [d.shape[1] * d.shape[2] for d, _, _ in frames]
    Sv = 4 if prec != abi.PRECISION_FP32 else 8
    Sv_c = [Sv + (4 if (prec != abi.PRECISION_FP32 and st[1].color_weight != 0.0) else 0)
            for st in structs]
    integ = sum(vis[j] * (16 + 2 * 512 * Sv_c[j]) + 4 * P[j] + 3 * P[j] for j in range(n))
    ray = sum(vis[j] * 512 * Sv_c[j] + 36 * P[j] + 3 * P[j] for j in range(n))
    frac = {}
    for name, alg in (("integrate", integ), ("raycast", ray)):
        t_ = stage_ms[name] / 1e3
        frac[name] = {"algorithmic_bytes_per_step": alg, "ms": stage_ms[name],
                      "achieved_gbs": alg / t_ / 1e9 if t_ > 0 else None,
                      "frac_of_measured_hbm": (alg / t_ / 1e9) / hbm if t_ > 0 else None}
    line = {
        "metric": METRIC, "value": world * n * K / elapsed, "unit": "frames/s", "n_gpus": world,
        "steps": K, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {0: "f32", 1: "f16/u16 voxels", 2: "f16/u16 voxels"}[prec],
        "data": "synthetic: seeded room scene (8 x 8 x 3 m, walls, 40 primitives) and "
                "cube scenes, Perlin albedo RGB",
        "config": {"workload": "cfg5: one 1280x720 RGB-D session (room, 4 mm voxels, 2^23 "
                               "buckets x 10, 2^22 blocks, 8 m range) batched with eight "
                               f"640x480 RGB-D sessions (cfg2), {args.precision}, one frame "
                               "of every session per step",
                   "precision": args.precision, "sessions_per_gpu": n,
                   "l2": "volumes and inputs exceed L2"},
        "stage_ms_per_step": stage_ms,
        "hbm_fraction": frac,
        "large_session": {"blocks_total": int(big_blocks),
                          "pool_blocks": int(t0s.num_blocks),
                          "frames_heap_exhausted": int(exhausted[0]),
                          "voxels": int(big_blocks) * 512,
                          "hash_load_factor": big_blocks / (t0s.num_buckets * t0s.bucket_size),
                          "visible_per_frame": float(vis[0])},
        "clocks": clocks,
        "e2e": {"value": None, "unit": "frames/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": None,
                "note": "device-resident frames; end to end is measured by cfg2/cfg3"},
    }
    print(json.dumps(line), flush=True)
    ranks.close()


def measure_serving(args, ranks, local, seconds, precision, clip_frames=16):
    """The serving configuration: sessions arrive as a Poisson process, are
    admitted by HBM budget into one dyn_server and stream depth at 30 Hz for
    their duration; the host loop pushes every due frame (the newest one when
    a session is behind: older due frames are dropped and counted), steps
    the server whenever frames wait (one fused step for all of them, at most
    two steps in flight) and releases sessions when their stream ends.
    Every session has its own seeded scene and trajectory, rendered as a
    clip of clip_frames frames that its stream replays forth and back.
    Returns frames completed per second of the run and the latency of each
    frame from its due time to the completion of its step."""
    import numpy as np
    import torch
    from dynamap_b200 import configs
    from dynamap_b200.session import Server
    world, rank = ranks.world, ranks.rank
    S = configs.SERVING
    rng = np.random.default_rng(args.seed * 7919 + rank)
    T = float(seconds)
    arrivals = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / S["rate_per_s"])
        if t >= T:
            break
        arrivals.append((t, str(rng.choice(S["kinds"])), float(rng.uniform(*S["duration_s"]))))
    kinds = sorted(set(S["kinds"]))
    workers = max(1, min(32, ((os.cpu_count() or 2) - 1) // max(world, 1)))
    warm = [(configs.serving_kind(k, clip_frames), 500 + i) for i, k in enumerate(kinds)]
    jobs = warm + [(configs.serving_kind(kind, clip_frames), 20000 + 1000 * rank + j)
                   for j, (_, kind, _) in enumerate(arrivals)]
    clips = make_many(jobs, clip_frames, workers)
    # page-locked clips: the server's steps read them directly
    pin = [torch.from_numpy(d).pin_memory() for d, _, _ in clips]
    pin_np = [x.numpy() for x in pin]
    structs = {k: configs.structs(configs.serving_kind(k, clip_frames)) for k in kinds}
    prec = PRECISIONS[precision]
    sv = Server(budget_bytes=int(S["budget_gb"] * 1e9), max_sessions=1024, device=local)
    fps = S["fps"]
    waiting, active = [], {}
    lat, drops, refused_waits, admitted, peak, frames_done = [], 0, 0, 0, 0, 0
    inflight = {}   # slot -> (step id, due time)
    queued = set()  # slots with a frame pushed for the next step
    ai = 0
    # warm-up (untimed): one session of each kind through a few frames, so
    # that module loading and first-launch costs stay out of the run
    for i, kind in enumerate(kinds):
        t_, g_, b_, s_ = structs[kind]
        slot = sv.admit(t_, g_, b_, s_, precision=prec, pose0=clips[i][2][0])
        for k in range(3):
            sv.push(slot, pin_np[i][k])
            sv.step()
            sv.result(slot, strict=False)
        sv.release(slot)
    sv.sync()
    ranks.barrier()
    n_pool = clip_frames
    clk = ClockSampler(local)
    clk.start()
    t0 = time.perf_counter()
    while True:
        now = time.perf_counter() - t0
        while ai < len(arrivals) and arrivals[ai][0] <= now:
            waiting.append((ai,) + arrivals[ai])
            ai += 1
        while waiting:  # FIFO admission
            j, ta, kind, dur = waiting[0]
            t_, g_, b_, s_ = structs[kind]
            clip = len(kinds) + j
            slot = sv.admit(t_, g_, b_, s_, precision=prec, pose0=clips[clip][2][0])
            if slot is None:
                refused_waits += 1
                break
            waiting.pop(0)
            admitted += 1
            active[slot] = dict(kind=kind, clip=clip, start=now, end=now + dur, k=0,
                                last_due=None)
        peak = max(peak, len(active))
        u = sv.usage()
        done_steps = u["steps_done"]
        for slot, (sid, due) in list(inflight.items()):
            if sid < done_steps:
                lat.append(now - due)
                frames_done += 1
                del inflight[slot]
        for slot, a in list(active.items()):
            if slot in queued or slot in inflight:
                continue
            if now >= a["end"]:
                sv.release(slot)
                del active[slot]
                continue
            due_k = int((now - a["start"]) * fps)
            if due_k < a["k"]:
                continue
            drops += due_k - a["k"]  # frames that came due while the slot was busy
            i = due_k % (2 * n_pool - 2)
            i = i if i < n_pool else 2 * n_pool - 2 - i  # forth and back through the clip
            assert sv.push(slot, pin_np[a["clip"]][i])
            a["k"] = due_k + 1
            a["last_due"] = a["start"] + due_k / fps
            queued.add(slot)
        if queued and u["steps"] - done_steps < 2:
            sid = u["steps"]
            sv.step()
            for slot in queued:
                inflight[slot] = (sid, active[slot]["last_due"])
            queued.clear()
        if now >= T and not inflight and not queued:
            break
        if now >= T + 30.0:
            break
        time.sleep(0.0002)
    elapsed = time.perf_counter() - t0
    clocks = clk.stop()
    sv.sync()
    usage = sv.usage()
    sv.close()
    del pin
    tot = (ranks.sum(frames_done), ranks.max(elapsed))
    lat.sort()
    q = lambda f: 1e3 * lat[min(len(lat) - 1, int(f * len(lat)))] if lat else None
    return {"fps": float(tot[0] / tot[1]), "seconds": T, "elapsed_s": elapsed,
            "precision": precision,
            "latency_ms": {"p50": q(0.5), "p99": q(0.99), "max": q(1.0),
                           "what": "frame due time -> step completion seen by the host loop"},
            "frames_completed": int(frames_done), "frames_dropped": int(drops),
            "sessions_admitted": admitted, "sessions_arrived": len(arrivals),
            "sessions_peak": peak, "admission_waits": refused_waits,
            "steps": int(usage["steps"]), "budget_bytes": int(usage["budget_bytes"]),
            "clip_frames": clip_frames, "clocks": clocks}


def run_serving(args):
    """--config cfg4: the serving configuration alone."""
    import torch
    from dynamap_b200 import configs
    from dynamap_b200.replicas import Ranks
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ranks = Ranks()  # each GPU serves its own arrivals: weak scaling
    r = measure_serving(args, ranks, local, args.serve_seconds, args.precision)
    S = configs.SERVING
    if ranks.rank == 0:
        line = {
            "metric": METRIC, "value": r["fps"], "unit": "frames/s",
            "n_gpus": ranks.world, "steps": r["steps"], "warmup": 0,
            "ms_per_step": 1e3 * r["elapsed_s"] / max(1, r["steps"]), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f16/u16 voxels" if PRECISIONS[args.precision] else "f32",
            "data": f"synthetic: every session its own seeded scene and trajectory, a "
                    f"{r['clip_frames']}-frame clip its stream replays forth and back",
            "config": {"workload": f"cfg4: Poisson arrivals {S['rate_per_s']}/s for "
                                   f"{r['seconds']:.0f} s, durations U{list(S['duration_s'])} s, "
                                   f"{S['fps']:.0f} Hz depth, 320x240/640x480/1280x720 at 2:2:1, "
                                   f"84/168/336 MB hash tables, {S['budget_gb']:.0f} GB budget, "
                                   f"{args.precision}",
                       "precision": args.precision, "serve_seconds": r["seconds"]},
            "latency_ms": r["latency_ms"],
            "frames_completed": r["frames_completed"], "frames_dropped": r["frames_dropped"],
            "sessions_admitted": r["sessions_admitted"],
            "sessions_arrived": r["sessions_arrived"], "sessions_peak": r["sessions_peak"],
            "admission_waits": r["admission_waits"], "budget_bytes": r["budget_bytes"],
            "clocks": r["clocks"],
            "e2e": {"value": r["fps"], "unit": "frames/s",
                    "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                    "note": "the serving loop is end to end: host frames in, poses out"},
        }
        print(json.dumps(line), flush=True)
    ranks.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cfg2")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-seconds", type=float, default=90.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-forms", dest="forms", action="store_false",
                    help="skip the mixed / band throughput passes of the default run")
    ap.add_argument("--fp64-frames", type=int, default=8,
                    help="frames scored against the FP64 oracle (0: skip)")
    ap.add_argument("--max-blocks", type=int, default=0,
                    help="cap the voxel-block pool (small profiling runs)")
    ap.add_argument("--sessions", type=int, default=32, help="sessions per GPU (cfg3)")
    ap.add_argument("--serve-seconds", type=float, default=40.0,
                    help="arrival window of the serving run (cfg4)")
    ap.add_argument("--no-batched", dest="batched", action="store_false",
                    help="skip the batched block (cfg3 mix) of the default run")
    ap.add_argument("--no-serving", dest="serving", action="store_false",
                    help="skip the serving block (cfg4, shortened) of the default run")
    ap.add_argument("--embed-serve-seconds", type=float, default=20.0,
                    help="arrival window of the default run's serving block")
    ap.add_argument("--precision", default="fp32", choices=sorted(PRECISIONS),
                    help="fp32: the drop-in path; mixed: f16/u16 voxels, compensated "
                         "normal equations, fast raycast; band: mixed with band-limited "
                         "allocation (no free-space carving)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
    elif args.config == "cfg3":
        run_batched(args)
    elif args.config == "cfg4":
        run_serving(args)
    elif args.config == "cfg5":
        run_large(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
