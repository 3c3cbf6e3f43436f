#!/usr/bin/env python
"""Headline benchmark: absolute-pose RANSAC frames/s on 1 B200 (replicas on N).

Workload (one "step"): the batched configuration -- 256 synthetic frames of
uneven size (N log-uniform in [500, 30000], inlier ratio U[0.10, 0.80], pixel
noise U[0.5, 2] px, 4 px threshold, 1000 samples per round, the reference's
adaptive stop rule, LM refinement) estimated in one CUDA-graph launch with the
inputs resident in device memory. L2 is flushed (256 MiB write) before every
timed step. Each rank of a multi-GPU run estimates its own 256 frames (frames
are independent: replicas, no collective on the path).

Also reported on the same frames: the end-to-end public call with host buffers
(e2e), a loop of plain per-frame calls (the reference's calling pattern),
success rate at 5 deg / 5 cm, per-kernel device times from CUDA events, the
FP32 roofline of the scoring kernel, and the FP64 CPU oracle on the host cores.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "frames/s & p50/p99 ms at >=99% success: served-batched vs plain call, 1 B200"
WORKLOAD = ("batched: 256 frames/GPU, N log-uniform [500,30000], inlier ratio U[0.10,0.80], "
            "sigma U[0.5,2] px, 640x480 f=525, 4 px, 1000 samples/round, p=0.9999, LM")
FLOP_PER_PAIR = 27  # projection 9 FMA, reciprocal, 2 residual FMA, r^2, score add


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=256)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--hr", type=int, default=0, help="scoring hypotheses per thread (4/8, 0 = auto)")
    ap.add_argument("--tensor", action="store_true",
                    help="score with the tensor-core shape (8192-point chunks) instead of autotuning")
    ap.add_argument("--case", default="", choices=["", "plain", "scoring", "batch64", "precision"],
                    help="scoring: one N=20000 frame, exactly 4096 samples; batch64: the batched workload's "
                         "first 64 frames in one graph (small cases for ncu)")
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        import datetime
        backend = "nccl"
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, v: float, device) -> float:
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.p = None
        # Raw samples: a temporary file unless TBR_CLOCKS_DIR names a directory to keep them in.
        import tempfile
        self.path = os.path.join(os.environ.get("TBR_CLOCKS_DIR", tempfile.gettempdir()), f"clocks_gpu{gpu}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(self.gpu), "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
            # The sampler is running (its first sample is in) before the timed region starts.
            t0 = time.time()
            while time.time() - t0 < 2.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.01)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.strip().split(", ") for r in open(self.path) if r.strip()]
        except Exception:
            rows = []
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(float(r[3]) for r in rows if len(r) > 3)}


def success(results, frames):
    from turboransac_b200 import scenes
    ok = 0
    for r, f in zip(results, frames):
        ae, te = scenes.pose_error(scenes.quat_to_rotmat(r["q"]), r["t"], f.R_gt, f.t_gt)
        ok += (ae < 5.0 and te < 5.0)
    return ok / len(frames)


def cpu_baseline(frames, seconds_target=15.0):
    """FP64 oracle (same algorithm, same samples) over frames with all host threads."""
    from oracle.oracle import Oracle
    o = Oracle()
    cores = os.cpu_count() or 1
    # Calibrate on a few frames, then size the sample to ~seconds_target.
    t0 = time.perf_counter()
    o.estimate_batch(frames[:cores], threads=cores)
    dt = time.perf_counter() - t0
    per_frame_wall = dt / min(len(frames), cores)
    m = int(max(cores, min(len(frames), seconds_target / max(per_frame_wall, 1e-6))))
    m = min(m, len(frames))
    sample = frames[:m]
    t0 = time.perf_counter()
    oq, ot, osmp = o.estimate_batch(sample, threads=cores)
    dt = time.perf_counter() - t0
    # one core, on a smaller sample (~5 s)
    m1 = int(max(1, min(len(frames), 5.0 / max(per_frame_wall * cores, 1e-6))))
    t0 = time.perf_counter()
    o.estimate_batch(frames[:m1], threads=1)
    dt1 = time.perf_counter() - t0
    model = ""
    try:
        model = next(l.split(":", 1)[1].strip() for l in open("/proc/cpuinfo") if l.startswith("model name"))
    except Exception:
        pass
    return {"value": m / dt, "unit": "frames/s", "cores": cores, "kind": "port",
            "sample": f"first {m} frames of the batched workload, FP64 oracle, {cores} threads over frames",
            "seconds": dt, "one_core": {"value": m1 / dt1, "frames": m1}, "cpu_model": model}, (oq, ot, osmp)


def precision_vs_oracle(frames, res, oracle_out):
    """Deviation of the GPU poses from the FP64 oracle's on the same frames and
    samples (the oracle run timed as the CPU baseline)."""
    import numpy as np
    oq, ot, osmp = oracle_out
    m = len(oq)
    rep = precision_report(frames[:m], res[:m], oq, ot)["all"]
    rep["frames"] = m
    rep["same_sample_count"] = float(np.mean([int(res[i]["samples"]) == int(osmp[i]) for i in range(m)]))
    rep["bar"] = "1e-6 rad / 1e-6 m against the FP64 CPU pipeline on identical Philox samples"
    return rep


def config0_plain(ctx, reps=3):
    """Plain single frames (N=2000, 40 % inliers, the reference's call): latency."""
    import numpy as np

    from turboransac_b200 import BundleOptions_cuda, Camera_cuda, RansacOptions_cuda, scenes
    ro = RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)
    frames = [scenes.plain_frame(i) for i in range(64)]
    lat, gpu, ok = [], [], 0
    for rep in range(1 + reps):
        for f in frames:
            t0 = time.perf_counter()
            st, pose, _ = ctx.estimate_absolute_pose(f.uv, f.xyz, Camera_cuda(1, 640, 480, list(f.K)), ro,
                                                     BundleOptions_cuda(), seed=f.seed)
            dt = 1000.0 * (time.perf_counter() - t0)
            if rep:
                lat.append(dt)
                gpu.append(st.details["gpu_ms"])
                ae, te = scenes.pose_error(pose.R(), pose.t, f.R_gt, f.t_gt)
                ok += (ae < 5.0 and te < 5.0)
    return {"config": "plain frame: N=2000, 40 % inliers, sigma 1 px, 4 px, 1000 samples/round, p=0.9999",
            "calls": len(lat), "frames_per_s": len(lat) / (sum(lat) / 1000.0),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "gpu_p50_ms": float(np.percentile(gpu, 50)), "success_rate": ok / len(lat)}


def config1_scoring(ctx, reps=5, hr=0):
    """Scoring-bound single frame: N=20000, 15 % inliers, exactly 4096 samples."""
    from turboransac_b200 import BundleOptions_cuda, Camera_cuda, RansacOptions_cuda, scenes
    f = scenes.scoring_frame(0)
    ro = RansacOptions_cuda(max_iterations=4096, max_reproj_error=4.0)
    cam = Camera_cuda(1, 640, 480, list(f.K))
    ms = []
    for i in range(2 + reps):
        st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, cam, ro, BundleOptions_cuda(), seed=f.seed,
                                                   force_samples=4096, hyp_per_thread=hr)
        if i >= 2:
            ms.append(st.details["gpu_ms"])
    d = st.details
    pairs = d["hypotheses"] * f.n
    return {"config": "scoring-bound frame: N=20000, 15 % inliers, exactly 4096 samples (early stop off)",
            "samples": d["samples"], "hypotheses": d["hypotheses"], "pairs": pairs,
            "gpu_ms_per_call": statistics.mean(ms), "pairs_per_s": pairs / (statistics.mean(ms) / 1000.0),
            "candidate_overflow": d["candidate_overflow"]}


def run_serving(ctx, seconds, rate=2000.0, pool=600, budget=8 << 30, shape=None):
    """Config 4: Poisson stream of independent frames (N log-uniform [300, 50000],
    inlier ratio U[0.05, 0.70], 1 px noise) through the continuous-batching server."""
    import threading

    import numpy as np

    from turboransac_b200 import Server, scenes
    from turboransac_b200._lib import TbrError
    reqs = [scenes.serving_request(i) for i in range(pool)]
    arrivals = scenes.poisson_arrivals(rate, seconds, seed=11)
    srv = Server(ctx, budget_bytes=budget, max_slots=1024, scoring_shape=shape)
    # warm the server (first steps pay one-time costs)
    for r in reqs[:32]:
        srv.submit(r)
    srv.drain()
    srv.poll()
    done, lock = {}, threading.Lock()
    stop = threading.Event()

    def poller():
        while not stop.is_set():
            got = srv.poll()
            if got:
                t = time.perf_counter()
                with lock:
                    for g in got:
                        done[g["id"]] = (g, t)
            else:
                time.sleep(0.0005)

    th = threading.Thread(target=poller, daemon=True)
    th.start()
    ids = {}
    t0 = time.perf_counter()
    for k, ta in enumerate(arrivals):
        while True:
            dt = t0 + ta - time.perf_counter()
            if dt <= 0:
                break
            time.sleep(min(dt, 0.001))
        while True:
            try:
                ids[srv.submit(reqs[k % pool])] = k % pool
                break
            except TbrError as e:  # queue full: back off until the server drains
                if "CAPACITY" not in str(e):
                    raise
                time.sleep(0.001)
    srv.drain()
    t_end = time.perf_counter()
    time.sleep(0.01)
    stop.set()
    th.join()
    for g in srv.poll():
        done[g["id"]] = (g, t_end)
    sst = srv.stats()
    srv.close()
    lat = np.array([g["latency_ms"] for g, _ in done.values()])
    ok = 0
    for rid, (g, _) in done.items():
        f = reqs[ids[rid]]
        ae, te = scenes.pose_error(scenes.quat_to_rotmat(g["q"]), g["t"], f.R_gt, f.t_gt)
        ok += (g["status"] == 0 and ae < 5.0 and te < 5.0)
    last = max(t for _, t in done.values())
    return {"offered_rate_hz": rate, "seconds": seconds, "requests": len(arrivals), "completed": len(done),
            "throughput_fps": len(done) / (last - t0), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "p999_ms": float(np.percentile(lat, 99.9)),
            "success_rate": ok / max(len(done), 1), "budget_bytes": budget,
            "mean_resident": sst["resident_sum"] / max(sst["steps"], 1), "steps": sst["steps"],
            "device_wait_ms": sst["device_wait_ms"], "host_ms": sst["host_stage_ms"] + sst["host_retire_ms"]
            + sst["host_launch_ms"],
            "workload": "N log-uniform [300,50000], w U[0.05,0.70], sigma 1 px, Poisson arrivals"}, reqs


def run_plain_serving(ctx, reqs, count=200):
    """The reference's calling pattern on the serving distribution: synchronous plain calls."""
    import numpy as np

    from turboransac_b200 import BundleOptions_cuda, Camera_cuda, RansacOptions_cuda
    ro = RansacOptions_cuda(max_iterations=1000, success_prob=0.9999, max_reproj_error=4.0)
    lat = []
    for f in reqs[:count]:
        t0 = time.perf_counter()
        ctx.estimate_absolute_pose(f.uv, f.xyz, Camera_cuda(1, 640, 480, list(f.K)), ro, BundleOptions_cuda(),
                                   seed=f.seed)
        lat.append(1000.0 * (time.perf_counter() - t0))
    return {"frames_per_s": len(lat) / (sum(lat) / 1000.0), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "frames": len(lat)}


def run_serving_capacity(ctx, reqs, repeats=10, budget=8 << 30, shape=None):
    """Served throughput at saturation: the serving requests submitted at once
    (repeats x the pool), completion rate of the continuous-batching server."""
    import numpy as np

    from turboransac_b200 import Server, scenes
    srv = Server(ctx, budget_bytes=budget, max_slots=1024, scoring_shape=shape)
    for r in reqs[:32]:
        srv.submit(r)
    srv.drain()
    srv.poll()
    pairs0 = srv.stats()["pairs_scored"]
    ids = {}
    t0 = time.perf_counter()
    for _ in range(repeats):
        for k, r in enumerate(reqs):
            ids[srv.submit(r)] = k
    srv.drain()
    dt = time.perf_counter() - t0
    got = []
    while True:
        g = srv.poll()
        if not g:
            break
        got += g
    sst = srv.stats()
    srv.close()
    lat = np.array([g["latency_ms"] for g in got])
    ok = 0
    for g in got:
        f = reqs[ids[g["id"]]]
        ae, te = scenes.pose_error(scenes.quat_to_rotmat(g["q"]), g["t"], f.R_gt, f.t_gt)
        ok += (g["status"] == 0 and ae < 5.0 and te < 5.0)
    return {"frames_per_s": len(got) / dt, "requests": len(got), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "success_rate": ok / max(len(got), 1),
            "load": f"{repeats} x {len(reqs)} serving requests submitted at once", "seconds": dt,
            "pairs_scored_per_s": (sst["pairs_scored"] - pairs0) / dt,
            "server": {"steps": sst["steps"], "mean_resident": sst["resident_sum"] / max(sst["steps"], 1),
                       "device_wait_ms": sst["device_wait_ms"], "host_stage_ms": sst["host_stage_ms"],
                       "host_retire_ms": sst["host_retire_ms"], "host_launch_ms": sst["host_launch_ms"]}}


def run_reference(args, world, rank):
    """--impl reference: the CPU implementation of the path on the host cores."""
    if rank != 0:
        return
    from turboransac_b200 import scenes
    frames = scenes.batched_frames(args.frames)
    from oracle.oracle import Oracle
    o = Oracle()
    cores = os.cpu_count() or 1
    # Every step estimates all frames of the workload (the same frames, seeds and
    # samples as the GPU arm). If a step is slow on this host, fewer warm-up
    # steps keep the run within a few minutes; the timed steps are all run.
    times = []
    t_start = time.perf_counter()
    warm = args.warmup
    i = 0
    while len(times) < args.steps:
        t0 = time.perf_counter()
        o.estimate_batch(frames, threads=cores)
        dt = time.perf_counter() - t0
        if i >= warm:
            times.append(dt)
        elif (args.warmup + args.steps) * dt > 240.0:
            warm = min(warm, 1)
        i += 1
    fps = len(frames) * len(times) / sum(times)
    rcuda = reference_cuda_build(frames, args)
    line = {"metric": METRIC, "value": fps, "unit": "frames/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": min(warm, i - len(times)), "ms_per_step": 1000.0 * statistics.mean(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "global_batch": len(frames), "parallelism": "host threads"},
            "impl": "reference", "same_config": True,
            "cpu_baseline": {"value": fps, "unit": "frames/s", "cores": cores, "kind": "port",
                             "sample": f"all {len(frames)} frames of the batched workload per step, "
                                       f"FP64 oracle (same algorithm, same samples), {cores} threads over frames",
                             "seconds_total": time.perf_counter() - t_start},
            "e2e": {"value": fps, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_cuda": rcuda}
    print(json.dumps(line), flush=True)


def reference_cuda_build(frames, args):
    """The reference's own CUDA build (its src/*.cu for sm_100a) on this GPU: one
    estimate_absolute_pose_cuda call per frame, as its evaluator loops, on the
    batched workload and on plain single frames (N=2000, 40 % inliers)."""
    import numpy as np
    import torch

    from oracle import refcuda
    from turboransac_b200 import scenes
    if not refcuda.available():
        return {"unavailable": "oracle/_ref/tbr_refcuda not built (make -C oracle refcuda needs the reference tree)"}
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}

    def measure(fr):
        r = refcuda.run(fr, warmup=8)
        ok = [scenes.pose_error(scenes.quat_to_rotmat(q), t, f.R_gt, f.t_gt) for f, q, t in zip(fr, r["q"], r["t"])]
        return {"frames": len(fr), "frames_per_s": len(fr) / (float(r["ms"].sum()) / 1000.0),
                "p50_ms": float(np.percentile(r["ms"], 50)), "p99_ms": float(np.percentile(r["ms"], 99)),
                "success_rate": float(np.mean([a < 5.0 and b < 5.0 for a, b in ok]))}

    sk = refcuda.scoring_kernel(scenes.scoring_frame(0))
    sk["config"] = "scoring-bound frame (N=20000, 15 % inliers): one round of 4096 samples, kernel only"
    return {"build": "reference src/entry.cu, turbo_ransac.cu, ba.cu, nvcc sm_100a -O3 -rdc=true",
            "timing": "host clock around each call; the reference's stdout sent to /dev/null",
            "batched_workload": measure(frames),
            "plain_frame": measure([scenes.plain_frame(i) for i in range(64)]),
            "scoring_kernel": sk}


def run_case_plain(args):
    """Plain single frames (N=2000, 40 % inliers, the reference's call): latency."""
    from turboransac_b200 import Context
    ctx = Context(0, 1 << 30)
    print(json.dumps(dict(case="plain", **config0_plain(ctx, reps=max(1, args.steps // 5)))), flush=True)
    ctx.close()


def run_case_scoring(args):
    """Scoring-bound single frame: N=20000, 15 % inliers, exactly 4096 samples."""
    from turboransac_b200 import Context
    ctx = Context(0, 2 << 30)
    print(json.dumps(dict(case="scoring", **config1_scoring(ctx, reps=args.steps, hr=args.hr))), flush=True)
    ctx.close()


def run_case_batch64(args):
    """First 64 frames of the batched workload, one captured graph per step."""
    from turboransac_b200 import Batch, Context, RansacOptions_cuda, scenes
    frames = scenes.batched_frames(64)
    ctx = Context(0, 2 << 30)
    if args.tensor:  # the tensor-core shape, as the main bench's --tensor
        b = Batch(ctx, frames, RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0), points_per_iter=128,
                  chunk_points=8192)
        best = {"forced": "tensor-core shape, 8192-point chunks"}
    else:
        b = Batch(ctx, frames, RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0))
        best, _ = b.autotune(repeats=2)  # the shape the main bench would take (graph launches only)
    ms = []
    for i in range(args.warmup + args.steps):
        b.run()
        b.sync()
        if i >= args.warmup:
            ms.append(b.results()[0]["gpu_ms"])
    # One host-stepped run (the kernels of the captured graph, launched one by
    # one): per-kernel CUDA-event times, and launches a profiler can attach to.
    prof, pairs = b.profile()
    print(json.dumps({"case": "batch64", "frames": 64, "scoring_shape": best, "ms_per_batch": statistics.mean(ms),
                      "frames_per_s": 64 / (statistics.mean(ms) / 1000.0), "pairs": pairs,
                      "kernels_ms": {k: v[0] for k, v in prof.items()}}), flush=True)
    b.close()
    ctx.close()


def precision_report(frames, gpu_res, oq, ot):
    """Per-frame deviation of the GPU pose from the FP64 oracle's (identical
    samples), grouped by noise, camera and geometry."""
    import math

    import numpy as np

    from turboransac_b200 import scenes

    def qang(a, b):
        a = np.asarray(a) / np.linalg.norm(a)
        b = np.asarray(b) / np.linalg.norm(b)
        sgn = 1.0 if float(np.dot(a, b)) >= 0 else -1.0
        return 4.0 * math.asin(min(1.0, float(np.linalg.norm(a - sgn * b)) / 2.0))

    rows = []
    for i, f in enumerate(frames):
        g = gpu_res[i]
        dr = qang(g["q"], oq[i])
        dt = float(np.max(np.abs(np.asarray(g["t"]) - ot[i])))
        ae, te = scenes.pose_error(scenes.quat_to_rotmat(g["q"]), np.asarray(g["t"]), f.R_gt, f.t_gt)
        rows.append((f.sigma, "narrow" if f.K[0] == 2000.0 else "normal", f.degenerate or "generic", dr, dt,
                     ae < 5.0 and te < 5.0))
    def summ(sel):
        if not sel:
            return None
        r = np.array([x[3] for x in sel])
        t = np.array([x[4] for x in sel])
        return {"frames": len(sel), "rot_dev_max_rad": float(r.max()), "rot_dev_p99_rad": float(np.percentile(r, 99)),
                "t_dev_max_m": float(t.max()), "t_dev_p99_m": float(np.percentile(t, 99)),
                "within_1e-6": float(np.mean((r < 1e-6) & (t < 1e-6))),
                "success_5deg_5cm": float(np.mean([x[5] for x in sel]))}
    out = {"all": summ(rows)}
    for s_ in (0.25, 1.0, 3.0):
        out[f"sigma_{s_}"] = summ([x for x in rows if x[0] == s_])
    for c in ("normal", "narrow"):
        out[f"camera_{c}"] = summ([x for x in rows if x[1] == c])
    for d in ("generic", "thin_depth", "plane"):
        out[f"geometry_{d}"] = summ([x for x in rows if x[2] == d])
    return out


def run_case_precision(args):
    """Config 3: FP32/FP64 split against the full-FP64 CPU pipeline on identical samples."""
    from oracle.oracle import Oracle
    from turboransac_b200 import Batch, Context, RansacOptions_cuda, scenes
    n_frames = args.frames
    frames = scenes.precision_frames(n_frames)
    ctx = Context(0, 6 << 30)
    res = []
    t0 = time.perf_counter()
    for i in range(0, n_frames, 1024):
        b = Batch(ctx, frames[i:i + 1024], RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0))
        b.run()
        b.sync()
        res += b.results()
        b.close()
    t_gpu = time.perf_counter() - t0
    t0 = time.perf_counter()
    oq, ot, _ = Oracle().estimate_batch(frames, threads=os.cpu_count() or 1)
    t_cpu = time.perf_counter() - t0
    rep = precision_report(frames, res, oq, ot)
    print(json.dumps({"case": "precision", "frames": n_frames, "gpu_s": t_gpu, "oracle_s": t_cpu,
                      "cores": os.cpu_count(), "report": rep}), flush=True)
    ctx.close()


def main():
    args = parse()
    if args.case == "precision":
        run_case_precision(args)
        return
    if args.case == "plain":
        run_case_plain(args)
        return
    if args.case == "scoring":
        run_case_scoring(args)
        return
    if args.case == "batch64":
        run_case_batch64(args)
        return
    world, rank, local, pg = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        if pg is not None:
            pg.destroy_process_group()
        return

    import numpy as np
    import torch

    from turboransac_b200 import (Batch, BundleOptions_cuda, Camera_cuda, Context, RansacOptions_cuda,
                                  estimate_batch, scenes)
    from turboransac_b200 import build as tbuild
    tbuild.build()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    frames = scenes.batched_frames(args.frames, first=rank * args.frames)
    ro = RansacOptions_cuda(max_iterations=1000, success_prob=0.9999, max_reproj_error=4.0)
    ctx = Context(local, 6 << 30)
    batch = Batch(ctx, frames, ro, hyp_per_thread=args.hr, points_per_iter=128 if args.tensor else 0,
                  chunk_points=8192 if args.tensor else 0)
    # Scoring shape chosen by the autotuner on this batch (before the timed region).
    tuned = None
    if not args.hr and not args.tensor:
        best, tried = batch.autotune(repeats=2)
        default = next(t for t in tried if t["points_per_iter"] == 128 and t["chunk_points"] == 0)
        tuned = {"best": best, "default_ms": default["ms"], "candidates": len(tried)}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    for _ in range(args.warmup):
        batch.run()
        batch.sync()
    res = batch.results()
    steps_per_run = max(r["steps"] for r in res)

    barrier(pg)
    torch.cuda.synchronize()
    dev_ms = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            batch.run()
            batch.sync()
            dev_ms.append(batch.results()[0]["gpu_ms"])
    torch.cuda.synchronize()
    barrier(pg)
    total_ms = max_over_ranks(pg, sum(dev_ms), dev)
    value = world * args.frames * args.steps / (total_ms / 1000.0)
    res = batch.results()
    succ = success(res, frames)
    print(f"[bench] batched: {value:.1f} frames/s, {total_ms / args.steps:.3f} ms/step, success {succ:.4f}",
          file=sys.stderr, flush=True)

    # Per-kernel device time (CUDA events on the launch stream) for the roofline.
    prof, pairs = batch.profile()
    score_ms, score_launches = prof["k_score"]
    achieved = FLOP_PER_PAIR * pairs / (score_ms / 1000.0) / 1e12
    peak_fp32 = fp32_peak_tflops(ctx)
    nominal = 148 * 256 * 1965e6 / 1e12
    # The scoring kernel that ran: the FP32 pass or the tensor-core shape.
    tensor = args.tensor or bool(tuned and tuned["best"]["points_per_iter"] == 128)
    kernel = "k_score_tc" if tensor else "k_score"
    traffic, traffic_source, pipes = stored_traffic(kernel, frames)

    # e2e: public call, host buffers in, results out, every step. Inputs in
    # page-locked host memory (as a data loader would hand them over); the
    # same call on ordinary (pageable) numpy arrays is reported beside it.
    import dataclasses

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = a
        return t

    pin_keep = []
    pframes = []
    for f in frames:
        tu, tx = pinned(f.uv), pinned(f.xyz)
        pin_keep += [tu, tx]
        pframes.append(dataclasses.replace(f, uv=tu.numpy(), xyz=tx.numpy()))

    def time_e2e(fr):
        ts = []
        for i in range(1 + max(1, args.steps // 2)):
            t0 = time.perf_counter()
            estimate_batch(ctx, fr, ro, as_array=True)
            dt = time.perf_counter() - t0
            if i:
                ts.append(dt)
        return world * args.frames * len(ts) / max_over_ranks(pg, sum(ts), dev)

    def time_e2e_submitted(fr):
        # The same public call in its submitted form, two batches in flight:
        # step i submits its batch, then collects step i - 1's (every step's
        # copies in and results out inside the timed region).
        from turboransac_b200 import estimate_batch_submit
        w0, w1 = estimate_batch_submit(ctx, fr, ro), estimate_batch_submit(ctx, fr, ro)  # untimed warm-up of
        w0.collect(as_array=True)                                                        # both buffer sets
        w1.collect(as_array=True)
        k = max(2, args.steps)
        t0 = time.perf_counter()
        prev = estimate_batch_submit(ctx, fr, ro)
        for _ in range(k - 1):
            cur = estimate_batch_submit(ctx, fr, ro)
            prev.collect(as_array=True)
            prev = cur
        prev.collect(as_array=True)
        dt = time.perf_counter() - t0
        return world * args.frames * k / max_over_ranks(pg, dt, dev)

    e2e_sync_fps = time_e2e(pframes)
    e2e_pageable_sync_fps = time_e2e(frames)
    e2e_fps = time_e2e_submitted(pframes)
    e2e_pageable_fps = time_e2e_submitted(frames)
    del pframes, pin_keep
    h2d = sum(40 * f.n for f in frames)
    d2h = args.frames * 264

    # Device-resident correspondences (e.g. a GPU matcher's output): the public
    # device call per step, results to the host.
    from turboransac_b200 import DeviceFrame, estimate_batch_device
    dframes = [DeviceFrame(f, device=dev) for f in frames]
    torch.cuda.synchronize()
    dev_t = []
    for i in range(1 + max(1, args.steps // 2)):
        t0 = time.perf_counter()
        estimate_batch_device(ctx, dframes, ro, as_array=True)
        dt = time.perf_counter() - t0
        if i:
            dev_t.append(dt)
    e2e_device_sync_fps = world * args.frames * len(dev_t) / max_over_ranks(pg, sum(dev_t), dev)
    # ... and in its submitted form, two batches in flight, as the host leg.
    from turboransac_b200 import estimate_batch_device_submit
    w0, w1 = estimate_batch_device_submit(ctx, dframes, ro), estimate_batch_device_submit(ctx, dframes, ro)
    w0.collect(as_array=True)
    w1.collect(as_array=True)
    k = max(2, args.steps)
    t0 = time.perf_counter()
    prev = estimate_batch_device_submit(ctx, dframes, ro)
    for _ in range(k - 1):
        cur = estimate_batch_device_submit(ctx, dframes, ro)
        prev.collect(as_array=True)
        prev = cur
    prev.collect(as_array=True)
    e2e_device_fps = world * args.frames * k / max_over_ranks(pg, time.perf_counter() - t0, dev)
    del dframes, w0, w1, prev, cur

    # Plain per-frame calls (the reference's calling pattern) on the same frames.
    plain = None
    if not args.no_plain:
        lat = []
        for f in frames:
            cam = Camera_cuda(1, 640, 480, list(f.K))
            t0 = time.perf_counter()
            ctx.estimate_absolute_pose(f.uv, f.xyz, cam, ro, BundleOptions_cuda(), seed=f.seed)
            lat.append(1000.0 * (time.perf_counter() - t0))
        plain = {"frames_per_s": len(lat) / (sum(lat) / 1000.0), "p50_ms": float(np.percentile(lat, 50)),
                 "p99_ms": float(np.percentile(lat, 99)), "frames": len(lat)}

    cpu = precision = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu, oracle_out = cpu_baseline(frames)
        precision = precision_vs_oracle(frames, res, oracle_out)
    c0 = config0_plain(ctx) if not args.no_plain else None
    c1 = config1_scoring(ctx)

    serving = None
    if args.serve_seconds > 0:
        shape = tuned["best"] if tuned else None
        serving, reqs = run_serving(ctx, args.serve_seconds, shape=shape)
        serving["plain_call"] = run_plain_serving(ctx, reqs)
        serving["throughput_vs_plain"] = serving["throughput_fps"] / serving["plain_call"]["frames_per_s"]
        serving["capacity"] = run_serving_capacity(ctx, reqs, shape=shape)
        # Latency under heavier offered loads (2 s each).
        serving["sweep"] = []
        for rate in (4000.0, 8000.0):
            r, _ = run_serving(ctx, 2.0, rate=rate, shape=shape)
            serving["sweep"].append({k: r[k] for k in ("offered_rate_hz", "throughput_fps", "p50_ms", "p99_ms",
                                                       "p999_ms", "success_rate")})
        serving["capacity_vs_plain"] = serving["capacity"]["frames_per_s"] / serving["plain_call"]["frames_per_s"]
        print(f"[bench] serving: {serving['throughput_fps']:.0f} frames/s p50 {serving['p50_ms']:.2f} ms "
              f"p99 {serving['p99_ms']:.2f} ms success {serving['success_rate']:.4f}", file=sys.stderr, flush=True)

    if rank == 0:
        clocks = clk.summary()
        line = {
            "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32 scoring / fp64 P3P, re-rank, LM solve",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "global_batch": world * args.frames,
                       "l2": "flushed before every timed step (256 MiB write)",
                       "engine_steps_per_batch": steps_per_run, "parallelism": f"replicas x{world}",
                       "scoring_shape": tuned if tuned else
                       ({"forced": "tensor-core shape, 8192-point chunks"} if args.tensor else
                        {"forced": f"hyp_per_thread={args.hr}"})},
            "success_rate": succ,
            "pairs_scored_per_batch": pairs,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak_fp32, "unit": "TFLOP/s",
                         "frac": achieved / peak_fp32 if peak_fp32 else None, "traffic": traffic,
                         "traffic_source": traffic_source, "pipes_ncu": pipes,
                         "kernel": kernel, "flop_per_pair": FLOP_PER_PAIR, "pairs_per_s": pairs / (score_ms / 1000.0),
                         "accounting": ("27 FP32-equivalent FLOP per pair: the projection's 18 on the tensor "
                                        "cores (tcgen05 TF32, split operands), the rest on the FP32 pipe")
                                       if tensor else "27 FP32 FLOP per pair on the FP32 pipe",
                         "peak_source": "FP32 FMA peak measured in this run (packed-FMA kernel); "
                                        f"nominal {nominal:.1f} TFLOP/s at 1965 MHz",
                         "launch_ms_avg": score_ms / max(score_launches, 1)},
            "kernels_ms_per_batch": {k: v[0] for k, v in prof.items()},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_fps, "unit": "frames/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "inputs": "page-locked host memory", "pageable_inputs_value": e2e_pageable_fps,
                    "call": "estimate_batch_submit(ctx, frames, ro) each step, then the previous step's "
                            "ticket.collect(as_array=True): two batches in flight, every step's copies in "
                            "and results out inside the timed region",
                    "one_call_at_a_time": {"value": e2e_sync_fps, "pageable_inputs_value": e2e_pageable_sync_fps,
                                           "call": "estimate_batch(ctx, frames, ro, as_array=True)"}},
            "e2e_device_inputs": {"value": e2e_device_fps, "unit": "frames/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": d2h,
                                  "inputs": "correspondences already in device memory (CUDA tensors)",
                                  "call": "estimate_batch_device_submit each step, then the previous step's "
                                          "ticket.collect(as_array=True)",
                                  "one_call_at_a_time": e2e_device_sync_fps},
            "plain_call": plain,
            "config0_plain": c0,
            "config1_scoring": c1,
            "precision": precision,
            "candidate_overflow_frames": int(sum(int(r["candidate_overflow"]) for r in res)),
            "serving": serving,
            "speedup_vs_plain": (value / plain["frames_per_s"]) if plain else None,
            # per graph launch: the reset, per engine step 8 RANSAC kernels + 3
            # refinement kernels + the loop test, and the last step's refinement
            "gpu_launches": args.steps * (1 + 12 * steps_per_run + 3),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    batch.close()
    ctx.close()
    if pg is not None:
        pg.destroy_process_group()


def stored_traffic(kernel: str, frames):
    """DRAM bytes of the scoring kernel's first launch on this workload (every
    frame active), from the ncu capture summarised under profiles/ (ncu does not
    run inside the bench): bytes per staged point of the captured case times
    this workload's staged points. Returns (bytes, a note naming the capture
    and its date, pipe utilisations of that capture) or (None, why, None)."""
    tpath = os.path.join(ROOT, "profiles", "k_score_traffic.json")
    try:
        k = json.load(open(tpath))["kernels"][kernel]
        pts = sum(((f.n + 63) // 64) * 64 for f in frames)
        return int(k["bytes_per_staged_point"] * pts), (
            f"not measured in this run: first engine step's launch (all frames active), ncu "
            f"dram__bytes_read.sum + dram__bytes_write.sum of the 64-frame case captured {k['captured']} "
            f"({k['bytes_per_staged_point']:.1f} B per staged point: each point's 40-byte record and each "
            f"hypothesis read once) x {pts} staged points; {k['summary']}"), k.get("pipes_first_launch")
    except Exception:
        return None, f"no stored ncu capture of {kernel} on this workload", None


def fp32_peak_tflops(ctx) -> float | None:
    import ctypes as C

    from turboransac_b200 import _lib
    L = _lib.lib()
    if not hasattr(L, "tbr_measure_fp32_peak"):
        return None
    L.tbr_measure_fp32_peak.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    v = C.c_double()
    if L.tbr_measure_fp32_peak(ctx.handle, C.byref(v)) != 0:
        return None
    return v.value


if __name__ == "__main__":
    main()
