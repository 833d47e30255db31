#!/usr/bin/env python
"""Benchmark of the multi-bounce trace loop: ray-bounces/s on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): the tetrahedron scene — four unit spheres on a regular
tetrahedron of edge 2.5, 6 x 8 x 8 patches each on 7 x 7 Chebyshev-Lobatto
nodes, coarse grid 17 x 17 — lit by 1,048,576 seeded rays from z = 5 over
[-3,3]^2 in a 10-degree cone about -z, at most 200 bounces, Newton tolerance
1e-12.  One step = one bbrt_trace call over all rays.

value     bounces of all rays / device time of one step of the learned-guess
          FP32/FP64 tracer (network trained on this GPU beforehand on a
          separately seeded ray set; inputs already in HBM; CUDA events on the
          launching stream; L2 flushed before each step outside the timed
          events).  The plain FP64 form (the reference's arithmetic, stage-1
          triangle start) and the split form alone are timed the same way and
          reported under "forms"; "accuracy" compares the learned form with the
          plain one ray by ray.
e2e       the same metric through bbrt_trace with pinned host buffers: the
          host->device copy of the rays and the device->host copy of the
          per-ray results are inside the timed region.
roofline  the dominant kernel (k_advance: BVH traversal and stage 1, the same
          in every form) against the pipe peaks measured in this process.
cpu_baseline  the reference's own OpenMP trace loop (oracle/_ref), or the
          oracle port when the reference was not built, on a bounded sample
          of the same rays on all host cores (rank 0, N = 1 only).

With --impl reference the reference's CPU implementation is timed instead
(rank 0 only; other ranks exit 0), on a bounded slice of the same workload
per step.  Multi-GPU: replicas — every rank traces its own seeded 1M rays
(weak scaling, no collective in the data path); value is the sum of all
ranks' bounces over the maximum rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ray-bounces/sec on 1 B200, learned vs plain Newton guess, at hit err ≤1e-10"
UNIT = "ray-bounces/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tetra_spheres")
    ap.add_argument("--rays", type=int, default=None)
    ap.add_argument("--cull", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=8.0, help="target wall time of the CPU sample")
    ap.add_argument("--train-rays", type=int, default=32 << 20,
                    help="rays of each scene traced to record training samples")
    ap.add_argument("--train-epochs", type=int, default=6)
    ap.add_argument("--guess-min-logit", type=float, default=0.0,
                    help="confidence logit above which Newton starts from the learned guess")
    ap.add_argument("--train-positives", type=int, default=16 << 20, help="converged Newton solves kept for training")
    ap.add_argument("--train-negatives", type=int, default=4 << 20, help="stage-1 misses kept for training")
    ap.add_argument("--accuracy-rays", type=int, default=262144, help="0 skips the accuracy comparison")
    ap.add_argument("--autotune", type=int, default=1, help="pick the launch schedule on the workload first")
    ap.add_argument("--multi-scene", type=int, default=64,
                    help="also time K uneven scenes traced together (bbrt_trace_batch) vs one after another")
    ap.add_argument("--forms", default="plain,split,learned",
                    help="forms to time besides the headline (learned); e.g. 'learned' alone for profiling")
    ap.add_argument("--second", default="ellipsoids",
                    help="second workload whose plain / split / learned forms are reported beside the "
                         "headline ('' skips it)")
    ap.add_argument("--second-rays", type=int, default=None, help="rays of the second workload (default: its own)")
    return ap.parse_args()


# plane height, half extent and cone half-angle of each workload's seeded source
TRAIN_SOURCE = {"tetra_spheres": (5.0, 3.0, 10.0), "ellipsoids": (8.0, 6.0, 20.0)}


def workload_config(name, n_rays, maxb, cn, tol, extra=None):
    desc = {
        "tetra_spheres": "4 unit spheres on a tetrahedron (edge 2.5), 6x8x8 patches each, 7x7 nodes (degree 6), "
                         "coarse 17x17 (16x16x2 triangles); rays from z=5 over [-3,3]^2 in a 10-degree cone about -z",
        "two_spheres": "2 unit spheres at (+-1.5,0,0), 6x4x4 patches each, 5x5 nodes, coarse 9x9; "
                       "128x128 plane grid on z=4 over [-3,3]^2, direction (0.3,0,-1)",
        "ellipsoids": "16 random ellipsoids (semi-axes U[0.2,1.2]) in [-6,6]^3, 6x8x8 patches each, 7x7 nodes, "
                      "coarse 17x17; rays from z=8 over [-6,6]^2 in a 20-degree cone",
    }[name]
    c = {"workload": f"{name}: {desc}", "rays": int(n_rays), "max_bounces": int(maxb), "coarse_n": int(cn),
         "newton_tol": tol, "precision": "fp64 (exact, reference operation order)", "guess": "triangle"}
    if extra:
        c.update(extra)
    return c


class ClockSampler:
    """nvidia-smi sampled every 200 ms in the background during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix="bbrt_clocks_", suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


def _hbm_peak():
    """Measured copy bandwidth of this pool's B200 (MEASURED_PEAKS.json) and
    its source, else the pool's earlier measurement (the fallback)."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


HBM_PEAK_GBS, HBM_PEAK_SOURCE = _hbm_peak()
# BVH node tests in FP32 with an FP64 re-test of the undecided (the library's default; BBRT_NODE_F32=0: FP64)
NODE_F32 = os.environ.get("BBRT_NODE_F32", "1") != "0"
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "k_advance_traffic.json")


def advance_roofline(st, fp64_peak, fp32_peak, l2_peak):
    """Roofline of the dominant kernel, k_advance, from its own counters and its
    own device time (CUDA events around each launch inside the library).

    Work per unit:
      BVH node test, FP32    16 FP32 FLOP (6 differences, 6 products, 4
                             margin adds), 40 B (FP32 box + links); the few
                             it leaves undecided add the FP64 test below
      BVH node test, FP64    12 FP64 FLOP, 64 B (box + links); 48 B (box)
                             as the re-test of an undecided FP32 test
      block / cell box test  18 FP32 FLOP, 24 B
      Moller-Trumbore test   28 FP64 FLOP up to the division-free rejection
                             (51 when it passes), 18 FP64 FLOP of corner
                             offsets, 104 B (three corners + cell normal/sagitta)
    The headline pipe is the one with the largest fraction of its peak."""
    nodes = st["node_tests"] - st["tail_node_tests"]
    boxes = st["cell_tests"] - st["tail_cell_tests"]
    mts = st["tri_tests"] - st["tail_tri_tests"]
    retest = st.get("node_tests_fp64", 0)   # whole step (the tail's few included)
    secs = st["advance_ms"] / 1e3
    if secs <= 0:
        return None
    if NODE_F32:
        f64, f32, nbytes = 12 * retest, 16 * nodes, 40 * nodes + 48 * retest
    else:
        f64, f32, nbytes = 12 * nodes, 0, 64 * nodes
    pipes = {
        "fp64": ((f64 + (28 + 18) * mts) / secs / 1e12, fp64_peak, "TFLOP/s"),
        "fp32": ((f32 + 18 * boxes) / secs / 1e12, fp32_peak, "TFLOP/s"),
        "l2": ((nbytes + 24 * boxes + 104 * mts) / secs / 1e9, l2_peak, "GB/s"),
        "hbm": ((nbytes + 24 * boxes + 104 * mts) / secs / 1e9, HBM_PEAK_GBS, "GB/s"),
    }
    best = max(pipes, key=lambda k: pipes[k][0] / pipes[k][1])
    a, p, u = pipes[best]
    traffic = None
    if os.path.exists(PROFILE_TRAFFIC):
        prof = json.load(open(PROFILE_TRAFFIC))
        # scale the captured launch's DRAM bytes to a whole step of k_advance launches by the work done
        if prof.get("node_tests"):
            traffic = prof["dram_bytes"] * nodes / prof["node_tests"] / max(1, st["rounds"])
    return {"bound": best, "achieved": a, "peak": p, "unit": u, "frac": a / p, "traffic": traffic,
            "kernel": "k_advance", "launches_per_step": int(st["rounds"]),
            "pipes": {k: {"achieved": v[0], "peak": v[1], "unit": v[2], "frac": v[0] / v[1]} for k, v in pipes.items()},
            "note": "algorithmic work of the k_advance launches of one step (device counters) over their summed "
                    "CUDA-event time; peaks: FP64/FP32 FMA and L2-resident reads measured in this process "
                    f"(bbrt_measure_pipe_peak), of measured; HBM {HBM_PEAK_GBS:.0f} GB/s, of {HBM_PEAK_SOURCE} "
                    f"({'MEASURED_PEAKS.json' if HBM_PEAK_SOURCE == 'measured' else 'no MEASURED_PEAKS.json: the pool fallback'}); the exact FP64 "
                    "path runs unfused mul/add (half the FMA peak at most); traffic per launch from the ncu "
                    "capture in profiles/, scaled by node tests"}


def cpu_baseline(patches, o, d, maxb, cn, tol, target_s):
    """The reference's trace loop (or the oracle port) on a bounded sample."""
    import oracle
    threads = os.cpu_count() or 1
    if oracle.reference_available():
        tmp = tempfile.mkdtemp(prefix="bbrt_bench_ref_")
        runner = oracle.Reference.from_patches(patches, tmpdir=tmp, coarse_n=cn, newton_tol=tol)
        kind = "reference"
    else:
        from billardballraytracing3d_b200 import _capi as C
        runner = oracle.Oracle(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol))
        kind = "port"
    probe = min(8192, o.shape[0])
    r = runner.trace(o[:probe], d[:probe], maxb, K=0, nthreads=threads)
    rate = probe / max(r["seconds"], 1e-6)
    n = int(min(o.shape[0], max(probe, rate * target_s)))
    r = runner.trace(o[:n], d[:n], maxb, K=0, nthreads=threads)
    bounces = int(r["bounce_count"].sum())
    return {"value": bounces / r["seconds"], "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"first {n} of the workload's rays ({bounces} bounces, {r['seconds']:.2f} s wall, "
                      f"OpenMP schedule(dynamic) over trace_ray)"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    from billardballraytracing3d_b200 import scenes
    import oracle
    patches, o, d, maxb, cn, tol = scenes.workload(args.workload, args.rays)
    threads = os.cpu_count() or 1
    if oracle.reference_available():
        runner = oracle.Reference.from_patches(patches, tmpdir=tempfile.mkdtemp(prefix="bbrt_ref_"),
                                               coarse_n=cn, newton_tol=tol)
        kind = "reference"
    else:
        from billardballraytracing3d_b200 import _capi as C
        runner = oracle.Oracle(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol))
        kind = "port"
    # size one step's slice for ~1.5 s of wall time on this host
    probe = min(8192, o.shape[0])
    pr = runner.trace(o[:probe], d[:probe], maxb, K=0, nthreads=threads)
    per = int(min(o.shape[0], max(1024, probe / max(pr["seconds"], 1e-6) * 1.5)))
    slices = [(k * per) % max(1, o.shape[0] - per + 1) for k in range(args.warmup + args.steps)]
    for k in range(args.warmup):
        s = slices[k]
        runner.trace(o[s:s + per], d[s:s + per], maxb, K=0, nthreads=threads)
    tot_s, tot_b = 0.0, 0
    for k in range(args.warmup, args.warmup + args.steps):
        s = slices[k]
        r = runner.trace(o[s:s + per], d[s:s + per], maxb, K=0, nthreads=threads)
        tot_s += r["seconds"]
        tot_b += int(r["bounce_count"].sum())
    value = tot_b / tot_s
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_s / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args.workload, o.shape[0], maxb, cn, tol,
                                      {"parallelism": f"OpenMP x{threads} host threads",
                                       "step": f"{per} rays per step (bounded slice of the workload)"}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"{args.steps} slices of {per} rays of the workload"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _trace_form(scene, to, td, n, maxb, outs, stream, flush, steps, warmup, dev, world, clocks=None):
    """Times `steps` device traces of the scene's current mode (after `warmup`
    untimed ones); returns (kernel seconds, wall seconds, last stats).

    The warm-up calls both forms of the call (without statistics, as timed,
    and with them), so that a graph-launched trace has captured both graphs
    before timing.  Graph-launched rounds carry no per-kernel events, so the
    per-kernel times of the returned statistics come from one extra
    host-driven step after the timed region (same kernels, same work)."""
    import torch
    stats = None
    for k in range(warmup):
        want = k == warmup - 1
        r = scene.trace_device(to.data_ptr(), td.data_ptr(), n, maxb, outs, stream=stream.cuda_stream,
                               want_stats=want)
        if want:
            stats = r
    torch.cuda.synchronize(dev)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    if clocks:
        clocks.start()
    torch.cuda.synchronize(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    wall0 = time.perf_counter()
    for k in range(steps):
        flush.zero_()
        evs[k][0].record(stream)
        scene.trace_device(to.data_ptr(), td.data_ptr(), n, maxb, outs, stream=stream.cuda_stream)
        evs[k][1].record(stream)
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - wall0
    if world > 1:
        dist.barrier()
    if stats is not None:
        # per-kernel device times of the timed kernels (the instances that
        # keep no counters): one host-driven-rounds step with kernel events only
        graph = scene.tuning()["graph_rounds"]
        if graph:
            scene.tuning(graph_rounds=0)
        host = scene.trace_device(to.data_ptr(), td.data_ptr(), n, maxb, outs, stream=stream.cuda_stream,
                                  want_stats=True, times_only=True)
        if graph:
            scene.tuning(graph_rounds=1)
        torch.cuda.synchronize(dev)
        stats = dict(stats, **{k: host[k] for k in ("order_ms", "advance_ms", "guess_ms", "newton_ms", "tail_ms")},
                     kernel_ms_from="one host-driven-rounds step after the timed region, kernel events only (the "
                                    "counters above come from a statistics step, whose kernels also count)")
    return sum(a.elapsed_time(b) for a, b in evs) / 1e3, wall, stats


def replica_rays(workload, o, d, rank):
    """Replicas (weak scaling): rank 0 traces the workload's own rays, every
    other rank as many rays of the same source with its own seed (the
    plane-grid workload has no seed: every rank traces the same grid)."""
    if rank == 0 or workload not in TRAIN_SOURCE:
        return o, d
    from billardballraytracing3d_b200 import scenes
    return scenes.cone_rays(o.shape[0], 1234 + rank, *TRAIN_SOURCE[workload])


def _max_over_ranks(kern_s, total_b, dev, world):
    """The job's time (max over ranks) and work (sum over ranks)."""
    if world == 1:
        return kern_s, total_b
    import torch
    import torch.distributed as dist
    t = torch.tensor([kern_s], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    b = torch.tensor([total_b], dtype=torch.int64, device=dev)
    dist.all_reduce(b, op=dist.ReduceOp.SUM)
    return float(t.item()), int(b.item())


def _newton_failures(status, C):
    return int(np.isin(status, [C.RAY_NEWTON_SINGULAR, C.RAY_NEWTON_NOCONV, C.RAY_NEWTON_DOMAIN]).sum())


def _accuracy(scene, o, d, maxb, C):
    """The learned FP32/FP64 form against the plain FP64 form (bit-identical to
    the reference) on the same rays, every bounce of every ray recorded: share
    of rays with the same status and hit-object sequence (also over the rays
    whose incidence cosine exceeds 1e-3 at every bounce), the largest
    difference of any hit point, end point and exit direction over those rays,
    and Newton failures of each form."""
    from billardballraytracing3d_b200 import api
    scene.set_modes(C.PREC_FP64, C.GUESS_TRIANGLE)
    a = api.trace_recording_all(scene, o, d, maxb)
    scene.set_modes(C.PREC_SPLIT, C.GUESS_LEARNED)
    b = api.trace_recording_all(scene, o, d, maxb)
    K = max(a["hit_object"].shape[1], b["hit_object"].shape[1])
    if a["hit_object"].shape[1] != K:
        scene.set_modes(C.PREC_FP64, C.GUESS_TRIANGLE)
        a = scene.trace(o, d, maxb, record=K)
    if b["hit_object"].shape[1] != K:
        scene.set_modes(C.PREC_SPLIT, C.GUESS_LEARNED)
        b = scene.trace(o, d, maxb, record=K)
    r = api.compare_traces(a, b, o)
    r.update({"newton_failures_plain": _newton_failures(a["status"], C),
              "newton_failures_learned": _newton_failures(b["status"], C),
              "off_patch_misses_learned": int(b["stats"]["off_patch"]),
              "went_inside_plain": int((a["status"] == C.RAY_WENT_INSIDE).sum()),
              "went_inside_learned": int((b["status"] == C.RAY_WENT_INSIDE).sum()),
              "recorded_bounces": int(K),
              "compared": "status and hit-object sequence; every recorded hit point, its (u, v) and the exit "
                          "direction held to 1e-10 vs the plain FP64 form; the end point (escaped rays: last hit + "
                          "scene diagonal x exit direction) reported beside them"})
    return r


def _form_report(secs, b, st, steps):
    """One timed form: rate, step time, Newton work per hit and kernel split."""
    bounces = max(1, st["bounces"])
    fails = sum(st["status_hist"][k] for k in (2, 3, 4))
    return {"value": b / secs, "unit": UNIT, "ms_per_step": 1e3 * secs / steps,
            "newton_iters_fp64": st["newton_iters"], "newton_iters_fp32": st["newton_iters_fp32"],
            "newton_iters_per_hit": (st["newton_iters"] + st["newton_iters_fp32"]) / bounces,
            "newton_iters_fp64_per_hit": st["newton_iters"] / bounces,
            "newton_failed_rays": int(fails), "newton_failure_rate": fails / max(1, st["rays"]),
            "off_patch_misses": st.get("off_patch", 0),
            "newton_ms": st["newton_ms"], "guess_ms": st["guess_ms"],
            "advance_ms": st["advance_ms"], "tail_ms": st["tail_ms"]}


def run_ours(args, rank, world, local_rank):
    import torch
    from billardballraytracing3d_b200 import _capi as C
    from billardballraytracing3d_b200 import api, scenes

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    patches, o, d, maxb, cn, tol = scenes.workload(args.workload, args.rays)
    o, d = replica_rays(args.workload, o, d, rank)
    n = o.shape[0]
    cfg = C.default_config(coarse_grid_n=cn, newton_tol=tol, cull=args.cull)
    scene = api.Scene(patches, config=cfg)
    scene.upload()
    lib = C.load_library()
    import ctypes
    peak = ctypes.c_double()
    C.check(lib, lib.bbrt_measure_pipe_peak(C.PIPE_FP64, ctypes.byref(peak)), "bbrt_measure_pipe_peak")
    fp64_peak = peak.value
    C.check(lib, lib.bbrt_measure_pipe_peak(C.PIPE_FP32, ctypes.byref(peak)), "bbrt_measure_pipe_peak")
    fp32_peak = peak.value
    C.check(lib, lib.bbrt_measure_pipe_peak(C.PIPE_L2, ctypes.byref(peak)), "bbrt_measure_pipe_peak")
    l2_peak = peak.value

    # launch schedule picked on the workload itself (plain form; results do not depend on it)
    tuned = scene.autotune(o, d, maxb, trials=2) if args.autotune else scene.tuning()
    # the learned guess: trained on this GPU by the project's own kernels on
    # samples that a plain trace of separately seeded rays records; with a
    # second workload, one network for both scenes (a scene set of the two),
    # each scene then given its share
    second = None
    train_src = TRAIN_SOURCE.get(args.workload, (5.0, 3.0, 10.0))
    train_o, train_d = scenes.cone_rays(args.train_rays, 99 + rank, *train_src)
    tcfg = dict(epochs=args.train_epochs, max_positive=args.train_positives, max_negative=args.train_negatives,
                min_logit=args.guess_min_logit)
    if args.second:
        s_patches, s_o, s_d, s_maxb, s_cn, s_tol = scenes.workload(args.second, args.second_rays)
        s_scene = api.Scene(s_patches, config=C.default_config(coarse_grid_n=s_cn, newton_tol=s_tol, cull=args.cull))
        s_scene.upload()
        s_to, s_td = scenes.cone_rays(args.train_rays, 199 + rank, *TRAIN_SOURCE.get(args.second, (5.0, 3.0, 10.0)))
        pair = api.SceneSet([scene, s_scene])
        training = pair.guess_train([train_o, s_to], [train_d, s_td], max(maxb, s_maxb), **tcfg)
        training["scenes"] = [args.workload, args.second]
        training["rays_per_scene"] = int(args.train_rays)
        pair.guess_export(0, scene)
        pair.guess_export(1, s_scene)
        pair.close()
        del s_to, s_td
        second = (s_scene, s_o, s_d, s_maxb, s_cn, s_tol, training)
    else:
        training = scene.guess_train(train_o, train_d, maxb, **tcfg)
    del train_o, train_d

    to = torch.from_numpy(np.ascontiguousarray(o)).to(dev)
    td = torch.from_numpy(np.ascontiguousarray(d)).to(dev)
    st_ = torch.empty(n, dtype=torch.int32, device=dev)
    bc = torch.empty(n, dtype=torch.int32, device=dev)
    ed = torch.empty((n, 3), dtype=torch.float64, device=dev)
    outs = dict(status=st_.data_ptr(), bounce_count=bc.data_ptr(), exit_dir=ed.data_ptr())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)   # > 126 MB L2
    # a real stream handle: torch's legacy default stream is handle 0, which the
    # C ABI reads as "the scene's own stream"
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    forms = set(args.forms.split(","))
    timed_forms = {}
    # the plain form (FP64, stage-1 triangle start: the reference's arithmetic)
    if "plain" in forms:
        scene.set_modes(C.PREC_FP64, C.GUESS_TRIANGLE)
        p_s, _, p_stats = _trace_form(scene, to, td, n, maxb, outs, stream, flush, args.steps, args.warmup, dev, world)
        p_s, p_b = _max_over_ranks(p_s, int(bc.sum().item()) * args.steps, dev, world)
        timed_forms["plain_fp64_triangle"] = (p_s, p_b, p_stats)
    # the split form alone (FP32 Newton phase, triangle start)
    if "split" in forms:
        scene.set_modes(C.PREC_SPLIT, C.GUESS_TRIANGLE)
        s_s, _, s_stats = _trace_form(scene, to, td, n, maxb, outs, stream, flush, args.steps, args.warmup, dev, world)
        s_s, s_b = _max_over_ranks(s_s, int(bc.sum().item()) * args.steps, dev, world)
        timed_forms["split_triangle"] = (s_s, s_b, s_stats)
    # the headline: the learned-guess FP32/FP64 tracer
    scene.set_modes(C.PREC_SPLIT, C.GUESS_LEARNED)
    clocks = ClockSampler(local_rank)
    kern_s, wall, stats = _trace_form(scene, to, td, n, maxb, outs, stream, flush, args.steps, args.warmup, dev,
                                      world, clocks)
    clk = clocks.stop()
    bounces_per_step = int(bc.sum().item())
    assert stats is None or stats["bounces"] == bounces_per_step
    kern_s, total_b = _max_over_ranks(kern_s, bounces_per_step * args.steps, dev, world)
    value = total_b / kern_s

    # e2e: host (pinned) buffers through the same C ABI call, copies inside the timed region
    ho = torch.from_numpy(np.ascontiguousarray(o)).pin_memory()
    hd = torch.from_numpy(np.ascontiguousarray(d)).pin_memory()
    hs = torch.empty(n, dtype=torch.int32).pin_memory()
    hb = torch.empty(n, dtype=torch.int32).pin_memory()
    he = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    out = C.TraceOut()
    out.status = ctypes.cast(ctypes.c_void_p(hs.data_ptr()), C.c_int_p)
    out.bounce_count = ctypes.cast(ctypes.c_void_p(hb.data_ptr()), C.c_int_p)
    out.exit_dir = ctypes.cast(ctypes.c_void_p(he.data_ptr()), C.c_double_p)
    e2e_steps = max(1, min(args.steps, 5))
    e2e_s = 0.0
    for k in range(e2e_steps + 1):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        C.check(lib, lib.bbrt_trace(scene.h, ctypes.c_void_p(ho.data_ptr()), ctypes.c_void_p(hd.data_ptr()), n, maxb,
                                    0, ctypes.byref(out), None, ctypes.c_void_p(stream.cuda_stream)), "bbrt_trace")
        if k > 0:
            e2e_s += time.perf_counter() - t0
    e2e_s, e2e_b = _max_over_ranks(e2e_s, int(hb.numpy().sum()) * e2e_steps, dev, world)
    e2e = {"value": e2e_b / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(ho.numel() * 8 + hd.numel() * 8),
           "d2h_bytes_per_step": int(hs.numel() * 4 + hb.numel() * 4 + he.numel() * 8),
           "note": "host wall clock around bbrt_trace (learned FP32/FP64 form) with pinned host arrays "
                   "(copies + kernels + sync)"}

    if rank != 0:
        return
    accuracy = _accuracy(scene, o[:args.accuracy_rays], d[:args.accuracy_rays], maxb, C) if args.accuracy_rays > 0 \
        else None
    per_launch_s = kern_s / args.steps
    roofline = advance_roofline(stats, fp64_peak, fp32_peak, l2_peak) if stats else None
    form = lambda secs, b, st: _form_report(secs, b, st, args.steps)  # noqa: E731
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * per_launch_s, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32 (BF16 MLP guess)", "data": "synthetic",
            "config": workload_config(args.workload, n, maxb, cn, tol,
                                      {"parallelism": "replicas" if world > 1 else "single GPU",
                                       "cull": args.cull,
                                       "precision": "split: FP32 Newton phase to |F|<1e-5, FP64 finish",
                                       "guess": "learned (BF16 MLP on tcgen05), triangle fallback",
                                       "schedule": tuned,
                                       "l2": "flushed before each step (256 MiB write), flush outside the timed events",
                                       "bounces_per_step": bounces_per_step}),
            "forms": dict({k: form(*v) for k, v in timed_forms.items()}, learned_split=form(kern_s, total_b, stats),
                          learned_over_plain=(value / (timed_forms["plain_fp64_triangle"][1] /
                                                       timed_forms["plain_fp64_triangle"][0])
                                              if "plain_fp64_triangle" in timed_forms else None)),
            "accuracy": accuracy,
            "guess_training": training,
            "e2e": e2e, "gpu_launches": int(stats["launches"]) * args.steps if stats else None,
            "roofline": roofline, "clocks": clk,
            "kernel_ms_per_step": {k: stats[k] for k in ("order_ms", "advance_ms", "guess_ms", "newton_ms", "tail_ms")}
            if stats else None,
            "wall_s_timed_region": wall,
            "counters_per_step": {k: v for k, v in (stats or {}).items() if k not in ("kernel_ms", "total_ms")}}
    if args.second:
        line["second_workload"] = second_workload(args, second, dev, stream, flush)
    if args.multi_scene > 0 and world == 1:
        line["multi_scene"] = multi_scene(args.multi_scene, args.steps, dev)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(patches, o, d, maxb, cn, tol, args.cpu_seconds)
    print(json.dumps(line), flush=True)


def second_workload(args, second, dev, stream, flush):
    """The second workload (default: the random-ellipsoid scene, 16 ellipsoids
    x 384 patches, 4,194,304 rays in a 20-degree cone, <= 100 bounces) traced
    in the plain FP64 form, the split form and the learned-guess form (the
    network trained for both scenes together), each timed like the headline;
    with Newton failure rates, Newton iterations per hit, and the learned
    form's accuracy against the plain one."""
    import torch
    from billardballraytracing3d_b200 import _capi as C
    sc, o, d, maxb, cn, tol, training = second
    n = o.shape[0]
    to = torch.from_numpy(np.ascontiguousarray(o)).to(dev)
    td = torch.from_numpy(np.ascontiguousarray(d)).to(dev)
    st_ = torch.empty(n, dtype=torch.int32, device=dev)
    bc = torch.empty(n, dtype=torch.int32, device=dev)
    ed = torch.empty((n, 3), dtype=torch.float64, device=dev)
    outs = dict(status=st_.data_ptr(), bounce_count=bc.data_ptr(), exit_dir=ed.data_ptr())
    steps, warmup = max(1, min(args.steps, 5)), 3
    forms = {}
    for name, prec, guess in (("plain_fp64_triangle", C.PREC_FP64, C.GUESS_TRIANGLE),
                              ("split_triangle", C.PREC_SPLIT, C.GUESS_TRIANGLE),
                              ("learned_split", C.PREC_SPLIT, C.GUESS_LEARNED)):
        sc.set_modes(prec, guess)
        secs, _, st = _trace_form(sc, to, td, n, maxb, outs, stream, flush, steps, warmup, dev, 1)
        forms[name] = _form_report(secs, int(bc.sum().item()) * steps, st, steps)
    forms["learned_over_plain"] = forms["learned_split"]["value"] / forms["plain_fp64_triangle"]["value"]
    acc = None
    if args.accuracy_rays > 0:
        m = min(n, args.accuracy_rays)
        acc = _accuracy(sc, o[:m], d[:m], maxb, C)
    sc.set_modes(C.PREC_FP64, C.GUESS_TRIANGLE)
    return {"config": workload_config(args.second, n, maxb, cn, tol), "steps": steps, "warmup": warmup,
            "forms": forms, "accuracy": acc, "guess_training": "the headline's (one network for both scenes)",
            "note": "device time per step (CUDA events, L2 flushed before each step), default launch schedule; "
                    "newton_failure_rate = rays failed by Newton / rays; newton_iters_per_hit = FP32 + FP64 "
                    "Newton iterations / ray-bounces"}


def multi_scene(k, steps, dev):
    """k independent scenes of uneven size (scenes.multi_scene_workload:
    1-32 obstacles of 96 or 384 patches at degree 4 or 6, 16k-1M rays each,
    <= 100 bounces, plain FP64): device time of tracing them as one scene set
    (bbrt_trace_set: one wavefront for all), together on their own streams
    (bbrt_trace_batch), and one after another; best of `steps` after a warm-up
    each; and the set's learned form (one network for all scenes, trained on
    this GPU) against its plain one.  Also the wall time of building the scenes (per-patch set-up on the
    GPU) and of building the set."""
    import torch
    from billardballraytracing3d_b200 import _capi as C
    from billardballraytracing3d_b200 import api, scenes
    work = scenes.multi_scene_workload(k)
    t0 = time.perf_counter()
    scs = [api.Scene(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol))
           for patches, o, d, maxb, cn, tol in work]
    for sc in scs:
        sc.upload()
    torch.cuda.synchronize(dev)
    create_s = time.perf_counter() - t0
    # the C ABI's scene creation alone (descriptors already built): the
    # per-patch set-up on the GPU vs on the host, every scene created,
    # uploaded and released in turn
    setup_cmp = {"scenes": k, "patches": int(sum(len(w[0]) for w in work)), "host_threads": os.cpu_count()}
    for where in (1, 0):
        t0 = time.perf_counter()
        for sc0, (patches, o, d, maxb, cn, tol) in zip(scs, work):
            sc = api.Scene(table=sc0.table, config=C.default_config(coarse_grid_n=cn, newton_tol=tol,
                                                                    setup_on_device=where))
            sc.upload()
            sc.close()
        torch.cuda.synchronize(dev)
        setup_cmp["gpu_s" if where else "host_s"] = time.perf_counter() - t0
    tens = []
    for patches, o, d, maxb, cn, tol in work:
        n = o.shape[0]
        tens.append(dict(o=torch.from_numpy(o).to(dev), d=torch.from_numpy(d).to(dev),
                         status=torch.zeros(n, dtype=torch.int32, device=dev),
                         bounce_count=torch.zeros(n, dtype=torch.int32, device=dev)))
    ns = [w[1].shape[0] for w in work]
    optr = [t["o"].data_ptr() for t in tens]
    dptr = [t["d"].data_ptr() for t in tens]
    outs = [dict(status=t["status"].data_ptr(), bounce_count=t["bounce_count"].data_ptr()) for t in tens]
    t0 = time.perf_counter()
    ss = api.SceneSet(scs)
    set_create_s = time.perf_counter() - t0
    st, _ = ss.trace_device(optr, dptr, ns, 100, outs)   # warm-up (graph capture)
    ss.trace_device(optr, dptr, ns, 100, outs, want_stats=False)
    bounces = st["bounces"]
    set_ms = min(ss.trace_device(optr, dptr, ns, 100, outs, want_stats=False)[1] for _ in range(steps))
    set_bc = [t["bounce_count"].clone() for t in tens]
    # the learned form of the set: one network for all 64 scenes, trained on
    # separately seeded rays of every scene's source
    train = [scenes.cone_rays(min(n, 1 << 17), 7000 + j, 8.0, 6.0, 20.0) for j, n in enumerate(ns)]
    set_training = ss.guess_train([t[0] for t in train], [t[1] for t in train], 100, epochs=4)
    del train
    ss.configure(C.PREC_SPLIT, C.GUESS_LEARNED)
    lst, _ = ss.trace_device(optr, dptr, ns, 100, outs)   # warm-up (graph capture)
    ss.trace_device(optr, dptr, ns, 100, outs, want_stats=False)
    learned_ms = min(ss.trace_device(optr, dptr, ns, 100, outs, want_stats=False)[1] for _ in range(steps))
    agree = float(sum(int((a == t["bounce_count"]).sum().item()) for a, t in zip(set_bc, tens)) / sum(ns))
    ss.configure(C.PREC_FP64, C.GUESS_TRIANGLE)
    api.trace_batch_device(scs, optr, dptr, ns, 100, outs)   # warm-up
    batch = min(api.trace_batch_device(scs, optr, dptr, ns, 100, outs, want_stats=False)[1] for _ in range(steps))
    same = all(torch.equal(a, t["bounce_count"]) for a, t in zip(set_bc, tens))
    for j in range(k):   # warm-up one at a time
        api.trace_batch_device([scs[j]], [optr[j]], [dptr[j]], [ns[j]], 100, [outs[j]], want_stats=False)
    seq = min(sum(api.trace_batch_device([scs[j]], [optr[j]], [dptr[j]], [ns[j]], 100, [outs[j]],
                                         want_stats=False)[1] for j in range(k)) for _ in range(steps))
    return {"scenes": k, "rays": int(sum(ns)), "patches": int(sum(len(w[0]) for w in work)),
            "bounces": int(bounces), "set_ms": set_ms, "batched_ms": batch, "sequential_ms": seq,
            "set_value": bounces / (set_ms / 1e3), "batched_value": bounces / (batch / 1e3),
            "sequential_value": bounces / (seq / 1e3), "unit": UNIT,
            "set_over_sequential": seq / set_ms, "set_over_batched": batch / set_ms,
            "set_results_equal_batched": bool(same),
            "learned_set_ms": learned_ms, "learned_set_value": lst["bounces"] / (learned_ms / 1e3),
            "learned_over_plain": (lst["bounces"] / learned_ms) / (bounces / set_ms),
            "learned_bounce_count_agreement": agree, "learned_newton_failed_rays": int(sum(lst["status_hist"][2:5])),
            "plain_newton_failed_rays": int(sum(st["status_hist"][2:5])), "learned_training": set_training,
            "scene_build_s": create_s, "set_build_s": set_create_s, "setup_compare": setup_cmp, "set_rounds": st["rounds"],
            "set_launches": st["launches"],
            "note": "device time of one bbrt_trace_set call (the set: one wavefront over all scenes, rays in and "
                    "results out included) vs one bbrt_trace_batch call (a wavefront per scene, scenes on their "
                    "own streams) vs the sum of one-scene calls; plain FP64 form, default schedule; scene_build_s: "
                    "wall time of creating and uploading the scenes (per-patch set-up on the GPU, BVH on the host)"}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
