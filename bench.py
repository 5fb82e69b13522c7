"""Benchmark of the uniform-grid hot path (voxel centroid downsample + radius
normals) on B200.

Workload (one step): the 2,000,000-point georeferenced scan-like point_xyzi
cloud (60% ground, 30% box faces, 10% clutter; offset (450000, 3900000, 50) m,
fed as f32(world - origin)), voxel-downsampled at leaf 0.1 m and at leaf 0.5 m,
each followed by radius normals (r = 0.5 m, viewpoint origin + (0, 0, 100)) on
the centroids -- the MvpPipeline chain.  The two leaf chains are independent and
run on two streams, one context each (--serial-leaves: one stream).  value = input points per second
through the whole step (2M points / step time), inputs resident in HBM, L2
flushed (256 MB write) between timed steps.  e2e = the same through the C ABI
with pinned host buffers (H2D of the inputs and D2H of all results inside the
timed region).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU (torchrun, one process per GPU): replicas -- every rank runs the
full workload on its own GPU (weak scaling); the step time is the max over
ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_POINTS = 2_000_000
LEAVES = (0.1, 0.5)
RADIUS = 0.5
VIEWPOINT = (0.0, 0.0, 100.0)  # origin + (0, 0, 100) in the cloud's local frame
WORKLOAD = "georef_scan_2M_xyzi: voxel leaf 0.1 + leaf 0.5, each -> radius normals r 0.5 on centroids"
METRIC = "M points/s voxel+normals (2M georeferenced point_xyzi, leaf 0.1 & 0.5, r 0.5)"
UNIT = "Mpoints/s"
L2_FLUSH_BYTES = 256 << 20
PROFILE_PASSES = 5  # untimed per-group profile passes (median)
# DRAM bytes (read + write) per launch of the dominant kernel group on this
# workload, mean over the leaf-0.1 and leaf-0.5 chains, from one ncu capture
# (profiles/k_normals_georef2M_leaf0.1.md); ncu cannot run inside the bench.
# ncu dram__bytes_read.sum + dram__bytes_write.sum of the normals launches of one step
# (leaf 0.1, leaf 0.5), profiles/dram_per_kernel_georef2M.md
MEASURED_TRAFFIC = {"normals": (88.3e6 + 41.3e6) / 2}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serial-leaves", action="store_true",
                    help="run the two leaf chains of a step on one stream, one after the other")
    ap.add_argument("--profile-all", action="store_true",
                    help="print the per-kernel-group timing table to stderr")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the many-clouds (batched vs per-cloud loop) measurement")
    ap.add_argument("--batched-clouds", type=int, default=256)
    ap.add_argument("--batched-scale", type=float, default=1.0,
                    help="scale of every cloud of the many-clouds measurement (profiling runs)")
    ap.add_argument("--only-batched", action="store_true",
                    help="run the many-clouds measurement alone and print its JSON (profiling runs)")
    ap.add_argument("--only-ransac", action="store_true",
                    help="run the RANSAC plane measurement alone (profiling runs)")
    ap.add_argument("--only-las", action="store_true",
                    help="run the LAS ingest -> streaming voxel measurement alone (profiling runs)")
    ap.add_argument("--no-shapes", action="store_true",
                    help="skip the 5M-point shapes radius-normals measurement")
    ap.add_argument("--no-cluster", action="store_true",
                    help="skip the Euclidean cluster-roots measurement")
    ap.add_argument("--no-plane-cov", action="store_true",
                    help="skip the GICP plane-covariance leg")
    ap.add_argument("--no-ransac", action="store_true",
                    help="skip the RANSAC plane leg")
    ap.add_argument("--no-las-stream", action="store_true",
                    help="skip the LAS ingest -> streaming voxel leg")
    ap.add_argument("--no-serving", action="store_true",
                    help="skip the serving-loop (Poisson arrivals) measurement")
    ap.add_argument("--serving-rates", default="100,500,1000,2000",
                    help="offered request rates (req/s) of the serving measurement")
    ap.add_argument("--serving-seconds", type=float, default=2.0)
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end (host buffers) measurements (profiling runs)")
    ap.add_argument("--e2e-inflight", type=int, default=E2E_INFLIGHT,
                    help="steps in flight in the end-to-end measurement")
    ap.add_argument("--neighbor-walk", type=int, default=-1, choices=[-1, 0, 1, 2],
                    help="the normals kernel's neighbour walk (-1: the built-in choice)")
    return ap.parse_args()


def bench_config(world: int) -> dict:
    """The workload, identical in both arms' lines."""
    return dict(workload=WORKLOAD, points=N_POINTS, leaves=list(LEAVES), radius=RADIUS,
                viewpoint=list(VIEWPOINT), parallelism=f"replicas x{world}")


VOXEL_GROUPS = ("begin", "bounds", "voxel_plan", "voxel_sort", "voxel_segments")


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def workload_cloud():
    from spatialrust_b200 import synthetic
    return synthetic.georef_scan(N_POINTS, seed=1)


# ---- CPU (reference restatement) -------------------------------------------

def cpu_crop(cloud, side=None):
    """The whole cloud (side None) or the x, y < side tile at full density."""
    if side is None:
        return cloud.x, cloud.y, cloud.z, cloud.intensity
    m = (cloud.x < side) & (cloud.y < side)
    return (np.ascontiguousarray(cloud.x[m]), np.ascontiguousarray(cloud.y[m]),
            np.ascontiguousarray(cloud.z[m]), np.ascontiguousarray(cloud.intensity[m]))


def cpu_step(crop, threads=0):
    """One step of the reference CPU path; threads 0 = the reference's own
    worker count for the sample (staging.rs:11-41)."""
    import oracle
    x, y, z, i = crop
    for leaf in LEAVES:
        v = oracle.voxel_centroid(x, y, z, [i], leaf=leaf)
        oracle.radius_normals_ref(v.x, v.y, v.z, RADIUS, 3, VIEWPOINT, threads=threads)


def cpu_threads(n_centroids: int) -> int:
    import oracle
    return oracle.parallel_worker_count(n_centroids, os.cpu_count() or 1)


CROP_SIDE = None  # the CPU runs the whole 2M-point step (about 2-3 s on 8 cores)
CPU_BUDGET_S = 12.0


def cpu_baseline(cloud):
    """Reference CPU path (C restatement: single-threaded hash voxel, KD-tree
    radius normals threaded as staging.rs does), whole steps repeated for
    about CPU_BUDGET_S seconds."""
    import oracle
    oracle.build()
    crop = cpu_crop(cloud, CROP_SIDE)
    times = []
    t_start = time.perf_counter()
    while not times or (time.perf_counter() - t_start < CPU_BUDGET_S and len(times) < 8):
        t0 = time.perf_counter()
        cpu_step(crop)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    v = oracle.voxel_centroid(*crop[:3], [crop[3]], leaf=LEAVES[0])
    return dict(value=len(crop[0]) / t / 1e6, unit=UNIT, cores=cpu_threads(len(v.x)),
                kind="port", seconds_per_step=t,
                sample=(f"the full step on all {len(crop[0])} points, {len(times)} step(s), "
                        f"median {t:.2f} s; voxel single-threaded (voxel.rs:502-520), normals on "
                        f"{cpu_threads(len(v.x))} threads (staging.rs:11-41); C restatement of "
                        "the reference's CPU path (Rust is not buildable here)"))


REFERENCE_BUDGET_S = 90.0  # timed CPU work of the reference arm


def run_reference(args):
    """The reference's CPU path (C restatement) on the box's host cores.  Each
    step is a bounded sample of the workload: the full 2M-point step when K of
    them fit in about REFERENCE_BUDGET_S, else the x, y < side tile of the same
    cloud at full density, sized from one timed full step so that K steps take
    about that long."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    cloud = workload_cloud()
    import oracle
    oracle.build()
    full = cpu_crop(cloud, None)
    t0 = time.perf_counter()
    cpu_step(full)  # the first warm-up step, at full size, also sizes the sample
    t_full = time.perf_counter() - t0
    frac = min(1.0, REFERENCE_BUDGET_S / (max(args.steps, 1) * t_full))
    side = None if frac >= 1.0 else 200.0 * float(np.sqrt(frac))
    crop = cpu_crop(cloud, side)
    # the sample runs with the worker count the reference uses on the whole workload
    v = oracle.voxel_centroid(*full[:3], [full[3]], leaf=LEAVES[0])
    threads = cpu_threads(len(v.x))
    for _ in range(max(args.warmup - 1, 0)):
        cpu_step(crop, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu_step(crop, threads)
    t = (time.perf_counter() - t0) / args.steps
    value = len(crop[0]) / t / 1e6
    line = dict(
        impl="reference", metric=METRIC, value=value, unit=UNIT, n_gpus=args.gpus,
        steps=args.steps, warmup=args.warmup, ms_per_step=t * 1e3, higher_is_better=True,
        scaling="weak", vs_baseline=None, dtype="f32", data="synthetic",
        config=bench_config(args.gpus),
        cpu_baseline=dict(value=value, unit=UNIT, cores=threads, kind="port",
                          sample=(f"each step: {len(crop[0])} of the {N_POINTS} points "
                                  + ("(the whole cloud)" if side is None else
                                     f"(the x, y < {side:.1f} m tile at full density)")
                                  + "; the reference is Rust and cannot be built here, so its "
                                  "CPU path runs as the C restatement in oracle/")),
        e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0),
    )
    print(json.dumps(line), flush=True)


# ---- multi-rank plumbing (replicas: no data-path collective) ---------------

def max_over_ranks(x: float, device=None) -> float:
    """The max of x over all ranks (the job's time is its slowest rank's)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_mpts(world: int, points_per_rank: int, ms_per_step: float) -> float:
    """Whole-job throughput: every rank processes its own replica of the
    workload each step; the step takes the slowest rank's time."""
    return world * points_per_rank / (ms_per_step / 1e3) / 1e6


# ---- GPU --------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["nvidia-smi unavailable"])
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
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
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return dict(sm_mhz=statistics.median(sm) if sm else None,
                    sm_max_mhz=max(smax) if smax else None, reasons=sorted(reasons),
                    samples=len(sm))


def algorithmic_bytes(group: str, info: dict, n_attrs: int = 1) -> float:
    """Compulsory bytes of one launch group, per the per-unit figures of the
    path's byte model: voxel 16 B/point read + 28 B/voxel written (sort and
    segment groups at their implementation minimum), normals 12 B/point read +
    20 B/point written."""
    n, v, u = info["points"], info["voxels"], info["cells"]
    cols = 3 + n_attrs
    if group == "voxel_sort":
        return n * 12.0 + max(info["voxel_sort_passes"], 1) * n * 24.0
    if group == "cell_sort":
        return v * 12.0 + max(info["cell_sort_passes"], 1) * v * 24.0
    if group == "voxel_segments":
        return n * 12.0 + n * 4.0 * cols + v * (4.0 * cols + 12.0)
    if group == "cells":
        return v * 12.0 + v * 12.0 + v * 16.0 + u * 12.0
    if group == "normals":
        return v * 12.0 + v * 20.0
    if group in ("voxel_hist", "bounds"):
        return n * 12.0
    if group == "cell_hist":
        return v * 12.0
    if group == "ranges":
        return u * 9 * 8.0 + u * 12.0
    if group == "hash":
        return u * 16.0
    return 0.0


def summary(line: dict) -> dict:
    """The line's key figures, printed last (a reader of the line's tail sees them)."""
    r1 = lambda v: None if v is None else round(v, 1)  # noqa: E731
    out = dict(value=round(line["value"], 1), e2e=r1(line["e2e"]["value"]),
               e2e_one_step_in_flight=r1(line["e2e_one_step_in_flight"]["value"]),
               e2e_pageable=r1(line["e2e_pageable"]["value"]),
               graph=r1(line["graph"]["value"]) if "graph" in line else None,
               roofline_frac=round(line["roofline"]["frac"], 4),
               roofline_voxel_frac=[round(x["frac"], 4) for x in line["roofline_voxel"]["leaves"]])
    b = line.get("batched")
    if b:
        out["batched"] = {k: (round(b[k], 3) if isinstance(b.get(k), float) else b.get(k))
                          for k in ("plain_ms", "batched_ms", "graph_ms", "speedup",
                                    "graph_speedup") if k in b}
    sh = line.get("shapes")
    if sh:
        out["shapes"] = dict(ms=round(sh["ms"], 3), mpts_s=round(sh["mpts_s"], 1))
    sv = line.get("serving")
    if sv and sv.get("rates"):
        top = sv["rates"][-1]
        out["serving"] = {k: round(top[k], 3) for k in ("offered_req_s", "achieved_req_s",
                                                        "frame_p50_ms", "frame_p99_ms")}
    cb = line.get("cpu_baseline")
    if cb:
        out["cpu_baseline"] = dict(value=round(cb["value"], 3), cores=cb["cores"])
    return out


def run_gpu(args):
    import torch
    import torch.distributed as dist

    from spatialrust_b200 import _native

    world, rank, local = dist_env()
    if world > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    cloud = workload_cloud()
    # A dedicated stream: the library and the timing events must share it (the
    # legacy default stream's handle is 0, which srcu_set_stream reads as
    # "the context's own stream").
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    # one context per leaf so both chains' results stay resident
    ctxs = [_native.Context(local) for _ in LEAVES]
    # The two leaf chains are independent: each context gets its own stream,
    # forked from and joined back to the timing stream every step, so their
    # latency-bound phases overlap (--serial-leaves runs both on one stream).
    leaf_streams = [stream] * len(LEAVES) if args.serial_leaves else \
        [torch.cuda.Stream(dev) for _ in LEAVES]
    for c, s in zip(ctxs, leaf_streams):
        c.set_stream(s.cuda_stream)
        c.set_neighbor_staging(args.neighbor_walk)
    cols = [torch.from_numpy(a).to(dev) for a in (cloud.x, cloud.y, cloud.z, cloud.intensity)]
    keep = _native._Keep()
    dcloud = _native.make_cloud(cols[0], cols[1], cols[2], [cols[3]], keep)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    fork = torch.cuda.Event()
    joins = [torch.cuda.Event() for _ in LEAVES]

    def step():
        if not args.serial_leaves:
            fork.record(stream)
            for s in leaf_streams:
                s.wait_event(fork)
        for c, leaf in zip(ctxs, LEAVES):
            c.voxel_normals_enqueue(dcloud, leaf, None, RADIUS, 3, VIEWPOINT, count_shell=False)
        if not args.serial_leaves:
            for s, e in zip(leaf_streams, joins):
                e.record(s)
                stream.wait_event(e)

    # warm-up (also sizes every buffer)
    for _ in range(max(args.warmup, 3)):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    infos = []
    nstats = []
    for c in ctxs:
        nstats.append(c.frame_check()[1])
        infos.append(c.chain_info())

    # untimed profile passes: which kernel group dominates, with the two chains
    # run one after the other so every group's time is its own.  Per group the
    # median over the passes, so that one late launch does not pick the group.
    for c in ctxs:
        c.profile_read(reset=True)
        c.profile_enable(_native.KERNEL_IDS)
        c.set_stream(stream.cuda_stream)
    passes = []
    for _ in range(PROFILE_PASSES):
        flush.zero_()
        for c, leaf in zip(ctxs, LEAVES):
            c.voxel_normals_enqueue(dcloud, leaf, None, RADIUS, 3, VIEWPOINT, count_shell=False)
        torch.cuda.synchronize()
        passes.append([c.profile_read(reset=True) for c in ctxs])
    # the voxel stage of each leaf alone (srcu_voxel_centroid_enqueue), one pair
    # of CUDA events around the whole stage, L2 flushed before each, median of
    # PROFILE_PASSES
    voxel_chain_ms = []
    for c, leaf in zip(ctxs, LEAVES):
        c.profile_enable([])  # no events inside the timed stage
        ms = []
        for _ in range(PROFILE_PASSES + 1):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            c.voxel_centroid_enqueue(dcloud, leaf)
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        voxel_chain_ms.append(statistics.median(ms[1:]))
        c.frame_check()
        c.profile_read(reset=True)
    for c, s in zip(ctxs, leaf_streams):
        c.set_stream(s.cuda_stream)
    group_ms = {g: statistics.median(sum(p[g]["total_ms"] for p in ps) for ps in passes)
                for g in _native.KERNEL_IDS}  # ms per step (both leaves)
    iso_group = {g: (group_ms[g], sum(p[g]["timed_regions"] for p in passes[0]))
                 for g in _native.KERNEL_IDS}  # (ms, launches) per step
    dominant = max(group_ms, key=group_ms.get)
    if args.profile_all and rank == 0:
        tot = sum(group_ms.values())
        for g, ms in sorted(group_ms.items(), key=lambda kv: -kv[1]):
            print(f"  {g:16s} {ms:9.4f} ms/step  {100 * ms / tot:5.1f}%", file=sys.stderr)
    for c in ctxs:
        c.profile_enable([dominant])

    # timed region
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    for s in range(args.steps):
        flush.zero_()  # outside the timed events
        ev[s][0].record(stream)
        step()
        ev[s][1].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clock = clocks.stop()
    ms_steps = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(ms_steps)
    prof = [c.profile_read(reset=True) for c in ctxs]
    for c in ctxs:
        c.profile_enable([])
        c.frame_check()  # device status of the last chain: raises on any failure
    launches = sum(p[g]["launches"] for p in prof for g in _native.KERNEL_IDS)
    dom_ms = sum(p[dominant]["total_ms"] for p in prof)
    dom_regions = sum(p[dominant]["timed_regions"] for p in prof)
    dom_bytes = sum(algorithmic_bytes(dominant, info) for info in infos) / len(infos)
    max_ms = max_over_ranks(total_ms, dev)
    ms_per_step = max_ms / args.steps
    value = job_mpts(world, N_POINTS, ms_per_step)

    # the same step replayed from CUDA graphs: each leaf chain captured once
    # (srcu_chain_graph_create) and launched on its stream every step
    graphs = [c.chain_graph(dcloud, [leaf], [RADIUS], None, 3, [VIEWPOINT], False)
              for c, leaf in zip(ctxs, LEAVES)]

    def graph_step():
        if not args.serial_leaves:
            fork.record(stream)
            for s in leaf_streams:
                s.wait_event(fork)
        for g in graphs:
            g.launch()
        if not args.serial_leaves:
            for s, e in zip(leaf_streams, joins):
                e.record(s)
                stream.wait_event(e)

    for _ in range(max(args.warmup, 3)):
        flush.zero_()
        graph_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    gev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    for s in range(args.steps):
        flush.zero_()
        gev[s][0].record(stream)
        graph_step()
        gev[s][1].record(stream)
    torch.cuda.synchronize()
    graph_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in gev), dev) / args.steps
    for g in graphs:
        g.close()
    for c in ctxs:
        c.frame_check()
    graph = dict(value=job_mpts(world, N_POINTS, graph_ms), unit=UNIT, ms_per_step=graph_ms,
                 api="srcu_chain_graph_create once per leaf context, srcu_graph_launch of both "
                     "on the two leaf streams every step (same fork, join and L2 flush)")

    # end to end through the C ABI with pinned host buffers, then with plain
    # (pageable) numpy buffers as a Rust caller's Vecs are
    if args.no_e2e:
        skipped = dict(value=None, unit=UNIT, skipped="--no-e2e")
        e2e = e2e_one_step = e2e_pageable = skipped
    else:
        e2e = run_e2e(ctxs, leaf_streams, cloud, args, torch, dev, stream,
                      inflight=args.e2e_inflight)
        e2e_one_step = run_e2e(ctxs, leaf_streams, cloud, args, torch, dev, stream, inflight=1)
        e2e_pageable = run_e2e(ctxs, leaf_streams, cloud, args, torch, dev, stream, pinned=False,
                               inflight=args.e2e_inflight)

    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = json.load(open(pp))
    hbm = peaks.get("hbm_gbs", 6650.0)
    avg_launch_ms = dom_ms / max(dom_regions, 1)
    achieved = dom_bytes / (avg_launch_ms / 1e3) / 1e9 if dom_regions else 0.0
    iso_ms, iso_regions = iso_group[dominant]
    iso_launch_ms = iso_ms / max(iso_regions, 1)
    iso_achieved = dom_bytes / (iso_launch_ms / 1e3) / 1e9 if iso_regions else 0.0
    roofline = dict(bound="hbm", kernel=dominant, achieved=achieved, peak=hbm, unit="GB/s",
                    frac=achieved / hbm, traffic=MEASURED_TRAFFIC.get(dominant),
                    traffic_source=("ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, "
                                    "profiles/dram_per_kernel_georef2M.md")
                    if dominant in MEASURED_TRAFFIC else None,
                    note=("the normals kernel is bound by issue and L1 latency on its "
                          "candidate walk (ncu: 65% issue active, 3% of DRAM peak), not by HBM")
                    if dominant == "normals" else None,
                    peak_source="MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks
                    else "fallback 6650 GB/s",
                    algorithmic_bytes_per_launch=dom_bytes, avg_launch_ms=avg_launch_ms,
                    isolated_split_ms={g: round(ms, 4) for g, ms in
                                       sorted(group_ms.items(), key=lambda kv: -kv[1]) if ms > 0},
                    timing=("CUDA events around each launch of the group in the timed region, "
                            "where the two leaf chains share the GPU" if not args.serial_leaves
                            else "CUDA events around each launch of the group in the timed region"),
                    isolated_avg_launch_ms=iso_launch_ms, isolated_achieved=iso_achieved,
                    isolated_frac=iso_achieved / hbm,
                    step_share=group_ms[dominant] / max(sum(group_ms.values()), 1e-9))
    # The voxel downsample alone against the HBM roofline: compulsory bytes
    # 16 B/point read + 28 B/voxel written (centroid + intensity, packed key,
    # count) over its kernels' time (bounds, plan, sort, segments), per leaf.
    vox_bytes = [N_POINTS * 16.0 + i["voxels"] * 28.0 for i in infos]
    roofline_voxel = dict(
        bound="hbm", unit="GB/s", peak=hbm,
        leaves=[dict(leaf=leaf, voxels=i["voxels"], algorithmic_bytes=b, chain_ms=ms,
                     achieved=b / (ms / 1e3) / 1e9, frac=b / (ms / 1e3) / 1e9 / hbm,
                     split_ms={g: round(statistics.median(ps[k][g]["total_ms"] for ps in passes), 4)
                               for g in VOXEL_GROUPS})
                for k, (leaf, i, b, ms) in enumerate(zip(LEAVES, infos, vox_bytes, voxel_chain_ms))],
        timing=("each leaf's voxel stage alone (srcu_voxel_centroid_enqueue: bounds, plan, sort, "
                "segments): one pair of CUDA events around it, L2 flushed before, median of "
                f"{PROFILE_PASSES}; split_ms: the isolated profile passes' per-group events"),
        byte_model="16 B/point read + 28 B/voxel written")
    line = dict(
        metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps,
        warmup=args.warmup, ms_per_step=ms_per_step, higher_is_better=True, scaling="weak",
        vs_baseline=None, dtype="f32", data="synthetic",
        config=bench_config(world),
        details=dict(voxels=[i["voxels"] for i in infos], cells=[i["cells"] for i in infos],
                     sort_passes=[[i["voxel_sort_passes"], i["cell_sort_passes"]] for i in infos],
                     normals=[{k: st[k] for k in ("valid_count", "invalid_count", "fp64_eigensolves")}
                              for st in nstats],
                     neighbor_walk=ctxs[0].neighbor_staging(),
                     l2="flushed by a 256 MB write before every timed step (outside the events)",
                     leaf_chains=("one stream, one after the other" if args.serial_leaves else
                                  "two streams (one context each), forked and joined every step")),
        e2e=e2e, e2e_one_step_in_flight=e2e_one_step, e2e_pageable=e2e_pageable,
        graph=graph, roofline=roofline, roofline_voxel=roofline_voxel,
        clocks=clock, gpu_launches=int(launches),
    )
    if not args.no_batched:
        line["batched"] = run_batched(args, torch, dev, stream)
    if not args.no_shapes:
        line["shapes"] = run_shapes(args, torch, dev, stream)
    if not args.no_cluster and rank == 0:
        line["cluster"] = run_cluster(args, torch, dev, stream, cloud)
    if not args.no_plane_cov and rank == 0:
        line["plane_cov"] = run_plane_cov(args, torch, dev, stream, cloud)
    if not args.no_ransac and rank == 0:
        line["ransac"] = run_ransac(args, torch, dev, stream, cloud)
    if not args.no_las_stream and rank == 0:
        line["las_stream"] = run_las_stream(args, torch, dev, stream, cloud)
    if not args.no_serving:
        line["serving"] = run_serving(args, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cloud)
    line["summary"] = summary(line)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    for c in ctxs:
        c.close()


def run_batched(args, torch, dev, stream):
    """Many uneven clouds: 256 clouds, sizes log-uniform in [10k, 1M] (~52M points),
    each the georeferenced scan mixture with its own seed and FP64 origin offset
    (up to 1e6 m), leaf in {0.05, 0.1, 0.2} m and normals at r = 5 x leaf.
    One batched chain (cloud id in the key high bits), as enqueued and as a
    replayed CUDA graph, against the plain loop of one chain per cloud."""
    from spatialrust_b200 import _native, synthetic
    clouds, leaves, radii = synthetic.batched_uneven(args.batched_clouds, seed=3,
                                                     scale=args.batched_scale)
    n = sum(c.n for c in clouds)
    cols = [torch.from_numpy(np.concatenate([getattr(c, k) for c in clouds])).to(dev)
            for k in ("x", "y", "z", "intensity")]
    offsets = np.concatenate([[0], np.cumsum([c.n for c in clouds])]).astype(np.int64)
    keep = _native._Keep()
    ctx = _native.Context(dev.index)
    ctx.set_stream(stream.cuda_stream)
    allc = _native.make_cloud(cols[0], cols[1], cols[2], [cols[3]], keep)
    vps = [VIEWPOINT] * len(clouds)
    per = [_native.make_cloud(*(c[offsets[b]:offsets[b + 1]] for c in cols[:3]),
                              [cols[3][offsets[b]:offsets[b + 1]]], keep)
           for b in range(len(clouds))]

    def plain():
        for b in range(len(clouds)):
            ctx.voxel_normals_enqueue(per[b], float(leaves[b]), None, float(radii[b]), 3, VIEWPOINT,
                                      count_shell=False)

    def batched():
        ctx.batch_voxel_normals_enqueue(allc, offsets, leaves.tolist(), radii.tolist(), 3, vps,
                                        count_shell=False)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    ms_plain = timed(plain, 2)
    ms_batched = timed(batched, 3)
    voxels = int(ctx.batch_voxel_offsets()[-1])
    info = ctx.chain_info()
    # where the batched chain spends its time (an untimed, event-bracketed pass)
    ctx.profile_read(reset=True)
    ctx.profile_enable(_native.KERNEL_IDS)
    batched()
    torch.cuda.synchronize()
    prof = ctx.profile_read(reset=True)
    ctx.profile_enable([])
    groups = {g: round(p["total_ms"], 3) for g, p in prof.items() if p["total_ms"] > 0}
    out = dict(workload=f"{len(clouds)} clouds, {n} points, log-uniform 10k-1M, leaf 0.05/0.1/0.2, "
                        "r = 5 x leaf", points=n, voxels=voxels,
               plain_ms=ms_plain, batched_ms=ms_batched,
               plain_mpts=n / ms_plain / 1e3, batched_mpts=n / ms_batched / 1e3,
               speedup=ms_plain / ms_batched, cells=info["cells"],
               sort_passes=[info["voxel_sort_passes"], info["cell_sort_passes"]],
               key_bits=[info["voxel_key_bits"], info["cell_key_bits"]], group_ms=groups)
    try:  # the same batched chain replayed from a CUDA graph
        g = ctx.chain_graph(allc, leaves.tolist(), radii.tolist(), offsets=offsets, viewpoints=vps)
        ms_graph = timed(g.launch, 3)
        out.update(graph_ms=ms_graph, graph_mpts=n / ms_graph / 1e3, graph_speedup=ms_plain / ms_graph)
        g.close()
    except Exception as e:
        out["graph_error"] = str(e)[:200]
    ctx.frame_check()
    ctx.close()
    return out


def run_shapes(args, torch, dev, stream):
    """Radius normals at scale: 5,000,000 points on 50 spheres, 30 planar
    patches and 20 cylinders with N(0, 0.005) surface noise, r = 0.3 m,
    uncapped neighbourhoods; device-resident input and output, one
    srcu_radius_normals call per step.  Reports the neighbour-count
    distribution the shapes actually give."""
    from spatialrust_b200 import _native, synthetic
    lib = _native.load()
    cloud = synthetic.shapes_scene(5_000_000, seed=2)
    n = cloud.n
    cols = [torch.from_numpy(a).to(dev) for a in (cloud.x, cloud.y, cloud.z)]
    outs = [torch.empty(n, dtype=torch.float32, device=dev) for _ in range(4)]
    counts = torch.empty(n, dtype=torch.int32, device=dev)
    keep = _native._Keep()
    dcloud = _native.make_cloud(cols[0], cols[1], cols[2], [], keep)
    nout = _native.SrcuNormalOut(*[o.data_ptr() for o in outs], counts.data_ptr(), 1)
    params = _native._normal_params(0.3, 3, None, False, count_shell=True)
    stats = _native.SrcuNormalStats()
    ctx = _native.Context(dev.index)
    ctx.set_stream(stream.cuda_stream)

    def step():
        ctx._check(lib.srcu_radius_normals(ctx.handle, ctypes.byref(dcloud), ctypes.byref(params),
                                           ctypes.byref(nout), ctypes.byref(stats)))

    for _ in range(2):
        step()
    torch.cuda.synchronize()
    reps = 5
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        step()
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    nb = counts.cpu().numpy()
    pct = np.percentile(nb, [5, 25, 50, 75, 95]).tolist()
    info = ctx.chain_info()
    ctx.close()
    return dict(workload="shapes 5M (spheres/planes/cylinders, noise 0.005), radius normals r 0.3",
                points=n, ms=ms, mpts_s=n / ms / 1e3, cells=info["cells"],
                neighbours=dict(mean=float(nb.mean()), p5=pct[0], p25=pct[1], p50=pct[2],
                                p75=pct[3], p95=pct[4], max=int(nb.max())),
                stats=_native._stats(stats))


def run_cluster(args, torch, dev, stream, cloud):
    """Euclidean cluster roots (srcu_euclidean_cluster_roots) on the 2M-point
    georeferenced scan at tolerance 0.1 and 0.3 m, device-resident; its CPU
    baseline is the reference's sparse-cell union-find (C restatement, one
    thread) on the same points."""
    import oracle
    from spatialrust_b200 import _native
    lib = _native.load()
    n = cloud.n
    cols = [torch.from_numpy(a).to(dev) for a in (cloud.x, cloud.y, cloud.z)]
    roots = torch.empty(n, dtype=torch.int32, device=dev)
    keep = _native._Keep()
    dcloud = _native.make_cloud(cols[0], cols[1], cols[2], [], keep)
    ctx = _native.Context(dev.index)
    ctx.set_stream(stream.cuda_stream)
    out = dict(workload="georef_scan_2M: Euclidean cluster roots", points=n, tolerances=[])
    for tol in (0.1, 0.3):
        def step():
            ctx._check(lib.srcu_euclidean_cluster_roots(ctx.handle, ctypes.byref(dcloud),
                                                        ctypes.c_float(tol), roots.data_ptr()))
        for _ in range(2):
            step()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(5):
            step()
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / 5
        r = roots.cpu().numpy().view(np.uint32)
        entry = dict(tolerance=tol, ms=ms, mpts_s=n / ms / 1e3,
                     components=int(len(np.unique(r))))
        if not args.no_cpu_baseline:
            t0 = time.perf_counter()
            oracle.euclidean_roots(cloud.x, cloud.y, cloud.z, tol, sparse=True)
            cpu_s = time.perf_counter() - t0
            entry["cpu_baseline"] = dict(
                value=n / cpu_s / 1e6, unit="Mpoints/s", cores=1, kind="port",
                sample=f"all {n} points once: the reference's sparse-cell union-find "
                       "(euclidean_cluster.rs -> uniform_grid.rs:148-250), C restatement")
        out["tolerances"].append(entry)
    ctx.close()
    return out


def hbm_peak():
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(pp)) if os.path.exists(pp) else {}
    return peaks.get("hbm_gbs", 6650.0), ("MEASURED_PEAKS.json hbm_gbs (measured)"
                                          if "hbm_gbs" in peaks else "fallback 6650 GB/s")


PLANE_RADIUS = 0.3
PLANE_EPS = 1e-3


def run_plane_cov(args, torch, dev, stream, cloud):
    """GICP plane covariances (srcu_plane_covariances) of every point of the
    2M-point scan, radius 0.3 m, eps 1e-3, device-resident in and out; CPU
    baseline: the FP64 oracle (KD-tree radius neighbourhoods, all host
    threads) on the same points."""
    import oracle
    from spatialrust_b200 import _native
    lib = _native.load()
    n = cloud.n
    cols = [torch.from_numpy(a).to(dev) for a in (cloud.x, cloud.y, cloud.z)]
    cov = torch.empty((n, 6), dtype=torch.float32, device=dev)
    keep = _native._Keep()
    dcloud = _native.make_cloud(cols[0], cols[1], cols[2], [], keep)
    ctx = _native.Context(dev.index)
    ctx.set_stream(stream.cuda_stream)
    stats = _native.SrcuNormalStats()

    def step():
        ctx._check(lib.srcu_plane_covariances(ctx.handle, ctypes.byref(dcloud),
                                              ctypes.c_float(PLANE_RADIUS),
                                              ctypes.c_float(PLANE_EPS), cov.data_ptr(),
                                              ctypes.byref(stats)))
    for _ in range(3):
        step()
    ctx.profile_enable(["normals"])
    ctx.profile_read(reset=True)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 5
    a.record(stream)
    for _ in range(reps):
        step()
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    prof = ctx.profile_read(reset=True)["normals"]
    kernel_ms = prof["total_ms"] / max(prof["timed_regions"], 1)
    out = dict(workload=f"georef_scan_2M: GICP plane covariances r {PLANE_RADIUS} eps {PLANE_EPS}",
               points=n, ms=ms, mpts_s=n / ms / 1e3, kernel_ms=kernel_ms,
               valid=int(stats.valid_count), fallback=int(stats.invalid_count),
               fp64_eigensolves=int(stats.fp64_eigensolves),
               timing="CUDA events around 5 synchronous calls (grid build + covariance kernel)")
    if not args.no_cpu_baseline:
        t0 = time.perf_counter()
        oracle.plane_covariances(cloud.x, cloud.y, cloud.z, PLANE_RADIUS, PLANE_EPS)
        cpu_s = time.perf_counter() - t0
        out["cpu_baseline"] = dict(
            value=n / cpu_s / 1e6, unit="Mpoints/s", cores=os.cpu_count() or 1, kind="port",
            sample=f"all {n} points once: KD-tree radius neighbourhoods, FP64 covariance and "
                   "Jacobi, C restatement of covariances_grid.rs:87-206")
    ctx.close()
    return out


RANSAC_POINTS = 460_000   # the size of the reference's own full-cloud RANSAC measurement
RANSAC_ITERS = 1000
RANSAC_THRESHOLD = 0.01


def run_ransac(args, torch, dev, stream, cloud):
    """RANSAC plane segmentation (srcu_ransac_plane_segment) of the first 460k
    points of the scan (ground plane + boxes + clutter), 1000 hypotheses,
    threshold 0.01, seed 42, positions device-resident; CPU baseline: the
    reference's CPU segmenter (C restatement, one thread) on the same points."""
    import oracle
    from spatialrust_b200 import _native
    n = RANSAC_POINTS
    x, y, z = (np.ascontiguousarray(a[:n]) for a in (cloud.x, cloud.y, cloud.z))
    cols = [torch.from_numpy(a).to(dev) for a in (x, y, z)]
    ctx = _native.Context(dev.index)
    ctx.set_stream(stream.cuda_stream)

    def step():
        return ctx.ransac_plane_segment(*cols, RANSAC_THRESHOLD, RANSAC_ITERS, 3, 42)
    for _ in range(3):
        step()
    ctx.profile_enable(["ransac"])
    ctx.profile_read(reset=True)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 10
    a.record(stream)
    for _ in range(reps):
        info, _ = step()
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    prof = ctx.profile_read(reset=True)["ransac"]
    ctx.profile_enable([])
    evals = n * RANSAC_ITERS
    out = dict(workload=(f"georef scan, first {n} points: RANSAC plane, {RANSAC_ITERS} "
                         f"hypotheses, threshold {RANSAC_THRESHOLD}, seed 42"),
               points=n, ms=ms, kernels_ms=prof["total_ms"] / reps,
               gevals_s=evals / ms / 1e6, inliers=info["inlier_count"],
               timing="CUDA events around 10 synchronous calls (hypotheses, scoring, selection, "
                      "mask, FP64 refine)")
    if not args.no_cpu_baseline:
        t0 = time.perf_counter()
        ref = oracle.ransac_plane(x, y, z, RANSAC_THRESHOLD, RANSAC_ITERS, 3, 42)
        cpu_s = time.perf_counter() - t0
        out["cpu_baseline"] = dict(
            value=1e3 * cpu_s, unit="ms", cores=1, kind="port",
            sample=f"the same {n} points, once: RansacPlaneSegmenter::segment_cpu "
                   "(plane.rs:266-345), C restatement, one thread",
            same_answer=bool(ref["inlier_count"] == info["inlier_count"]
                             and ref["best_index"] == info["best_hypothesis"]))
    ctx.close()
    return out


LAS_TILES = 8          # the 2M scan tiled 8 times, 250 m apart in x: 16M points
LAS_CHUNK = 1 << 20    # records per decode call / points per streaming push
STREAM_LEAF = 0.1


def run_las_stream(args, torch, dev, stream, cloud):
    """LAS ingest -> bounded streaming voxel.  16M LAS 1.4 point-format-1
    records (28 B: mm-scaled i32 XYZ, intensity, classification, GPS time) of
    the scan tiled 8x, decoded on the device with the FP64 origin subtracted
    (srcu_las_decode), then pushed in 1M-point chunks through the streaming
    voxel at leaf 0.1 with intensity (f32) and GPS time (f64) averaged
    (srcu_stream_voxel_*).  decode: device-resident records -> columns, kernel
    time by CUDA events; stream: device-resident columns -> voxels; e2e:
    pinned host LAS bytes -> H2D + decode per chunk -> push -> finish -> all
    voxels fetched to the host."""
    import oracle
    from spatialrust_b200 import _native, las
    n1 = cloud.n
    n = n1 * LAS_TILES
    origin = tuple(float(v) for v in cloud.origin)
    wx = np.concatenate([cloud.x.astype(np.float64) + origin[0] + 250.0 * t
                         for t in range(LAS_TILES)])
    wy = np.tile(cloud.y.astype(np.float64) + origin[1], LAS_TILES)
    wz = np.tile(cloud.z.astype(np.float64) + origin[2], LAS_TILES)
    buf = las.encode_las(wx, wy, wz, point_format=1, scale=(0.001,) * 3,
                         offset=tuple(np.floor(origin)),
                         intensity=np.tile((cloud.intensity * 65535).astype(np.int64), LAS_TILES),
                         classification=np.arange(n) % 8,
                         gps_time=1.4e9 + np.arange(n) * 1e-5)
    del wx, wy, wz
    h = las.parse_header(buf)
    rl = h.record_length
    pinned = torch.empty(n * rl, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = np.frombuffer(buf, np.uint8, n * rl, h.offset_to_point_data)
    rec_dev = pinned.to(dev)
    ctx = _native.Context(dev.index)
    ctx.set_stream(stream.cuda_stream)
    lib = ctx._lib
    f32 = dict(dtype=torch.float32, device=dev)
    cols = dict(x=torch.empty(n, **f32), y=torch.empty(n, **f32), z=torch.empty(n, **f32),
                intensity=torch.empty(n, **f32),
                classification=torch.empty(n, dtype=torch.uint8, device=dev),
                gps_time=torch.empty(n, dtype=torch.float64, device=dev))
    fmt = _native.SrcuLasFormat(1, rl, (ctypes.c_double * 3)(*h.scale),
                                (ctypes.c_double * 3)(*h.offset), 1, 0,
                                (ctypes.c_double * 3)(*origin))

    def las_out(lo, hi):
        ptrs = [cols[k][lo:hi].data_ptr() for k in
                ("x", "y", "z", "intensity", "classification", "gps_time")]
        return _native.SrcuLasOut(*ptrs, 0, 0, 0, 1)

    full_out = las_out(0, n)

    def decode_all():
        ctx._check(lib.srcu_las_decode(ctx.handle, ctypes.c_void_p(rec_dev.data_ptr()), n, 1,
                                       ctypes.byref(fmt), ctypes.byref(full_out)))
    for _ in range(3):
        decode_all()
    ctx.profile_enable(["las_decode"])
    ctx.profile_read(reset=True)
    for _ in range(10):
        decode_all()
    prof = ctx.profile_read(reset=True)["las_decode"]
    ctx.profile_enable([])
    dec_ms = prof["total_ms"] / max(prof["timed_regions"], 1)
    bytes_per_rec = rl + 4 * 4 + 1 + 8
    hbm, peak_src = hbm_peak()
    achieved = n * bytes_per_rec / (dec_ms / 1e3) / 1e9

    def stream_all():
        sv = _native.StreamVoxel(ctx, STREAM_LEAF, [False, True])
        for lo in range(0, n, LAS_CHUNK):
            hi = min(n, lo + LAS_CHUNK)
            sv.push(cols["x"][lo:hi], cols["y"][lo:hi], cols["z"][lo:hi],
                    [cols["intensity"][lo:hi], cols["gps_time"][lo:hi]])
        info = sv.finish()
        return sv, info

    sv, info = stream_all()
    sv.close()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3
    t0 = time.perf_counter()
    a.record(stream)
    for _ in range(reps):
        sv, info = stream_all()
        sv.close()
    b.record(stream)
    torch.cuda.synchronize()
    stream_ms = a.elapsed_time(b) / reps
    stream_wall_ms = (time.perf_counter() - t0) * 1e3 / reps

    vmax = n  # voxel capacity of the pinned result buffers
    res_host = dict(x=torch.empty(vmax, dtype=torch.float32, pin_memory=True),
                    y=torch.empty(vmax, dtype=torch.float32, pin_memory=True),
                    z=torch.empty(vmax, dtype=torch.float32, pin_memory=True),
                    intensity=torch.empty(vmax, dtype=torch.float64, pin_memory=True),
                    gps_time=torch.empty(vmax, dtype=torch.float64, pin_memory=True))
    attr_ptrs = (ctypes.c_void_p * 2)(res_host["intensity"].data_ptr(),
                                      res_host["gps_time"].data_ptr())
    fetch_out = _native.SrcuStreamVoxelOut(res_host["x"].data_ptr(), res_host["y"].data_ptr(),
                                           res_host["z"].data_ptr(),
                                           ctypes.cast(attr_ptrs, ctypes.c_void_p), None, None, 0)

    # the records of chunk k + 1 cross the link on their own stream while chunk k
    # is decoded and pushed (two device staging buffers)
    copy_stream = torch.cuda.Stream(dev)
    stage = [torch.empty(LAS_CHUNK * rl, dtype=torch.uint8, device=dev) for _ in range(2)]
    copied = [torch.cuda.Event() for _ in range(2)]
    chunks = [(lo, min(n, lo + LAS_CHUNK)) for lo in range(0, n, LAS_CHUNK)]

    def h2d(k):
        lo, hi = chunks[k]
        with torch.cuda.stream(copy_stream):
            stage[k & 1][:(hi - lo) * rl].copy_(pinned[lo * rl:hi * rl], non_blocking=True)
            copied[k & 1].record(copy_stream)

    def e2e_once():
        sv = _native.StreamVoxel(ctx, STREAM_LEAF, [False, True])
        h2d(0)
        for k, (lo, hi) in enumerate(chunks):
            if k + 1 < len(chunks):
                h2d(k + 1)  # its buffer's previous decode has returned
            stream.wait_event(copied[k & 1])
            o = las_out(lo, hi)
            ctx._check(lib.srcu_las_decode(ctx.handle, ctypes.c_void_p(stage[k & 1].data_ptr()),
                                           hi - lo, 1, ctypes.byref(fmt), ctypes.byref(o)))
            sv.push(cols["x"][lo:hi], cols["y"][lo:hi], cols["z"][lo:hi],
                    [cols["intensity"][lo:hi], cols["gps_time"][lo:hi]])
        inf = sv.finish()
        ctx._check(lib.srcu_stream_voxel_fetch(sv._h, 0, inf["voxels"], ctypes.byref(fetch_out)))
        sv.close()
        return inf, None
    e2e_once()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    a.record(stream)
    inf, res = e2e_once()
    b.record(stream)
    torch.cuda.synchronize()
    e2e_ms = a.elapsed_time(b)
    wall_ms = (time.perf_counter() - t0) * 1e3
    out = dict(
        workload=(f"LAS 1.4 format 1 ({rl} B records, mm scale), {n} points (georef scan x"
                  f"{LAS_TILES}) -> FP64-origin decode -> streaming voxel leaf {STREAM_LEAF} "
                  "(intensity f32 + GPS time f64 averaged)"),
        points=n, voxels=int(info["voxels"]), device_runs=int(info["device_runs"]),
        partial_records=int(info["partial_records"]),
        decode=dict(kernel_ms=dec_ms, grecords_s=n / dec_ms / 1e6,
                    roofline=dict(bound="hbm", achieved=achieved, peak=hbm, unit="GB/s",
                                  frac=achieved / hbm, peak_source=peak_src,
                                  algorithmic_bytes_per_record=bytes_per_rec)),
        stream=dict(ms=stream_ms, wall_ms=stream_wall_ms, mpts_s=n / stream_ms / 1e3,
                    timing="CUDA events around 3 device-resident streams (16 pushes + finish)"),
        e2e=dict(ms=e2e_ms, wall_ms=wall_ms, mpts_s=n / e2e_ms / 1e3,
                 h2d_bytes=n * rl, d2h_bytes=int(inf["voxels"]) * (12 + 8 * 2),
                 api="pinned host records -> device (chunk k + 1 copied on a second stream while "
                     "chunk k is decoded) -> srcu_las_decode -> srcu_stream_voxel_push/finish/"
                     "fetch (positions and both attribute means into pinned host buffers)"),
    )
    if not args.no_cpu_baseline:
        rec1 = pinned.numpy()[: n1 * rl]
        t0 = time.perf_counter()
        d = oracle.las_decode(rec1, 1, rl, h.scale, h.offset, origin)
        oracle.stream_voxel(d["x"], d["y"], d["z"], [d["intensity"], d["gps_time"]], leaf=STREAM_LEAF)
        cpu_s = time.perf_counter() - t0
        out["cpu_baseline"] = dict(
            value=n1 / cpu_s / 1e6, unit="Mpoints/s", cores=1, kind="port",
            sample=f"the first {n1} records once: LAS decode + global streaming voxel "
                   "(streaming.rs:414-676 semantics, C restatement, one thread, no disk spool)")
    del rec_dev, pinned
    ctx.close()
    return out


def run_serving(args, device):
    """The serving loop (srcu_server_*) under open-loop Poisson arrivals.

    Requests: spinning-LiDAR frames (64 beams x 2048 azimuths = 131,072
    points, ray-cast against ground + 100 boxes, max range 120 m, N(0, 0.02)
    range noise) and, with probability 0.1, map chunks of 1-4M points (the
    scan mixture); each runs voxel 0.2 m -> radius normals 0.6 m.  Frames and
    chunks arrive as two independent Poisson streams (0.9 and 0.1 of the
    offered rate, i.e. one Poisson stream whose requests are chunks with
    probability 0.1).  Each stream's arrival clock runs in its own host thread,
    which hands every arrival to a small pool of submitting threads (2 for
    frames, 4 for chunks: a chunk's copy into the pinned arena takes ~10 ms);
    another thread polls results.  Latency = submit -> results in pinned host
    memory."""
    import threading

    from spatialrust_b200 import _native, synthetic
    scene = synthetic.lidar_scene(seed=4)
    frames = [synthetic.lidar_frame(seed=i, scene=scene) for i in range(4)]
    chunks = [synthetic.map_chunk(n, seed=50 + i)
              for i, n in enumerate((1_000_000, 2_500_000, 4_000_000))]
    srv = _native.Server(device, hbm_budget_bytes=40 << 30)
    leaf, radius = 0.2, 0.6
    next_id = [0]
    id_lock = threading.Lock()

    def submit(c):
        with id_lock:
            rid = next_id[0]
            next_id[0] += 1
        while not srv.submit(rid, c.x, c.y, c.z, c.intensity, leaf=leaf, radius=radius):
            time.sleep(0.0005)  # queue full: back off (counted as rejected by the server)

    def drain(count):
        got = 0
        while got < count:
            if srv.poll(wait_us=5000, fetch=False) is not None:
                got += 1

    # warm-up: every frame and chunk once, then a short burst
    for c in frames + chunks:
        submit(c)
    drain(len(frames) + len(chunks))
    out = dict(workload="LiDAR frames 64x2048 (131,072 pts) + 10% map chunks 1M/2.5M/4M pts; "
                        "voxel 0.2 m -> normals r 0.6 m; Poisson arrivals; HBM budget 40 GB; "
                        "3 batch slots (<= 1M pts per batched chain) + 1 bulk slot",
               rates=[])
    for rate in [float(r) for r in args.serving_rates.split(",") if r]:
        srv.reset_stats()
        done = threading.Event()
        counts = {"frames": 0, "chunks": 0, "points": 0}

        from concurrent.futures import ThreadPoolExecutor
        count_lock = threading.Lock()

        def submit_counted(c, key):
            submit(c)
            with count_lock:
                counts[key] += 1
                counts["points"] += c.n

        def stream_of(pool, share, key, seed, workers):
            # Arrival times are kept by this thread; each arrival is handed to a
            # worker, so one slow copy (a 4M-point chunk is 64 MB) does not
            # delay the arrivals behind it.
            rng = np.random.default_rng(seed)
            t_next = time.perf_counter()
            end = t_next + args.serving_seconds
            k = 0
            with ThreadPoolExecutor(max_workers=workers) as ex:
                while True:
                    t_next += rng.exponential(1.0 / (rate * share))
                    if t_next >= end:
                        break
                    while True:
                        dt = t_next - time.perf_counter()
                        if dt <= 0:
                            break
                        time.sleep(dt if dt > 0.002 else 0)
                    c = pool[k % len(pool)]
                    k += 1
                    ex.submit(submit_counted, c, key)

        t0 = time.perf_counter()
        ths = [threading.Thread(target=stream_of, args=(frames, 0.9, "frames", int(rate), 2)),
               threading.Thread(target=stream_of, args=(chunks, 0.1, "chunks", int(rate) + 7, 4))]
        for t in ths:
            t.start()
        poller_count = [0]

        def poller():
            while not (done.is_set() and poller_count[0] >= counts["frames"] + counts["chunks"]):
                if srv.poll(wait_us=2000, fetch=False) is not None:
                    poller_count[0] += 1

        pt = threading.Thread(target=poller)
        pt.start()
        for t in ths:
            t.join()
        done.set()
        pt.join()
        wall = time.perf_counter() - t0
        st = srv.stats()
        n_req = counts["frames"] + counts["chunks"]
        out["rates"].append(dict(
            offered_req_s=rate, requests=n_req, frames=counts["frames"], chunks=counts["chunks"],
            achieved_req_s=n_req / wall, mpts_s=counts["points"] / wall / 1e6,
            frame_p50_ms=st["frame_p50_ms"], frame_p99_ms=st["frame_p99_ms"],
            chunk_p50_ms=st["bulk_p50_ms"], chunk_p99_ms=st["bulk_p99_ms"],
            all_p50_ms=st["all_p50_ms"], all_p99_ms=st["all_p99_ms"], batches=st["batches"],
            rejected_submits=st["rejected"], failed=st["failed"], wall_s=wall))
    srv.close()
    return out


E2E_INFLIGHT = 2  # steps in flight in the e2e measurement


def run_e2e(ctxs, leaf_streams, cloud, args, torch, dev, stream, pinned=True,
            inflight=E2E_INFLIGHT):
    """Synchronous srcu_voxel_normals calls with host inputs and outputs, one
    call per leaf and step: pinned buffers, or (pinned=False) plain numpy arrays
    in pageable memory, as the reference's Rust arm passes its Vecs.  `inflight`
    steps run at once, as a caller with a stream of clouds would run them: one
    host thread per (slot, leaf), each on its own context and stream with its
    own output buffers, slot s taking steps s, s + inflight, ...; every call
    copies its inputs to the device and its results back inside the timed
    region (--serial-leaves: one thread, one step at a time).  Device time:
    every stream waits on the start event, and the timing stream joins them all
    before the end event."""
    import threading

    from spatialrust_b200 import _native
    lib = _native.load()
    serial = args.serial_leaves
    if serial:
        inflight = 1
    slots = max(1, inflight)
    slot_ctxs = [list(ctxs)] + [[_native.Context(dev.index) for _ in LEAVES]
                                for _ in range(slots - 1)]
    slot_streams = [([stream] * len(LEAVES) if serial else list(leaf_streams))] + [
        [torch.cuda.Stream(dev) for _ in LEAVES] for _ in range(slots - 1)]
    for cs, ss in zip(slot_ctxs, slot_streams):
        for c, st in zip(cs, ss):
            c.set_stream(st.cuda_stream)
            c.set_neighbor_staging(args.neighbor_walk)
    n = cloud.n

    def host(a):  # a torch CPU tensor: pinned, or a view of a pageable numpy array
        return a.pin_memory() if pinned else a

    pin = [host(torch.from_numpy(a.copy())) for a in (cloud.x, cloud.y, cloud.z, cloud.intensity)]
    keep = _native._Keep()
    attr_in = keep.add((ctypes.c_void_p * 1)(pin[3].data_ptr()))
    hcloud = _native.SrcuCloud(pin[0].data_ptr(), pin[1].data_ptr(), pin[2].data_ptr(),
                               ctypes.cast(attr_in, ctypes.c_void_p), 1, 0, n)
    outs = {}
    for sl in range(slots):
        for k in range(len(LEAVES)):
            vcols = [host(torch.empty(n, dtype=torch.float32)) for _ in range(4)]
            ncols = [host(torch.empty(n, dtype=torch.float32)) for _ in range(4)]
            attr_out = keep.add((ctypes.c_void_p * 1)(vcols[3].data_ptr()))
            # the reference's output schema: centroid columns and the four normal
            # columns (no per-voxel or neighbour counts)
            vout = _native.SrcuVoxelOut(vcols[0].data_ptr(), vcols[1].data_ptr(),
                                        vcols[2].data_ptr(), ctypes.cast(attr_out, ctypes.c_void_p),
                                        0, 0, 0)
            nout = _native.SrcuNormalOut(*[c.data_ptr() for c in ncols], 0, 0)
            outs[sl, k] = (vcols, ncols, vout, nout, ctypes.c_uint64(0), _native.SrcuNormalStats())
    params = [(_native._voxel_params(leaf, None),
               _native._normal_params(RADIUS, 3, VIEWPOINT, False, count_shell=False))
              for leaf in LEAVES]
    voxels = [0] * len(LEAVES)
    errors = []

    def call(sl, k):
        vp, np_ = params[k]
        _, _, vout, nout, nv, stats = outs[sl, k]
        st = lib.srcu_voxel_normals(slot_ctxs[sl][k].handle, ctypes.byref(hcloud),
                                    ctypes.byref(vp), ctypes.byref(np_), ctypes.byref(vout),
                                    ctypes.byref(nout), ctypes.byref(nv), ctypes.byref(stats))
        if st != 0:
            errors.append((sl, k, st))
        voxels[k] = int(nv.value)

    def run(steps):
        if serial:
            for _ in range(steps):
                for k in range(len(LEAVES)):
                    call(0, k)
        else:
            def worker(sl, k):
                for _ in range(sl, steps, slots):
                    call(sl, k)
            ths = [threading.Thread(target=worker, args=(sl, k))
                   for sl in range(slots) for k in range(len(LEAVES))]
            for t in ths:
                t.start()
            for t in ths:
                t.join()
        if errors:
            sl, k, st = errors[0]
            slot_ctxs[sl][k]._check(st)

    run(max(args.warmup, 3) * slots)
    torch.cuda.synchronize()
    steps = max(args.steps, 3 * slots)
    all_streams = {s for ss in slot_streams for s in ss}
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for s in all_streams:
        if s is not stream:
            s.wait_event(start)
    run(steps)
    for s in all_streams:
        if s is not stream:
            done = torch.cuda.Event()
            done.record(s)
            stream.wait_event(done)
    end.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(end) / steps
    for cs in slot_ctxs[1:]:
        for c in cs:
            c.close()
    for c, st in zip(ctxs, leaf_streams):
        c.set_stream(st.cuda_stream)
    h2d = len(LEAVES) * n * 16
    d2h = sum(v * (16 + 16) for v in voxels)
    return dict(value=N_POINTS / (ms / 1e3) / 1e6, unit=UNIT, ms_per_step=ms,
                h2d_bytes_per_step=h2d, d2h_bytes_per_step=d2h, steps_in_flight=slots,
                api=("srcu_voxel_normals (include/srcuda.h), "
                     + ("pinned" if pinned else "pageable (plain numpy)") + " host buffers, one "
                     "call per leaf and step" + ("" if serial else
                                                 f", {slots} steps in flight from "
                                                 f"{slots * len(LEAVES)} host threads")))


def main():
    args = parse()
    if args.only_batched:
        import torch
        torch.cuda.set_device(0)
        dev = torch.device("cuda", 0)
        stream = torch.cuda.Stream(dev)
        torch.cuda.set_stream(stream)
        print(json.dumps(run_batched(args, torch, dev, stream)), flush=True)
        return
    if args.only_ransac:
        import torch
        torch.cuda.set_device(0)
        dev = torch.device("cuda", 0)
        stream = torch.cuda.Stream(dev)
        torch.cuda.set_stream(stream)
        args.no_cpu_baseline = True
        print(json.dumps(run_ransac(args, torch, dev, stream, workload_cloud())), flush=True)
        return
    if args.only_las:
        import torch
        torch.cuda.set_device(0)
        dev = torch.device("cuda", 0)
        stream = torch.cuda.Stream(dev)
        torch.cuda.set_stream(stream)
        args.no_cpu_baseline = True
        print(json.dumps(run_las_stream(args, torch, dev, stream, workload_cloud())), flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
