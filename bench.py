#!/usr/bin/env python
"""Benchmark of the plain LBVH build on B200: Mprims/s and fraction of the HBM roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload clustered16M|sphere2M|uniform64K]

One step = one complete build (scene box and centroids, Morton keys, the three-pass stable radix
sort, one pass that emits the radix tree, gathers and rearranges the triangles and refits the
boxes, and the pass over the nodes that straddle its blocks) of the workload's triangle soup.  Default workload: the 16,777,216-triangle
Gaussian-mixture scene (seeded synthetic data; the reference publishes no scene set).  The
805 MB input soup is larger than the 126 MB L2, so steps run back to back without a flush.

Prints one JSON line (rank 0).  Fields beyond the base contract:
  roofline      dominant kernel's algorithmic bytes / its CUDA-event duration vs measured HBM
  stage_ms      per-stage device times (CUDA events on the build stream, profiled steps)
  cpu_baseline  the CPU restatement of the reference build timed on this host's cores
  e2e           through the public C ABI from pinned host memory: H2D of the soup (in chunks,
                each chunk's first pass behind the copy of the next), the build, D2H of the root
                node record, every step; also with host bounds, and the bare upload for scale
  batched       the 4096-mesh batch (log-uniform 64..262,144 triangles per mesh) built by one
                lvbh_build_batched call vs the plain builder called once per mesh, identical trees
  served        the build server under Poisson arrivals, 100,000 requests per rate (sizes
                log-uniform in 1,024..4,194,304, each request its own window of a seeded clustered
                soup; device-resident inputs at 2000 and 5000 req/s, pinned host inputs uploaded
                inside the latency at 2000 req/s): p50/p99/p99.9 latency, batch sizes and
                builds/s beside the plain per-request builder on the same trace (1 GPU only)
  trace         closest-hit traversal of 4,194,304 rays through the built 2M-triangle sphere
  obj           OBJ ingest: the sphere's 80 MB OBJ text -> soup + bounds on the GPU, and end to
                end through parse + build from pinned host text, beside the oracle's parse
  pt            path-trace bounces: 1920 x 1080 pixels, one bounce each per step, on the sphere
  mesh          the indexed leaf format (no 48-byte triangle copies) beside the soup build of
                the same indexed mesh, and traversal through both layouts
Under torchrun (N > 1) each rank builds its own replica (the build has no shardable exchange).

    python bench.py --workload batch | served | trace | obj | pt | mesh     one part alone
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "webgpu-lvbh-demo_b200")
for _p in (REPO, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "LBVH build Mprims/s"
UNIT = "Mprims/s"

# Algorithmic HBM bytes per triangle of each stage (fixed traffic model, 340 B in all): bounds
# read 48; Morton read 48 + key 4; sort 48 (3 LSD passes of 30-bit keys: histogram read 4,
# pass 1 read 4 write 8, passes 2-3 read 8 write 8); leaf gather perm 4 + gather 48 + write 48
# and tree keys 4 + parents 8 + child links 8 + node words 56 + parent reads 8 + flag atomics 8,
# both done by the one tree-pass kernel (the gather stage is fused into it).  The
# straddling-node pass completes part of the same tree and has no bytes of its own.  The model
# is fixed; the build moves less in its first two stages (box and centroids: read 48, write 12;
# keys from the centroids: read 12, write 4 - 76 bytes where the model counts 100).
MODEL_BYTES = {"bounds": 48, "morton": 52, "sort": 48, "gather": 0, "tree": 192, "top": 0}
KERNELS = {"bounds": ("k_bounds_cen", 1), "morton": ("k_morton_cen", 1), "sort": ("k_scatter", 3),
           "gather": (None, 0), "tree": ("k_tree_climb", 1), "top": ("k_top_group", 1)}
# box and centroids, Morton keys (+ the first pass's tile histograms), 3 sort passes x (chunk
# scan, scatter) and 2 tile-histogram passes, tree, straddling pass (group level, then global)
LAUNCHES_PER_BUILD = 12
MODEL_TOTAL = sum(MODEL_BYTES.values())  # 340 B per triangle


def load_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_scenes():
    """lvbh/scenes.py (pure numpy) loaded by its path, so that the reference arm does not import
    the lvbh package, whose __init__ loads the CUDA library."""
    import importlib.util
    mod = sys.modules.get("lvbh_scenes_standalone")
    if mod is None:
        spec = importlib.util.spec_from_file_location("lvbh_scenes_standalone",
                                                      os.path.join(PKG, "lvbh", "scenes.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[spec.name] = mod
        spec.loader.exec_module(mod)
    return mod


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def make_workload(name: str):
    scenes = load_scenes()
    if name == "clustered16M":
        return scenes.clustered_soup(1 << 24, seed=2), "clustered_soup_16M"
    if name == "clustered4M":  # the same distribution at 2^22 triangles (profiling captures)
        return scenes.clustered_soup(1 << 22, seed=2), "clustered_soup_4M"
    if name == "sphere2M":
        return scenes.sphere_mesh(1024, seed=1), "sphere_mesh_2M"
    if name == "uniform64K":
        return scenes.uniform_soup(65_536, seed=0), "uniform_soup_64K"
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.ident = None
        try:
            import torch
            self.ident = "GPU-" + str(torch.cuda.get_device_properties(index).uuid)
        except Exception:
            pass
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            ident = ["--id=" + self.ident] if self.ident else []
            self.proc = subprocess.Popen(["nvidia-smi", *ident, f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def wait_ready(self, timeout=5.0):
        t0 = time.perf_counter()
        while self.proc and not self.lines and time.perf_counter() - t0 < timeout:
            time.sleep(0.05)

    def count(self, t0, t1):
        return sum(1 for t, _ in self.lines if t0 <= t <= t1)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, t0=None, t1=None):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ts, ln in self.lines:
            if t0 is not None and not (t0 <= ts <= t1):
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0,
                    "raw": [ln for _, ln in self.lines[:3]]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    """Largest value of x over all ranks (the slowest rank's time)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(tri, bounds=None):
    """The oracle (CPU restatement of the reference build) on all host cores."""
    import oracle
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    oracle.build(tri, bounds, threads=cores)
    dt = time.perf_counter() - t0
    return {"value": tri.shape[0] / dt / 1e6, "unit": UNIT, "cores": cores, "kind": "port",
            "cpu_model": cpu_model(),
            "sample": f"one full build of the {tri.shape[0]:,}-triangle workload "
                      f"({dt:.2f} s wall, OpenMP over {cores} threads)"}


def cpu_baseline_table(big=None, big_all_cores_s=None):
    """The CPU restatement on one thread and on all host cores for the three plain-build
    workloads (65,536 uniform, the 2,097,152-triangle sphere, the 16,777,216-triangle clustered
    scene): one build each, Mprims/s.  `big`: the clustered soup when already generated,
    `big_all_cores_s`: its all-core time when already measured."""
    import oracle
    scenes = load_scenes()
    cores = os.cpu_count() or 1
    rows = []
    for wname, gen in (("uniform_soup_64K", lambda: scenes.uniform_soup(65_536, seed=0)),
                       ("sphere_mesh_2M", lambda: scenes.sphere_mesh(1024, seed=1)),
                       ("clustered_soup_16M", lambda: big if big is not None else scenes.clustered_soup(1 << 24, seed=2))):
        tri = gen()
        for threads in (1, cores):
            if wname == "clustered_soup_16M" and threads == cores and big_all_cores_s:
                dt = big_all_cores_s
            else:
                t0 = time.perf_counter()
                oracle.build(tri, None, threads=threads)
                dt = time.perf_counter() - t0
            rows.append({"workload": wname, "num_tris": int(tri.shape[0]), "threads": threads,
                         "s": round(dt, 4), "mprims_per_s": tri.shape[0] / dt / 1e6})
    return {"cpu_model": cpu_model(), "cores": cores, "kind": "port", "rows": rows}


def run_reference(args, world, rank):
    """--impl reference: the CPU restatement of the reference's build (the oracle) on all host
    threads, each step one full build of the workload.  The scene generator is loaded without
    the lvbh package, so no CUDA library of this project is loaded by this arm."""
    if rank != 0:
        return
    import oracle
    tri, wname = make_workload(args.workload)
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle.build(tri, None, threads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.build(tri, None, threads=cores)
    dt = (time.perf_counter() - t0) / args.steps
    v = tri.shape[0] / dt / 1e6
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/u32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": wname, "num_tris": int(tri.shape[0]), "parallelism": "replicas",
                       "bounds": "reduced over all vertices"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "cpu_model": cpu_model(),
                             "sample": f"one full build of the {tri.shape[0]:,}-triangle workload per step"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's WGSL build needs browser WebGPU (unavailable on this box); "
                    "this arm times its C++ restatement, which produces the same output"}
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    import lvbh
    from lvbh import empty_outputs

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    tri, wname = make_workload(args.workload)
    n = tri.shape[0]
    builder = lvbh.BVHBuilder(local, reserve_tris=n)
    stream = torch.cuda.Stream(dev)
    dtri = torch.from_numpy(tri).to(dev)
    outs = empty_outputs(n, dev)
    peak, peak_kind = load_peaks()

    def step(profile=False, sync=False):
        return builder.build_soup(dtri, None, outputs=outs, stream=stream, sync=sync, profile=profile)

    clocks = ClockSampler(local).__enter__()
    clocks.wait_ready()
    # warm-up (graph capture happens on the first call)
    for _ in range(args.warmup):
        step(sync=True)
    torch.cuda.synchronize(dev)

    # timed region: K graph-replayed builds back to back on `stream`
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize(dev)
    h0 = time.perf_counter()
    ev0.record(stream)
    for _ in range(args.steps):
        step(sync=False)
    ev1.record(stream)
    builder.sync()
    torch.cuda.synchronize(dev)
    h1 = time.perf_counter()
    # The sampler ticks every 200 ms; when the timed region was shorter than a few ticks, the
    # same builds keep running (untimed) until three samples are in, and those are reported.
    h2 = h1
    while clocks.count(h0, h2) < 3 and h2 - h1 < 3.0:
        for _ in range(20):
            step(sync=False)
        builder.sync()
        h2 = time.perf_counter()
    clock_summary = clocks.summary(h0, h2)
    clock_summary["window_s"] = round(h2 - h0, 3)
    clock_summary["timed_region_s"] = round(h1 - h0, 3)
    clocks.__exit__()
    barrier(world)
    ms = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(ms, world)
    value = world * n / (ms * 1e-3) / 1e6

    # per-stage CUDA events on the build stream, K profiled builds
    stages = {k: [] for k in lvbh.STAGE_NAMES}
    for _ in range(args.steps):
        res = step(profile=True, sync=True)
        for k, v in res.stage_ms.items():
            stages[k].append(v)
    stage_ms = {k: statistics.mean(v) for k, v in stages.items() if k != "upload"}
    # the dominant kernel: the longest single launch with bytes of its own
    dom = max((k for k in MODEL_BYTES if MODEL_BYTES[k]), key=lambda k: stage_ms[k] / KERNELS[k][1])
    kname, launches = KERNELS[dom]
    launch_ms = stage_ms[dom] / launches
    dom_bytes = MODEL_BYTES[dom] * n / launches
    achieved = dom_bytes / (launch_ms * 1e-3) / 1e9
    traffic = load_traffic(kname, n)
    roofline = {"bound": "hbm", "kernel": kname, "launch_ms": launch_ms,
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "traffic": traffic,
                "algorithmic_bytes": dom_bytes,
                "whole_build": {"model_bytes_per_tri": MODEL_TOTAL,
                                "achieved_gbs": MODEL_TOTAL * n / (ms * 1e-3) / 1e9,
                                "frac_of_measured": MODEL_TOTAL * n / (ms * 1e-3) / 1e9 / peak,
                                "frac_of_8tbs": MODEL_TOTAL * n / (ms * 1e-3) / 1e9 / 8000.0}}

    # end to end through the public API from pinned host memory (the library uploads a large
    # soup in chunks and runs each chunk's first pass behind the copy of the next): without
    # host bounds (the box reduced on the device, the headline) and with them (MODEL_BOUNDS
    # given, as the reference's caller always does)
    htri = torch.from_numpy(tri).pin_memory()
    hroot = torch.empty(16, dtype=torch.int32).pin_memory()
    v = tri.reshape(-1, 3, 4)[:, :, :3]
    host_box = np.concatenate([v.min(axis=(0, 1)), v.max(axis=(0, 1))]).astype(np.float32)

    def e2e_run(bounds):
        ms = []
        for i in range(args.warmup + args.steps):
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            builder.build_soup(htri.numpy(), bounds, outputs=outs, stream=stream, sync=True)
            with torch.cuda.stream(stream):
                hroot.copy_(outs["nodes"][0], non_blocking=True)
            e1.record(stream)
            e1.synchronize()
            if i >= args.warmup:
                ms.append(e0.elapsed_time(e1))
        return max_over_ranks(statistics.mean(ms), world)

    e2e = e2e_run(None)
    e2e_hb = e2e_run(host_box)
    # the pure upload of the same bytes, for scale
    dst = torch.empty_like(dtri)
    up_ms = []
    for i in range(args.warmup + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            dst.copy_(htri.view(dst.shape), non_blocking=True)
            e1.record(stream)
        e1.synchronize()
        if i >= args.warmup:
            up_ms.append(e0.elapsed_time(e1))
    del dst
    up = max_over_ranks(statistics.mean(up_ms), world)
    e2e_line = {"value": world * n / (e2e * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": e2e,
                "h2d_bytes_per_step": 48 * n, "d2h_bytes_per_step": 64,
                "bounds": "reduced on the device",
                "host_bounds": {"value": world * n / (e2e_hb * 1e-3) / 1e6, "unit": UNIT,
                                "ms_per_step": e2e_hb, "h2d_bytes_per_step": 48 * n,
                                "d2h_bytes_per_step": 64},
                "upload_only_ms": up, "upload_gbs": 48 * n / (up * 1e-3) / 1e9}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(tri)
        if not args.no_cpu_table:
            cpu["table"] = cpu_baseline_table(big=tri, big_all_cores_s=n / (cpu["value"] * 1e6))

    builder.close()
    del dtri, outs, htri
    torch.cuda.empty_cache()
    batched = served = obj = trace = None
    if not args.no_batched:
        batched = run_batched(args, world, rank, local)
        torch.cuda.empty_cache()
    if not args.no_served and world == 1:
        served = run_served(args, world, rank, local)
        torch.cuda.empty_cache()
    if not args.no_trace:
        trace = run_trace(args, world, rank, local)
        torch.cuda.empty_cache()
    if not args.no_obj:
        obj = run_obj(args, world, rank, local)
        torch.cuda.empty_cache()
    pt = mesh = None
    if not args.no_pt:
        pt = run_pt(args, world, rank, local)
        torch.cuda.empty_cache()
    if not args.no_mesh:
        mesh = run_mesh(args, world, rank, local)
    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32/u32", "data": "synthetic",
            "config": {"workload": wname, "num_tris": n, "parallelism": "replicas" if world > 1 else "single",
                       "bounds": "reduced on the device over all vertices",
                       "l2": "input soup 805 MB > 126 MB L2; no flush", "graph": True},
            "gpu_launches": LAUNCHES_PER_BUILD * args.steps,
            "roofline": roofline, "stage_ms": stage_ms, "cpu_baseline": cpu, "e2e": e2e_line,
            "clocks": clock_summary, "batched": batched, "served": served, "trace": trace, "obj": obj,
            "pt": pt, "mesh": mesh}
    line["summary"] = summarize(line)  # last, so that a tail of the output still holds it
    print(json.dumps(line), flush=True)


def summarize(line):
    """The headline figures of every part, compact, for the end of the JSON line."""
    r = lambda x, d=3: None if x is None else round(float(x), d)  # noqa: E731
    out = {"build_ms": r(line["ms_per_step"], 4), "stage_ms": {k: r(v, 4) for k, v in line["stage_ms"].items()},
           "roofline_frac": r(line["roofline"]["frac"]),
           "whole_build_frac": r(line["roofline"]["whole_build"]["frac_of_measured"]),
           "e2e_mprims_per_s": r(line["e2e"]["value"], 1),
           "e2e_ms": r(line["e2e"]["ms_per_step"], 3),
           "e2e_host_bounds_ms": r(line["e2e"]["host_bounds"]["ms_per_step"], 3),
           "upload_only_ms": r(line["e2e"]["upload_only_ms"], 3)}
    b = line.get("batched")
    if b:
        out["batched"] = {"ms_per_batch": r(b["ms_per_batch"]), "builds_per_s": r(b["builds_per_s"], 0),
                          "speedup_vs_per_mesh": r(b["speedup_vs_per_mesh"], 2),
                          "identical_trees": b["identical_trees"], "num_tris": b["num_tris"]}
    sv = line.get("served")
    if sv:
        out["served"] = [{"mode": x["mode"], "rate": x["rate"], "requests": x["requests"],
                          "p50_p99_p999_ms": [r(x["latency_ms"][k]) for k in ("p50", "p99", "p999")],
                          "mean_batch_reqs": r(x["mean_batch_reqs"], 2), "builds_per_s": r(x["builds_per_s"], 1),
                          "plain_p50_p99_ms": [r(x["plain"]["latency_ms"][k]) for k in ("p50", "p99")]}
                         for x in sv["rates"]]
    for k, f in (("trace", "mrays_per_s"), ("pt", "mpix_bounces_per_s"), ("obj", "parse_ms")):
        if line.get(k):
            out[k + "_" + f] = r(line[k][f], 1 if f != "parse_ms" else 4)
    if line.get("mesh"):
        out["mesh_build_ms"] = r(line["mesh"]["build_mesh_ms"], 4)
    return out


def run_batched(args, world, rank, local, clocks=None):
    """The 4096-mesh batch: one lvbh_build_batched call vs the plain builder called once per
    mesh (lvbh_build_soup through the C ABI, argument structs prepared outside the timed
    region, no host wait between meshes).  Returns a dict for the JSON line."""
    import ctypes

    import numpy as np
    import torch

    import lvbh
    from lvbh import _native, empty_outputs, scenes

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    count = args.batch_meshes
    t_gen = time.perf_counter()
    tri, offs = scenes.mesh_batch(count=count, seed=3)
    t_gen = time.perf_counter() - t_gen
    n = int(offs[-1])
    sizes = np.diff(offs)
    builder = lvbh.BVHBuilder(local, reserve_tris=int(sizes.max()))
    stream = torch.cuda.Stream(dev)
    dtri = torch.from_numpy(tri).to(dev)
    outs = empty_outputs(n, dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def batched(profile=False, sync=False, graph=True, o=outs):
        return builder.build_batched(dtri, offs, outputs=o, stream=stream, sync=sync,
                                     profile=profile, graph=graph, autotune=True)

    for _ in range(args.warmup):  # the first build of this size histogram tunes
        batched(sync=True)
    tuned = builder.tunables()
    torch.cuda.synchronize(dev)
    barrier(world)
    ev0.record(stream)
    for _ in range(args.steps):
        batched()
    ev1.record(stream)
    builder.sync()
    torch.cuda.synchronize(dev)
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world)
    stages = {k: [] for k in lvbh.STAGE_NAMES}
    for _ in range(min(args.steps, 5)):
        r = batched(profile=True, sync=True)
        for k, v in r.stage_ms.items():
            stages[k].append(v)
    stage_ms = {k: statistics.mean(v) for k, v in stages.items() if k != "upload"}

    # the plain builder once per mesh, into a second set of outputs
    outs_b = empty_outputs(n, dev)
    L, ctx = _native.lib, builder.ctx
    sp = ctypes.c_void_p(stream.cuda_stream)
    calls = []
    for i in range(count):
        a, b = int(offs[i]), int(offs[i + 1])
        r = _native.Result()
        r.num_tris = r.num_nodes = b - a
        if b > a:
            r.nodes = outs_b["nodes"][a].data_ptr()
            r.tris = outs_b["tris"][a].data_ptr()
            r.parents = outs_b["parents"][2 * a].data_ptr()
            r.leaf_index = outs_b["leaf_index"][a].data_ptr()
            r.morton = outs_b["morton"][a].data_ptr()
        calls.append((ctypes.c_void_p(dtri[a].data_ptr() if b > a else 0), b - a, r))

    def per_mesh(graph):
        flags = _native.OUT_CALLER | _native.ASYNC | (0 if graph else _native.NO_GRAPH)
        for p, m, r in calls:
            rc = L.lvbh_build_soup(ctx, p, m, None, flags, ctypes.byref(r), sp)
            if rc:
                _native.check(ctx, rc)
        _native.check(ctx, L.lvbh_sync(ctx))

    loop = {}
    for graph in (False, True):
        per_mesh(graph)  # warm-up
        torch.cuda.synchronize(dev)
        reps = 2
        ev0.record(stream)
        for _ in range(reps):
            per_mesh(graph)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        loop["graph" if graph else "no_graph"] = ev0.elapsed_time(ev1) / reps
    base_ms = max_over_ranks(min(loop.values()), world)
    identical = all(torch.equal(outs[k], outs_b[k]) for k in outs)

    # end to end: pinned host soup in, every mesh's root record out, each step
    htri = torch.from_numpy(tri).pin_memory()
    roots = torch.empty((count, 16), dtype=torch.int32).pin_memory()
    root_idx = torch.from_numpy(offs[:-1][sizes > 0]).to(dev)
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        builder.build_batched(htri.numpy(), offs, outputs=outs, stream=stream, sync=True)
        with torch.cuda.stream(stream):
            roots[: root_idx.numel()].copy_(outs["nodes"].index_select(0, root_idx), non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        if i >= args.warmup:
            e2e_ms.append(e0.elapsed_time(e1))
    e2e = max_over_ranks(statistics.mean(e2e_ms), world)
    builder.close()
    return {"workload": f"mesh_batch_{count}", "meshes": count, "num_tris": n,
            "mesh_tris": {"min": int(sizes.min()), "max": int(sizes.max()), "mean": float(sizes.mean())},
            "ms_per_batch": ms, "builds_per_s": world * count / (ms * 1e-3),
            "mprims_per_s": world * n / (ms * 1e-3) / 1e6,
            "per_mesh_loop_ms": loop, "per_mesh_builds_per_s": world * count / (base_ms * 1e-3),
            "speedup_vs_per_mesh": base_ms / ms, "identical_trees": bool(identical),
            "stage_ms": stage_ms, "kernels_per_batch": 8 if tuned["digit_bits"] == 10 else 9,
            "graph_nodes_per_batch": 11 if tuned["digit_bits"] == 10 else 12,
            "tunables": {"chosen": {k: tuned[k] for k in ("digit_bits", "tree_block")},
                         "candidates_ms": dict(zip(["10-bit/256", "10-bit/128", "8-bit/256", "8-bit/128"],
                                                   tuned["candidates_ms"]))},
            "e2e": {"value": world * n / (e2e * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": e2e,
                    "h2d_bytes_per_step": 48 * n, "d2h_bytes_per_step": 64 * int(root_idx.numel())},
            "generate_s": round(t_gen, 1)}


def run_trace(args, world, rank, local):
    """Closest-hit traversal throughput (the consumer of the BVH layout, pathtracer.js:495-628):
    the 2,097,152-triangle displaced sphere built once, then `args.rays` rays per step (origins
    on a radius-3 sphere, directions toward [-1, 1]^3) traced through lvbh_trace, CUDA events
    around each call; the CPU restatement traces a sample on all host cores."""
    import ctypes

    import numpy as np
    import torch

    import lvbh
    from lvbh import _native, scenes

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    tri = scenes.sphere_mesh(1024, seed=1)
    builder = lvbh.BVHBuilder(local)
    res = builder.build_soup(torch.from_numpy(tri).to(dev))
    rays = scenes.sphere_rays(args.rays, seed=11)
    drays = torch.from_numpy(rays).to(dev)
    n = tri.shape[0]
    prim = torch.empty(args.rays, dtype=torch.int32, device=dev)
    t = torch.empty(args.rays, dtype=torch.float32, device=dev)
    st = torch.empty(args.rays, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    ptrs = [ctypes.c_void_p(x.data_ptr()) for x in (res.nodes, res.tris, drays, prim, t, st)]

    def step():
        _native.check(builder.ctx, _native.lib.lvbh_trace(builder.ctx, ptrs[0], ptrs[1], n, ptrs[2],
                                                          args.rays, ptrs[3], ptrs[4], ptrs[5],
                                                          ctypes.c_void_p(stream.cuda_stream)))

    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = max_over_ranks(statistics.median(times), world)
    hits = int((prim >= 0).sum().item())
    out = {"workload": "sphere_mesh_2M_trace", "rays": args.rays, "ms_per_step": ms,
           "mrays_per_s": world * args.rays / (ms * 1e-3) / 1e6, "hit_fraction": hits / args.rays,
           "max_stack": int(st.max().item())}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        ref = res.to_numpy()
        sample = rays[: min(args.rays, 1 << 18)]
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        oracle.trace(ref["nodes"], ref["tris"], sample, threads=cores)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": sample.shape[0] / dt / 1e6, "unit": "Mrays/s", "cores": cores,
                               "kind": "port", "sample": f"{sample.shape[0]:,} rays of the same set"}
    builder.close()
    return out


def run_obj(args, world, rank, local):
    """OBJ ingest (parseObj, parse-obj.js:3-88, the step main.js:72-73 runs before each build):
    the 2,097,152-triangle displaced sphere written as an exporter writes it (1,050,625 `v`
    lines with six decimals, 2,097,152 `f` lines; 80 MB) and parsed by lvbh_parse_obj.
    Device-resident text per step, CUDA events around the call (which includes its host
    round trips); end to end from pinned host text through parse, build and the root record
    back on the host; the oracle's single-threaded parse of the same text as the CPU baseline
    (the reference's parser is single-threaded JavaScript)."""
    import ctypes

    import numpy as np
    import torch

    import lvbh
    from lvbh import _native, empty_outputs, scenes

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    xyz, idx = scenes.sphere_mesh(args.obj_quads, seed=1, indexed=True)
    text = scenes.obj_text(xyz, idx)
    nbytes = len(text)
    dtext = torch.frombuffer(bytearray(text), dtype=torch.uint8).to(dev)
    htext = torch.frombuffer(bytearray(text), dtype=torch.uint8).pin_memory()
    ntri = idx.shape[0] + 2
    builder = lvbh.BVHBuilder(local, reserve_tris=ntri)
    stream = torch.cuda.current_stream(dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    tri = ctypes.c_void_p()
    n = ctypes.c_uint32()
    b6 = (ctypes.c_double * 6)()
    line = ctypes.c_uint64()

    def parse(ptr, flags):
        _native.check(builder.ctx, _native.lib.lvbh_parse_obj(builder.ctx, ptr, nbytes, flags, ctypes.byref(tri),
                                                              ctypes.byref(n), b6, ctypes.byref(line), sptr))

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    dptr = ctypes.c_void_p(dtext.data_ptr())
    for _ in range(args.warmup):
        parse(dptr, 0)
    assert n.value == ntri
    ms = max_over_ranks(statistics.median([timed(lambda: parse(dptr, 0)) for _ in range(args.steps)]), world)

    outs = empty_outputs(ntri, dev)
    hroot = torch.empty(16, dtype=torch.int32).pin_memory()
    hptr = ctypes.c_void_p(htext.data_ptr())

    def obj_to_bvh():
        parse(hptr, _native.INPUT_HOST)
        soup = lvbh._device_floats(tri.value, 12 * n.value, dev)
        bounds32 = np.array(list(b6), dtype=np.float32)
        builder.build_soup(soup, bounds32, outputs=outs, stream=stream, sync=True)
        hroot.copy_(outs["nodes"][0], non_blocking=True)

    for _ in range(args.warmup):
        obj_to_bvh()
    e2e = max_over_ranks(statistics.median([timed(obj_to_bvh) for _ in range(args.steps)]), world)
    peak, peak_kind = load_peaks()
    alg = nbytes + 48 * ntri  # text read once, soup written once
    wname = "sphere_mesh_2M_obj" if args.obj_quads == 1024 else f"sphere_mesh_{2 * args.obj_quads ** 2}_obj"
    out = {"workload": wname, "text_bytes": nbytes, "num_tris": ntri,
           "parse_ms": ms, "parse_gbs": world * nbytes / (ms * 1e-3) / 1e9,
           "parse_mtris_per_s": world * ntri / (ms * 1e-3) / 1e6,
           "roofline": {"bound": "hbm", "scope": "whole parse (text read once + soup written once)",
                        "algorithmic_bytes": alg, "achieved": alg / (ms * 1e-3) / 1e9, "peak": peak,
                        "unit": "GB/s", "frac": alg / (ms * 1e-3) / 1e9 / peak, "peak_kind": peak_kind},
           "e2e": {"what": "pinned host text -> parse -> build -> root record on the host",
                   "ms_per_step": e2e, "value": world * nbytes / (e2e * 1e-3) / 1e6, "unit": "MB/s of OBJ text",
                   "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": 64}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        t0 = time.perf_counter()
        ref_tri, _ = oracle.parse_obj(text)
        dt = time.perf_counter() - t0
        got = lvbh._device_floats(tri.value, 12 * n.value, dev).cpu().numpy().reshape(-1, 12)
        out["same_as_oracle"] = bool(np.array_equal(got.view(np.uint32), ref_tri.view(np.uint32)))
        out["cpu_baseline"] = {"value": nbytes / dt / 1e6, "unit": "MB/s of OBJ text", "cores": 1, "kind": "port",
                               "sample": "the whole 80 MB text, parse only", "ms": dt * 1e3}
    builder.close()
    return out


def run_pt(args, world, rank, local):
    """Path-trace bounces (sample(), pathtracer.js:360-392 -> ptStep :655-713): the built
    2,097,152-triangle displaced sphere under the reference's camera (1.5 x the model's extent
    away, looking at its centre), a 1920 x 1080 image, one lvbh_pt_sample per step (every
    pixel's path one bounce on; four rgba32f state planes ping-ponged in HBM), CUDA events
    around each call; the oracle's bounce of the same frame on all host cores as the CPU
    baseline."""
    import numpy as np
    import torch

    import lvbh
    from lvbh import scenes

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    tri = scenes.sphere_mesh(1024, seed=1)
    builder = lvbh.BVHBuilder(local)
    res = builder.build_soup(torch.from_numpy(tri).to(dev))
    w, h = args.pt_width, args.pt_height
    pos, lat = lvbh.camera([float(x) for x in res.bounds])
    bufs = [torch.zeros((4, h, w, 4), dtype=torch.float32, device=dev) for _ in range(2)]
    stream = torch.cuda.current_stream(dev)
    k = [0]

    def step():
        i = k[0]
        builder.pt_sample(res, None if i == 0 else bufs[i % 2], bufs[(i + 1) % 2], w, h, pos, lat, reset=i == 0)
        k[0] += 1

    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = max_over_ranks(statistics.median(times), world)
    st = bufs[k[0] % 2].cpu().numpy()
    out = {"workload": "sphere_mesh_2M_pt_1080p", "width": w, "height": h, "samples_run": k[0],
           "ms_per_bounce": ms, "mpix_bounces_per_s": world * w * h / (ms * 1e-3) / 1e6,
           "state_bytes_per_bounce": 128 * w * h,
           "state_gbs": world * 128 * w * h / (ms * 1e-3) / 1e9,
           "mean_samples_per_pixel": float(st[2][..., 3].mean())}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        ref = res.to_numpy()
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        oracle.pt_step(ref["nodes"], ref["tris"], None, w, h, pos, lat, True)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": w * h / dt / 1e6, "unit": "Mpixel-bounces/s", "cores": cores,
                               "kind": "port", "sample": f"the first bounce of the {w} x {h} frame"}
    builder.close()
    return out


def run_mesh(args, world, rank, local):
    """The indexed leaf format on the 2,097,152-triangle displaced sphere as an indexed mesh
    (1,050,625 vertex rows of 16 B, 2,097,152 index triples): lvbh_build_mesh (no 48-byte
    triangle is gathered or written; the leaves are index triples) beside lvbh_build_indexed
    (gather to the soup, soup build with the rearranged soup out) on the same mesh, identical
    trees; then closest-hit traversal of args.rays rays through both layouts."""
    import numpy as np
    import torch

    import lvbh
    from lvbh import empty_outputs, scenes

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    xyz, idx = scenes.sphere_mesh(1024, seed=1, indexed=True)
    n = idx.shape[0]
    v4 = np.zeros((xyz.shape[0], 4), np.float32)
    v4[:, :3] = xyz
    dv4 = torch.from_numpy(v4).to(dev)
    dxyz = torch.from_numpy(np.ascontiguousarray(xyz)).to(dev)
    didx = torch.from_numpy(idx.astype(np.uint32).view(np.int32)).to(dev)
    builder = lvbh.BVHBuilder(local, reserve_tris=n)
    stream = torch.cuda.current_stream(dev)
    om, os_ = empty_outputs(n, dev, mesh=True), empty_outputs(n, dev)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        times = []
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        return max_over_ranks(statistics.median(times), world)

    ms_mesh = timed(lambda: builder.build_mesh(dv4, didx, outputs=om, stream=stream))
    ms_soup = timed(lambda: builder.build_indexed(dxyz, didx, outputs=os_, stream=stream))
    rm = builder.build_mesh(dv4, didx, outputs=om, stream=stream)
    rs = builder.build_indexed(dxyz, didx, outputs=os_, stream=stream)
    same = all(torch.equal(om[k], os_[k]) for k in ("nodes", "parents", "leaf_index", "morton"))
    rays = torch.from_numpy(scenes.sphere_rays(args.rays, seed=11)).to(dev)
    tm = timed(lambda: builder.trace_mesh(rm, dv4, rays))
    ts = timed(lambda: builder.trace(rs, rays))
    out = {"workload": "sphere_mesh_2M_indexed", "num_tris": n, "num_verts": int(v4.shape[0]),
           "build_mesh_ms": ms_mesh, "build_indexed_soup_ms": ms_soup,
           "mesh_mprims_per_s": world * n / (ms_mesh * 1e-3) / 1e6,
           "soup_mprims_per_s": world * n / (ms_soup * 1e-3) / 1e6,
           "identical_trees": bool(same),
           "leaf_bytes": {"mesh": 12 * n + 16 * int(v4.shape[0]), "soup": 48 * n},
           "trace_mrays_per_s": {"mesh": world * args.rays / (tm * 1e-3) / 1e6,
                                 "soup": world * args.rays / (ts * 1e-3) / 1e6}}
    builder.close()
    return out


def percentiles(x):
    import numpy as np
    a = np.asarray(x, dtype=np.float64)
    if a.size == 0:
        return {"p50": None, "p99": None, "p999": None}
    return {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)),
            "p999": float(np.percentile(a, 99.9))}


def clustered_pool(n, seed, dev):
    """n triangles of the clustered distribution (64 isotropic Gaussians, means uniform in
    [0,1]^3, sigma log-uniform in [0.002, 0.05], 10 % uniform background, vertex offsets uniform
    in [-0.001, 0.001]^3) drawn on the device with torch from `seed`: the served requests' input
    pool, made in milliseconds instead of seconds of numpy per soup (same recipe as
    scenes.clustered_soup, not the same numbers)."""
    import math
    import torch
    from lvbh import scenes
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    k = 64
    means = torch.rand((k, 3), generator=g, device=dev, dtype=torch.float64)
    sig = torch.exp(torch.rand(k, generator=g, device=dev, dtype=torch.float64)
                    * (math.log(0.05) - math.log(0.002)) + math.log(0.002))
    nb = int(round(n * 0.1))
    nc = n - nb
    which = torch.randint(0, k, (nc,), generator=g, device=dev)
    c = torch.empty((n, 3), dtype=torch.float64, device=dev)
    c[:nc] = means[which] + torch.randn((nc, 3), generator=g, device=dev, dtype=torch.float64) * sig[which, None]
    c[nc:] = torch.rand((nb, 3), generator=g, device=dev, dtype=torch.float64)
    c = c[torch.randperm(n, generator=g, device=dev)].float()
    tri = torch.empty((n, 12), dtype=torch.float32, device=dev)
    for v in range(3):
        off = torch.rand((n, 3), generator=g, device=dev) * 2.0 - 1.0
        tri[:, 4 * v:4 * v + 3] = c + off * 0.001
        tri[:, 4 * v + 3] = float(scenes.PAD)
    return tri


def run_served(args, world, rank, local):
    """Served builds (the served-requests workload): Poisson arrivals at each rate of the plan,
    `count` requests per rate, sizes log-uniform in [1024, 4194304] triangles of the clustered
    distribution, a 96 GB budget.  Request i draws its own soup and window from the trace's
    generator: triangles [o_i, o_i + n_i) of one of `--serve-pool` seeded clustered soups of
    2^22 triangles - an i.i.d. sample of its soup's mixture, since the soups are drawn triangle
    by triangle.  Inputs are either device-resident (the server keeps vertex state on the GPU)
    or pinned host memory, uploaded inside each request's latency.  Latency = submit -> the
    request's batch finished on the GPU (server clock).  Beside it the plain per-request builder
    (lvbh_build_soup, one request at a time in arrival order) serves the first
    `--serve-plain-max` requests of the same trace from the same inputs."""
    import ctypes
    from collections import deque

    import numpy as np
    import torch

    import lvbh
    from lvbh import _native, scenes
    from lvbh.server import Server

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    plan = []
    for item in args.serve_plan.split(","):
        mode, rate, count = item.split(":")
        plan.append((mode, float(rate), int(count)))
    pool_n = 1 << 22
    pool = [clustered_pool(pool_n, 100 + k, dev) for k in range(args.serve_pool)]
    hpool = None
    if any(m == "host" for m, _, _ in plan):
        hpool = [p.cpu().pin_memory().numpy() for p in pool]
    torch.cuda.synchronize(dev)
    srv = Server(local, hbm_budget=96 << 30, slots=3, max_batch_tris=1 << 24, max_batch_reqs=4096)
    plain = lvbh.BVHBuilder(local, reserve_tris=pool_n)
    pstream = torch.cuda.Stream(dev)
    pouts = lvbh.empty_outputs(pool_n, dev)
    out = {"workload": "served_requests", "budget_gb": 96, "slots": 3, "pool_soups": len(pool),
           "pool_tris": pool_n, "rates": []}

    def src(mode, j, o, m):
        return pool[j][o:o + m] if mode == "device" else hpool[j][o:o + m]

    def plain_build(x, m):
        plain.build_soup(x, None, outputs={k: v[: m * (2 if k == "parents" else 1)] for k, v in pouts.items()},
                         stream=pstream, graph=False)

    # warm-up of both paths: every kernel, every slot, the result memory, both input kinds
    wsizes = scenes.request_sizes(args.warmup * 64, seed=99)
    modes = sorted({m for m, _, _ in plan})
    for mode in modes:
        wt = [srv.submit(src(mode, i % len(pool), 0, int(m))) for i, m in enumerate(wsizes)]
        for t in wt:
            srv.wait(t)
            srv.release(t)
        for i, m in enumerate(wsizes[: args.warmup * 8]):
            plain_build(src(mode, i % len(pool), 0, int(m)), int(m))
    torch.cuda.synchronize(dev)
    L, h = _native.lib, srv._h
    rinfo = _native.RequestInfo()
    for mode, rate, count in plan:
        seed = int(rate) * 7 + (1 if mode == "host" else 0)
        sizes = scenes.request_sizes(count, seed=seed)
        rng = np.random.default_rng(seed + 1)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, count))
        which = rng.integers(0, len(pool), count)
        offs = np.floor(rng.random(count) * (pool_n - sizes + 1)).astype(np.int64)
        srcs = [src(mode, int(which[i]), int(offs[i]), int(sizes[i])) for i in range(count)]
        infos = []
        outstanding = deque()

        # one client thread: submits at the arrival times and, between arrivals, polls the
        # oldest outstanding requests and releases the finished ones
        def reap(block=False):
            while outstanding:
                t = outstanding[0]
                rc = (L.lvbh_wait(h, t, -1, None, ctypes.byref(rinfo)) if block
                      else L.lvbh_poll(h, t, None, ctypes.byref(rinfo)))
                if rc == _native.EBUSY:
                    return
                if rc != _native.OK:
                    raise lvbh.LvbhError(rc, "served request failed")
                infos.append((rinfo.latency_ms, rinfo.queued_ms, rinfo.batch_reqs))
                L.lvbh_request_release(h, t)
                outstanding.popleft()

        s0 = srv.stats()
        t0 = time.perf_counter()
        for i in range(count):
            while time.perf_counter() - t0 < arrivals[i]:
                reap()
            outstanding.append(srv.submit(srcs[i]))
            srv._keep.clear()
        while outstanding:
            reap(block=True)
        t_end = time.perf_counter()
        s1 = srv.stats()
        lat = [x[0] for x in infos]
        span = max(t_end - t0, 1e-9)
        nb = max(1, s1["batches"] - s0["batches"])
        served = {"mode": mode, "rate": rate, "requests": count,
                  "inputs": ("device-resident windows of the pool soups" if mode == "device" else
                             "pinned host windows of the pool soups, uploaded inside the latency"),
                  "h2d_bytes": int(48 * sizes.sum()) if mode == "host" else 0,
                  "latency_ms": percentiles(lat), "queued_ms": percentiles([x[1] for x in infos]),
                  "exec_ms": percentiles([x[0] - x[1] for x in infos]),
                  "builds_per_s": count / span, "mprims_per_s": float(sizes.sum()) / span / 1e6,
                  "arrival_span_s": float(arrivals[-1]), "served_span_s": span,
                  "batches": s1["batches"] - s0["batches"], "mean_batch_reqs": count / nb,
                  "batch_reqs_p50_p99": [float(np.percentile([x[2] for x in infos], q)) for q in (50, 99)],
                  "max_batch_seen": s1["max_batch_seen"],
                  "admission_waits": s1["admission_waits"] - s0["admission_waits"],
                  "peak_result_gb": s1["peak_bytes"] / 2**30}
        # the plain per-request builder on the first requests of the same trace
        pc = min(count, args.serve_plain_max)
        plat = []
        t0 = time.perf_counter()
        for i in range(pc):
            while time.perf_counter() - t0 < arrivals[i]:
                pass
            plain_build(srcs[i], int(sizes[i]))
            plat.append((time.perf_counter() - t0 - arrivals[i]) * 1e3)
        pspan = time.perf_counter() - t0
        served["plain"] = {"requests": pc, "latency_ms": percentiles(plat), "builds_per_s": pc / pspan}
        out["rates"].append(served)
        del srcs
    st = srv.stats()
    out["server_stats"] = {k: st[k] for k in ("batches", "completed", "failed", "max_batch_seen")}
    srv.close()
    plain.close()
    del pool, hpool
    torch.cuda.empty_cache()
    return out


def load_traffic(kernel: str, n: int):
    """dram read + write bytes per launch of `kernel` from the committed ncu capture summary
    (profiles/traffic.json: bytes per triangle, scaled to n triangles), or None."""
    try:
        with open(os.path.join(REPO, "profiles", "traffic.json")) as f:
            t = json.load(f)["kernels"][kernel]
        return t["dram_bytes_per_tri"] * n
    except Exception:
        return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="clustered16M")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cpu-table", action="store_true")
    ap.add_argument("--batch-meshes", type=int, default=4096)
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--no-obj", action="store_true")
    ap.add_argument("--no-trace", action="store_true")
    # served requests: mode (device | host input) : rate (req/s) : requests, comma-separated
    ap.add_argument("--serve-plan", default="device:2000:100000,device:5000:100000,host:2000:100000")
    ap.add_argument("--serve-plain-max", type=int, default=10_000)
    ap.add_argument("--serve-pool", type=int, default=16)
    ap.add_argument("--rays", type=int, default=1 << 22)
    ap.add_argument("--obj-quads", type=int, default=1024)  # OBJ workload: sphere grid side
    ap.add_argument("--pt-width", type=int, default=1920)
    ap.add_argument("--pt-height", type=int, default=1080)
    ap.add_argument("--no-pt", action="store_true")
    ap.add_argument("--no-mesh", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.workload == "batch":
            out = run_batched(args, world, rank, local)
            if rank == 0:
                print(json.dumps(out), flush=True)
        elif args.workload == "trace":
            out = run_trace(args, world, rank, local)
            if rank == 0:
                print(json.dumps(out), flush=True)
        elif args.workload == "mesh":
            out = run_mesh(args, world, rank, local)
            if rank == 0:
                print(json.dumps(out), flush=True)
        elif args.workload == "pt":
            out = run_pt(args, world, rank, local)
            if rank == 0:
                print(json.dumps(out), flush=True)
        elif args.workload == "obj":
            out = run_obj(args, world, rank, local)
            if rank == 0:
                print(json.dumps(out), flush=True)
        elif args.workload == "served":
            out = run_served(args, world, rank, local)
            if rank == 0:
                print(json.dumps(out), flush=True)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
