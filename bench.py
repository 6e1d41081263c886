"""Benchmark of the graph-cut hot path: min s-t cut of the tet cell graph.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one full graph_cut (reduced-graph build, multi-discharge
push-relabel with global relabels, final residual BFS, label scatter)
of the benchmark-scale graph: a seeded defective (3,5) torus-knot tube
(~2M faces) over a Kuhn lattice of ~80M tets (the stand-in for the
reference's 12M-point CGAL Delaunay), lambda_fill = 10.

* ``value``: tets/s with every input resident in HBM (C ABI, device
  pointers).  Inputs (2.6 GB of topology) exceed the 126 MB L2, so no
  flush is needed between steps.
* ``e2e``: the same metric through the drop-in ``wtivo_gpupr.graph_cut_fast``
  with host vertices/labels, tets/neighbors copied from pinned host memory
  every step, and the labels read back.
* ``roofline``: the dominant kernel (the persistent solver: one launch per
  cut, CUDA events around it, live in this run) by algorithmic bytes against
  the measured HBM copy bandwidth; its DRAM traffic from an ncu capture; for
  context, the rate at which this GPU serves independent random 4-byte reads.
* ``batch`` / ``serve`` / ``labels`` / ``audit`` / ``raw`` / ``config1`` /
  ``noalloc`` / ``autotune``: the batched cut of 64 uneven graphs, the serving
  loop under Poisson arrivals, the tet-centroid label sampler, the watertight
  audit (of the cut surface and of a closed 5.24M-face sphere), 16 seeds of
  the integer raw graph through gpupr_solve_ell (one checked against the BK
  oracle at full size), the 500k-point proxy Delaunay cut, the
  allocation-free solve beside the allocating one, and the autotuner's choice
  (tuned on another graph of the same generator).
* ``solve_only``: the solver's own device time per cut, beside the
  reference arm's ``solve_seconds`` for the same graph.
* ``cpu_baseline``: the CPU oracle (single-threaded Boykov-Kolmogorov, with
  the reference's graph reduction) on a bounded sample of the same workload.
* ``--impl reference``: the reference's own module (compiled from its
  sources into oracle/_ref) on the same graph: its host graph build on all
  host threads and its CUDA push-relabel on this GPU.

Multi-GPU: a single cut does not shard (every round and BFS level would
need a boundary exchange), so N GPUs run N independent replicas (weak
scaling, no collective on the data path); timing is the max over ranks.

``--only LEG[,LEG...]`` runs the timed cut and only the named extra legs
(e2e, cpu, batch, serve, labels, audit, raw, config1, noalloc, autotune);
with ``--n-tets`` it makes the small cases that ncu captures use.
"""
from __future__ import annotations

import argparse
import contextlib
import gc
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "wtivo-watertightvoxel_b200"
for _p in (str(PKG), str(ROOT)):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "cut solve tets/s (12M-pt-scale graph, ~80M tets, 1 B200)"
WORKLOAD = "torus-knot (3,5) tube, 2% patches dropped, inner shell 0.002, noise 1e-4; Kuhn lattice ~80M tets; lambda_fill=10"

# algorithmic bytes per unit of the solver: a discharge node visit
# reads nbr 16 + res 16 + rev 1 + term 4 + excess 8 + height 4 + 4 neighbour
# heights 16, queue read+write 8 = 73 B; each push adds res+reverse res 8 and
# two excess updates 16 = 24 B; a BFS frontier expansion reads the node's
# neighbour row 16 and in-arc mask 1 + 4 neighbour heights 16 and writes a
# label + queue entry 8 = 41 B; every global relabel streams over each node
# twice: the seed (term 4, height write 4, pair 16 + res 16 read and the
# in-arc mask 1 written) and the active sweep (height 4 + excess 8) = 53 B.
B_VISIT, B_PUSH, B_BFS, B_SWEEP = 73, 24, 41, 53


LEGS = ("e2e", "cpu", "batch", "serve", "labels", "audit", "raw", "config1", "noalloc", "autotune",
        "bottom_up")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n-tets", type=float, default=80e6)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-tets", type=float, default=8e6)
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-graph batch (config 3)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving loop (config 5)")
    ap.add_argument("--serve-seconds", type=float, default=8.0)
    ap.add_argument("--no-labels", action="store_true", help="skip the tet-centroid label leg")
    ap.add_argument("--no-autotune", action="store_true",
                    help="time the built-in grid/relabel rule instead of the autotuned table")
    ap.add_argument("--no-audit", action="store_true", help="skip the watertight audit leg")
    ap.add_argument("--no-raw", action="store_true", help="skip the raw integer graph leg (config 4)")
    ap.add_argument("--raw-seeds", type=int, default=16)
    ap.add_argument("--no-raw-check", action="store_true",
                    help="skip the full-size BK check of the first raw seed")
    ap.add_argument("--only", default="", help="comma list of extra legs to run: " + ",".join(LEGS)
                    + " ('cut' alone: the timed cut and no extra leg)")
    a = ap.parse_args()
    only = {x.strip() for x in a.only.split(",") if x.strip()}
    bad = only - set(LEGS) - {"cut"}
    if bad:
        ap.error(f"unknown legs {sorted(bad)}")
    off = {"e2e": a.no_e2e, "cpu": a.no_cpu_baseline, "batch": a.no_batch, "serve": a.no_serve,
           "labels": a.no_labels, "audit": a.no_audit, "raw": a.no_raw, "autotune": a.no_autotune}
    a.legs = ((only - {"cut"}) if only else set(LEGS)) - {k for k, v in off.items() if v}
    return a


def peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text()), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0}, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"bench_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = [r.split(",") for r in self.path.read_text().strip().splitlines() if r.count(",") >= 8]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], [], set()
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip() == "Active":
                    reasons.add(nm)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job(units_per_rank, ms_local, world):
    """Weak-scaling aggregate: every rank processed units_per_rank in
    ms_local; the job took the slowest rank's time.  Returns (ms, units/s)."""
    ms = max_over_ranks(ms_local, world)
    return ms, world * units_per_rank / (ms * 1e-3)


def bench_config(N, free_n, g, args, world):
    """The workload keys both arms report, so their configs compare equal."""
    return {"workload": WORKLOAD, "n_tets": int(N), "free_nodes": int(free_n),
            "lattice": [int(x) for x in g["shape"]], "lambda_fill": 10.0, "seed": args.seed,
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2_flush": "none needed: inputs (2.6 GB topology) exceed the 126 MB L2"}


def make_graph(n_tets, seed):
    import synth

    return synth.config2(seed, n_tets=int(n_tets))


@contextlib.contextmanager
def no_gc():
    """A timed loop of many host calls without the Python collector's pauses
    (the bench process holds many large objects by the later legs)."""
    gc.collect()
    gc.disable()
    try:
        yield
    finally:
        gc.enable()


@contextlib.contextmanager
def quiet_stdout():
    sys.stdout.flush()
    fd = os.dup(1)
    dn = os.open(os.devnull, os.O_WRONLY)
    os.dup2(dn, 1)
    try:
        yield
    finally:
        sys.stdout.flush()
        os.dup2(fd, 1)
        os.close(fd)
        os.close(dn)


def host_cpu():
    """The host's CPU model and logical CPU count, reported beside CPU timings."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count() or 1}


def cpu_baseline(args, seed):
    """Single-threaded BK oracle on a smaller graph of the same family."""
    from oracle import oracle as orc

    g = make_graph(args.cpu_sample_tets, seed)
    t0 = time.perf_counter()
    orc.graph_cut(g["vertices"], g["tets"], g["neighbors"], g["labels"], 10.0, solver="bk")
    dt = time.perf_counter() - t0
    return {"value": g.n_tets / dt, "unit": "tets/s", "cores": 1, "kind": "port",
            "sample": f"same generator at {g.n_tets} tets (one full cut: reduction + BK + "
                      f"scatter, {dt:.2f} s, oracle/wtivo_oracle.c)", "host": host_cpu()}


def run_ours(args, world, rank, local):
    import torch

    import gpupr_capi
    import wtivo_gpupr

    dev = torch.device("cuda", local)
    tune = None
    if "autotune" in args.legs:
        # the library's autotuner, run on another graph of the same generator
        # and size (seed + 1); its table then serves the timed cuts
        gt = make_graph(args.n_tets, args.seed + 1)
        tt = torch.from_numpy(gt["tets"]).to(dev)
        tn = torch.from_numpy(gt["neighbors"]).to(dev)
        t0 = time.perf_counter()
        tune = gpupr_capi.autotune(gt["vertices"], tt, tn, gt["labels"], 10.0, reps=3)
        tune = {k: (round(v, 3) if isinstance(v, float) else v) for k, v in tune.items()}
        tune["tuning_s"] = round(time.perf_counter() - t0, 2)
        tune["tuned_on"] = f"seed {args.seed + 1} graph of the same generator and size"
        del gt, tt, tn
        torch.cuda.empty_cache()
    g = make_graph(args.n_tets, args.seed)
    N = g.n_tets
    tets = torch.from_numpy(g["tets"]).to(dev)
    nbrs = torch.from_numpy(g["neighbors"]).to(dev)
    V = torch.from_numpy(g["vertices"]).to(dev)
    L = torch.from_numpy(g["labels"]).to(dev)
    out = torch.empty(N, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()

    for _ in range(args.warmup):
        _, st = gpupr_capi.graph_cut(V, tets, nbrs, L, 10.0, out=out)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    with Clocks(local) as clk, no_gc():
        barrier(world)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            _, st = gpupr_capi.graph_cut(V, tets, nbrs, L, 10.0, out=out)
            stats.append(st)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    ms = e0.elapsed_time(e1) / args.steps
    ms_max, value = whole_job(N, ms, world)
    clocks = clk.summary()

    # roofline of the dominant kernel, from the same timed steps
    dis_ms = sum(s["discharge_ms"] for s in stats)
    bfs_ms = sum(s["bfs_ms"] for s in stats)
    visits = sum(s["node_visits"] for s in stats)
    pushes = sum(s["pushes"] for s in stats)
    bfsv = sum(s["bfs_visits"] for s in stats)
    pk, pk_kind = peaks()
    if int(stats[-1]["engine"]) == 2:
        # persistent engine: one cooperative launch holds every round and
        # every BFS level; its duration is the solve's device time
        kern = "k_solve_persistent"
        sweeps = sum(int(s["global_relabels"]) * int(s["free_n"]) for s in stats)
        nbytes = B_VISIT * visits + B_PUSH * pushes + B_BFS * bfsv + B_SWEEP * sweeps
        kms, launches = sum(s["solve_device_ms"] for s in stats), len(stats)
    elif dis_ms >= bfs_ms:
        kern = "k_discharge"
        nbytes = B_VISIT * visits + B_PUSH * pushes
        kms, launches = dis_ms, sum(s["discharge_launches"] for s in stats)
    else:
        kern = "k_bfs_level"
        nbytes = B_BFS * bfsv
        kms, launches = bfs_ms, sum(s["bfs_launches"] for s in stats)
    achieved = nbytes / (kms * 1e-3) / 1e9 if kms > 0 else 0.0
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        try:
            traffic = json.loads(tfile.read_text()).get(kern)
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "kernel": kern, "achieved": round(achieved, 1),
                "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 4),
                "peak_source": pk_kind, "traffic": traffic,
                "algorithmic_bytes_per_step": int(nbytes / args.steps),
                "kernel_ms_per_step": round(kms / args.steps, 3),
                "launches_per_step": int(launches / args.steps),
                "engine": int(stats[-1]["engine"]),
                "phase_ms_per_step": {"solve": round(sum(s["solve_device_ms"] for s in stats) / args.steps, 3),
                                      "build": round(sum(s["build_device_ms"] for s in stats) / args.steps, 3),
                                      "global_relabel": round(bfs_ms / args.steps, 3),
                                      "discharge": round(dis_ms / args.steps, 3)},
                "bfs_steps_by_frontier": {"le_1024": int(stats[-1]["bfs_steps_by_frontier"][0]),
                                          "le_16384": int(stats[-1]["bfs_steps_by_frontier"][1]),
                                          "larger": int(stats[-1]["bfs_steps_by_frontier"][2]),
                                          "ms": [round(x, 3) for x in stats[-1]["bfs_ms_by_frontier"]]},
                "discharge_rounds_by_active": {
                    "le_4096": int(stats[-1]["discharge_rounds_by_active"][0]),
                    "le_131072": int(stats[-1]["discharge_rounds_by_active"][1]),
                    "larger": int(stats[-1]["discharge_rounds_by_active"][2]),
                    "ms": [round(x, 3) for x in stats[-1]["discharge_ms_by_active"]]}}
    if rank == 0:
        rs = random_sector_rate(dev)
        roofline["random_sector_gbs"] = round(rs, 1)
        if isinstance(traffic, (int, float)) and kms > 0:
            dram = traffic / (kms / max(launches, 1) * 1e-3) / 1e9
            roofline["traffic_gbs"] = round(dram, 1)
            roofline["traffic_frac_of_random_sector_rate"] = round(dram / rs, 4)

    # e2e through the drop-in module: pinned host topology, host V/labels
    e2e = None
    if "e2e" in args.legs:
        pt = torch.from_numpy(g["tets"]).pin_memory()
        pn = torch.from_numpy(g["neighbors"]).pin_memory()
        # every input in pinned host memory: numpy views of pinned buffers, which
        # the drop-in copies with direct DMA instead of staging them
        pV = torch.from_numpy(np.ascontiguousarray(g["vertices"])).pin_memory()
        pL = torch.from_numpy(np.ascontiguousarray(g["labels"])).pin_memory()
        hV, hL = pV.numpy(), pL.numpy()
        # double-buffered topology: step k+1's upload runs on a copy stream
        # while step k cuts (every step still copies its own inputs in).
        # Both are non-default streams: work on the legacy default stream
        # would wait for every other stream and serialise the two.
        bufs = [(torch.empty_like(tets), torch.empty_like(nbrs)) for _ in range(2)]
        copy_stream = torch.cuda.Stream(dev)
        cut_stream = torch.cuda.Stream(dev)
        ready = [torch.cuda.Event(), torch.cuda.Event()]
        # freed[j]: recorded on the cut stream once the cut that read buffer j
        # has returned.  Step k's upload waits on that event alone, never on
        # the cut stream as a whole: waiting on the stream while step k-1's
        # cut is in flight would also wait for its solve whenever the solve
        # launch got there first (measured: 114 ms uploads instead of 47).
        freed = [torch.cuda.Event(), torch.cuda.Event()]

        def upload(k):
            """Step k's topology, in 64 MiB pieces with at most one piece in
            the copy queue, so the cut's own host copies are never queued
            behind gigabytes of it (runs on a host thread during the cut)."""
            dt_, dn_ = bufs[k % 2]
            copy_stream.wait_event(freed[k % 2])
            piece = torch.cuda.Event()
            rows = 1 << 22
            with torch.cuda.stream(copy_stream):
                for i in range(0, pt.shape[0], rows):
                    dt_[i:i + rows].copy_(pt[i:i + rows], non_blocking=True)
                    dn_[i:i + rows].copy_(pn[i:i + rows], non_blocking=True)
                    piece.record(copy_stream)
                    piece.synchronize()
                ready[k % 2].record(copy_stream)

        def cut(k):
            cut_stream.wait_event(ready[k % 2])
            dt_, dn_ = bufs[k % 2]
            with torch.cuda.stream(cut_stream):   # the module runs on the current stream
                r_ = wtivo_gpupr.graph_cut_fast(hV, dt_, dn_, hL, 10.0)
            freed[k % 2].record(cut_stream)
            return r_

        def serial_step():
            upload(0)
            return cut(0)

        import threading

        serial_step()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(world)
        a.record(cut_stream)
        for _ in range(args.steps):
            r = serial_step()
        b.record(cut_stream)
        torch.cuda.synchronize()
        serial_ms = a.elapsed_time(b) / args.steps
        barrier(world)
        gc.collect()
        gc.disable()
        a.record(cut_stream)
        upload(0)
        cut_wall, up_wall, join_wall, build_s, solve_s = [], [], [], [], []

        def timed_upload(k, delay):
            # the next step's topology goes up once this step's own inputs
            # are on the device (the previous step's build time), so the two
            # transfers do not share the link
            time.sleep(delay)
            t0 = time.perf_counter()
            upload(k)
            up_wall.append(time.perf_counter() - t0)

        delay = 0.0
        for k in range(args.steps):
            th = None
            if k + 1 < args.steps:
                th = threading.Thread(target=timed_upload, args=(k + 1, delay))
                th.start()
            t0 = time.perf_counter()
            r = cut(k)
            delay = float(r[14])
            cut_wall.append(time.perf_counter() - t0)
            build_s.append(delay)
            solve_s.append(float(r[16]))
            t0 = time.perf_counter()
            if th is not None:
                th.join()
            join_wall.append(time.perf_counter() - t0)
        b.record(cut_stream)
        torch.cuda.synchronize()
        gc.enable()
        ems, evalue = whole_job(N, a.elapsed_time(b) / args.steps, world)
        serial_ms = max_over_ranks(serial_ms, world)
        h2d = pt.numel() * 4 + pn.numel() * 4 + hV.nbytes + hL.nbytes
        e2e = {"value": round(evalue, 1), "unit": "tets/s",
               "ms_per_step": round(ems, 3), "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(N),
               "serial_ms_per_step": round(serial_ms, 3),
               "overlapped_step_host_ms": {
                   "cut_call": round(1e3 * float(np.median(cut_wall)), 2),
                   "next_upload": round(1e3 * float(np.median(up_wall)), 2) if up_wall else None,
                   "wait_for_upload_after_cut": round(1e3 * float(np.median(join_wall)), 2),
                   "dropin_build_s": round(float(r[14]), 4), "dropin_solve_s": round(float(r[16]), 4),
                   "dropin_native_total_s": round(float(r[17]), 4)},
               "per_step_host_ms": {"cut_call": [round(1e3 * x, 2) for x in cut_wall],
                                    "dropin_build": [round(1e3 * x, 2) for x in build_s],
                                    "dropin_solve": [round(1e3 * x, 2) for x in solve_s],
                                    "next_upload": [round(1e3 * x, 2) for x in up_wall]},
               "api": "wtivo_gpupr.graph_cut_fast with host vertices/labels (pinned) and labels "
                      "returned to numpy; each step's tets/neighbors copied from pinned memory, step "
                      "k+1's copy on a second stream while step k solves, started after step k's own "
                      "input copies (serial_ms_per_step: no overlap)"}
        assert np.array_equal(np.asarray(r[0]), out.cpu().numpy()), "e2e labels differ"
        del bufs, pt, pn, pV, pL, r

    legs = args.legs if rank == 0 else set()
    cpu = cpu_baseline(args, args.seed) if "cpu" in legs else None
    batch = run_batch(args, local) if "batch" in legs else None
    serve = run_serve(args) if "serve" in legs else None
    labels = run_labels(args, local, g) if "labels" in legs else None
    audit = run_audit(args, local, g, out, tets, nbrs) if "audit" in legs else None
    bottom_up = run_bottom_up_ab(args, local, (V, tets, nbrs, L)) if "bottom_up" in legs else None
    del tets, nbrs, V, L, out
    torch.cuda.empty_cache()
    raw = run_raw(args, local) if "raw" in legs else None
    config1 = run_config1(args, local) if "config1" in legs else None
    noalloc = run_noalloc(args, local) if "noalloc" in legs else None

    s0 = stats[-1]
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "tets/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_max, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32/int64 (exact integer flow; FP64 capacities)",
        "data": "synthetic (seeded generator; no CGAL/OpenVDB in the image)",
        "config": bench_config(N, int(s0["free_n"]), g, args, world),
        "solve_only": {"ms": round(float(np.median([s["solve_device_ms"] for s in stats])), 3),
                       "what": "median CUDA-event time of the solve phase (push-relabel, every "
                               "global relabel, final BFS) per cut, inputs in HBM"},
        "flow": int(s0["adjusted_flow"]),
        "solve": {"rounds": int(s0["rounds"]), "global_relabels": int(s0["global_relabels"]),
                  "bfs_levels": int(s0["bfs_levels"]), "node_visits": int(s0["node_visits"]),
                  "pushes": int(s0["pushes"]), "solve_device_ms": round(s0["solve_device_ms"], 3),
                  "build_device_ms": round(s0["build_device_ms"], 3),
                  "blocks_per_sm": int(s0["solve_blocks_per_sm"]),
                  "relabel_work_factor": float(s0["relabel_work_factor"]),
                  "free_nodes_per_s": round(s0["free_n"] / (s0["solve_device_ms"] * 1e-3), 1),
                  "one_sweep_floor_ms": round(60.0 * s0["free_n"] / (pk["hbm_gbs"] * 1e9) * 1e3, 4)},
        "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks,
        "batch": batch, "serve": serve, "labels": labels, "audit": audit, "raw": raw,
        "config1": config1, "noalloc": noalloc, "bottom_up": bottom_up, "autotune": tune,
        "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
    }
    return line


def cuda_ms(fn, reps, stream):
    """Mean device time of fn() over reps calls (CUDA events on stream)."""
    import torch

    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def random_sector_rate(dev):
    """Context for the solver's roofline: the rate at which this GPU serves
    independent random 4-byte reads from a 2 GiB array (each moves one 32-byte
    sector), measured with torch's gather (a library kernel) as GB/s of
    sectors.  The solver's accesses are of that kind."""
    import torch

    src = torch.empty(1 << 29, dtype=torch.float32, device=dev)
    idx = torch.randint(0, 1 << 29, (1 << 26,), device=dev)
    for _ in range(2):
        torch.index_select(src, 0, idx)
    ms = cuda_ms(lambda: torch.index_select(src, 0, idx), 5, torch.cuda.current_stream(dev))
    del src, idx
    torch.cuda.empty_cache()
    return (1 << 26) * 32 / (ms * 1e-3) / 1e9


def run_labels(args, local, g):
    """Tet-centroid labels of the benchmark lattice from a narrow-band UDF
    brick grid of the knot mesh at the reference's input resolution (voxel
    1/1536 of the unit query box, band 3 voxels, threshold 1/1536 - 1e-4),
    everything resident in HBM; parity against the oracle on a strided
    sample of the tets; CPU baseline: the oracle on 2M tets, 1 core."""
    import torch

    import gpupr_capi
    import synth
    from oracle import oracle as orc

    dev = torch.device("cuda", local)
    V, T = g["vertices"], g["tets"]
    lo, hi = V.min(0), V.max(0)
    mesh_n = (g["mesh_V"] - lo) / (hi - lo)          # the query box is the unit cube
    R = 1536.0
    t0 = time.perf_counter()
    grid = synth.brick_udf(mesh_n, g["mesh_F"], 1.0 / R, 3.0)
    grid_s = time.perf_counter() - t0
    thr = 1.0 / R - 1e-4
    dgrid = dict(grid)
    dgrid["table"] = torch.from_numpy(np.ascontiguousarray(grid["table"]).reshape(-1)).to(dev)
    dgrid["values"] = torch.from_numpy(np.ascontiguousarray(grid["values"]).reshape(-1)).to(dev)
    dV = torch.from_numpy(V).to(dev)
    dT = torch.from_numpy(T).to(dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        return gpupr_capi.sample_tet_labels(dgrid, dV, dT, lo, hi, 0.0, thr, device_out=True)

    for _ in range(3):
        lab, _ = step()
    ms = cuda_ms(step, 5, stream)
    lab = lab.cpu().numpy()
    idx = np.arange(0, len(T), 97)
    want, _ = orc.sample_tet_labels(grid, V, T[idx], lo, hi, 0.0, thr)
    n_cpu = min(2_000_000, len(T))
    t0 = time.perf_counter()
    orc.sample_tet_labels(grid, V, T[:n_cpu], lo, hi, 0.0, thr)
    cpu_s = time.perf_counter() - t0
    nb = grid["values"].shape[0]
    alg = len(T) * 17 + V.nbytes + nb * 2048 + grid["table"].nbytes   # tets + label, vertices, grid once
    pk, pk_kind = peaks()
    gbs = alg / (ms * 1e-3) / 1e9
    return {"config": "80.3M benchmark tets, knot UDF bricks at 1/1536 (band 3 voxels), inputs in HBM",
            "tets_per_s": round(len(T) / (ms * 1e-3), 1), "ms": round(ms, 3),
            "parity_sample": int(len(idx)), "identical_to_oracle": bool(np.array_equal(lab[idx], want)),
            "bricks": int(nb), "grid_bytes": int(nb * 2048 + grid["table"].nbytes),
            "grid_build_s_host": round(grid_s, 2), "label0_fraction": round(float((lab == 0).mean()), 4),
            "roofline": {"bound": "hbm", "kernel": "k_sample_labels", "achieved": round(gbs, 1),
                         "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": round(gbs / pk["hbm_gbs"], 4),
                         "peak_source": pk_kind, "algorithmic_bytes": int(alg)},
            "cpu_baseline": {"value": round(n_cpu / cpu_s, 1), "unit": "tets/s", "cores": 1, "kind": "port",
                             "sample": f"first {n_cpu} tets, oracle/wtivo_oracle.c"}}


def _cut_capacity(nbr, cap, src, snk, part):
    """Capacity of the cut (S = part 0, T = part 1) in the input raw graph."""
    import torch

    p = part.long()
    valid = nbr >= 0
    pu = torch.where(valid, p[nbr.long().clamp_min(0)], torch.zeros_like(nbr).long())
    nl = (cap.long() * (valid & (p[:, None] == 0) & (pu == 1))).sum()
    s, k = src.long(), snk.long()
    return int((nl + torch.where(p == 0, k, torch.zeros_like(k)).sum()
                + torch.where(p == 1, s, torch.zeros_like(s)).sum()).item())


def run_raw(args, local):
    """Config 4: integer raw graphs (all nodes free, given integer n-links and
    t-links; gpupr_solve_ell), args.raw_seeds seeds (default 16) of the
    2M-point size.  Qhull needs about two minutes per 2M-point seed, so the
    bench uses the lattice stand-in (the Delaunay form is tested at full size
    in the GPU tests): per seed a 125^3-cube jittered Kuhn lattice of the unit
    cube (11.7M nodes), n-links round(1e4 area / mean area), noisy sphere-SDF
    t-links.  Inputs in HBM.  Timed: the seeds one after the other, and all of
    them as one disjoint-union graph; every seed's flow equals the capacity of
    its returned cut, the union equals the separate solves, and the first
    seed's flow and partition are compared with the BK oracle at full size
    (whose single-core time is the CPU baseline)."""
    import torch

    import gpupr_capi
    import synth
    from oracle import oracle as orc

    dev = torch.device("cuda", local)
    t0 = time.perf_counter()
    graphs = [synth.config4(args.seed + k, n_points=2_000_000, use_delaunay=False)
              for k in range(args.raw_seeds)]
    gen_s = time.perf_counter() - t0
    dg = [tuple(torch.from_numpy(np.ascontiguousarray(x)).to(dev)
                for x in (g["nbr"], g["cap"].view(np.int32), g["src"].view(np.int32),
                          g["snk"].view(np.int32))) for g in graphs]
    sizes = [int(d[0].shape[0]) for d in dg]
    total = int(sum(sizes))
    stream = torch.cuda.current_stream(dev)
    for d in dg[:3]:
        gpupr_capi.solve_ell(*d)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with no_gc():
        a.record(stream)
        res, call_ms = [], []
        for d in dg:
            t0 = time.perf_counter()
            res.append(gpupr_capi.solve_ell(*d))
            call_ms.append(1e3 * (time.perf_counter() - t0))
        b.record(stream)
        torch.cuda.synchronize()
    seq_ms = a.elapsed_time(b)
    certified = all(_cut_capacity(*d, r[1]) == r[0] for d, r in zip(dg, res))
    # the seeds as one disjoint-union graph
    off = np.concatenate([[0], np.cumsum(sizes)])
    un = (torch.cat([torch.where(d[0] >= 0, d[0] + int(o), d[0]) for d, o in zip(dg, off[:-1])]),
          *(torch.cat([d[i] for d in dg]) for i in (1, 2, 3)))
    gpupr_capi.solve_ell(*un)
    torch.cuda.synchronize()
    a.record(stream)
    uflow, upart, ust = gpupr_capi.solve_ell(*un)
    b.record(stream)
    torch.cuda.synchronize()
    union_ms = a.elapsed_time(b)
    union_same = uflow == sum(r[0] for r in res) and all(
        torch.equal(upart[int(off[i]):int(off[i + 1])], res[i][1]) for i in range(len(dg)))
    check = None
    if not args.no_raw_check:
        g = graphs[0]
        src, snk = g["src"].astype(np.int64), g["snk"].astype(np.int64)
        term = (src - snk).astype(np.int32)
        t0 = time.perf_counter()
        f_bk, _, _, p_bk = orc.maxflow_bk(g["nbr"], g["cap"], term)
        cpu_s = time.perf_counter() - t0
        check = {"seed": args.seed, "identical_to_oracle": bool(
                     f_bk + int(np.minimum(src, snk).sum()) == res[0][0]
                     and np.array_equal(res[0][1].cpu().numpy(), p_bk)),
                 "oracle_s": round(cpu_s, 2),
                 "source_side_nodes": int(sizes[0] - int(res[0][1].sum().item()))}
        # the workload's n-links (1e4 x area / mean) dwarf the t-links, so its
        # minimum cut takes every source t-link; the same graph with n-links of
        # 30 x area / mean cuts along the sphere: checked against BK as well
        gw = synth.config4(args.seed, n_points=2_000_000, use_delaunay=False, nlink_scale=30.0)
        dw = tuple(torch.from_numpy(np.ascontiguousarray(x)).to(dev)
                   for x in (gw["nbr"], gw["cap"].view(np.int32), gw["src"].view(np.int32),
                             gw["snk"].view(np.int32)))
        fw, pw, stw = gpupr_capi.solve_ell(*dw)
        sw, kw = gw["src"].astype(np.int64), gw["snk"].astype(np.int64)
        fbw, _, _, pbw = orc.maxflow_bk(gw["nbr"], gw["cap"], (sw - kw).astype(np.int32))
        check["weak_nlinks_30"] = {
            "identical_to_oracle": bool(fbw + int(np.minimum(sw, kw).sum()) == fw
                                        and np.array_equal(pw.cpu().numpy(), pbw)),
            "source_side_nodes": int(len(pbw) - int(pbw.sum())), "flow": int(fw),
            "solve_device_ms": round(stw["solve_device_ms"], 3)}
        del dw, gw
        cpu = {"value": round(sizes[0] / cpu_s, 1), "unit": "nodes/s", "cores": 1, "kind": "port",
               "sample": f"seed {args.seed}, {sizes[0]} nodes: BK max flow + partition, "
                         "oracle/wtivo_oracle.c", "host": host_cpu()}
    else:
        cpu = None
    st0 = res[0][2]
    return {"config": f"{len(dg)} seeds of the raw integer graph, each a 125^3-cube Kuhn lattice "
                      "(11.7M nodes; lattice stand-in for the 2M-point Delaunay), integer n-links "
                      "round(1e4 area/mean), noisy sphere-SDF t-links, inputs in HBM",
            "seeds": len(dg), "nodes_per_seed": sizes[0], "nodes": total,
            "flows": [int(r[0]) for r in res], "every_cut_capacity_equals_flow": bool(certified),
            "sequential_ms": round(seq_ms, 3), "nodes_per_s": round(total / (seq_ms * 1e-3), 1),
            "sequential_call_ms": [round(x, 2) for x in call_ms],
            "sequential_solve_device_ms": [round(r[2]["solve_device_ms"], 2) for r in res],
            "union_ms": round(union_ms, 3), "union_nodes_per_s": round(total / (union_ms * 1e-3), 1),
            "union_identical_to_separate": bool(union_same),
            "seed0": {"ms": round(st0["solve_device_ms"], 3), "rounds": int(st0["rounds"]),
                      "global_relabels": int(st0["global_relabels"])},
            "oracle_check": check, "generation_s_host": round(gen_s, 1), "cpu_baseline": cpu}


def run_config1(args, local):
    """Config 1 at its stated size: holed icosphere (r 0.4, subdivision 5, 5%
    of faces deleted), 500k-point proxy at res 256, Qhull Delaunay in Morton
    cell order (~3.2M tets), lambda_fill 10.  Device time of the cut through
    the C ABI with inputs in HBM, and the drop-in graph_cut_fast with host
    vertices and labels; labels and flow compared with the oracle, whose
    single-core time is the CPU baseline."""
    import torch

    import gpupr_capi
    import synth
    import wtivo_gpupr
    from oracle import oracle as orc

    dev = torch.device("cuda", local)
    g = synth.config1(args.seed, n_points=500_000)
    tets, nbrs, V, L = (torch.from_numpy(np.ascontiguousarray(g[k])).to(dev)
                        for k in ("tets", "neighbors", "vertices", "labels"))
    out = torch.empty(g.n_tets, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(3):
        _, st = gpupr_capi.graph_cut(V, tets, nbrs, L, 10.0, out=out)
    ms = cuda_ms(lambda: gpupr_capi.graph_cut(V, tets, nbrs, L, 10.0, out=out), 5, stream)
    walls = []
    for _ in range(5):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = wtivo_gpupr.graph_cut_fast(g["vertices"], tets, nbrs, g["labels"], 10.0)
        walls.append(time.perf_counter() - t0)
    t0 = time.perf_counter()
    lab, ost = orc.graph_cut(g["vertices"], g["tets"], g["neighbors"], g["labels"], 10.0)
    cpu_s = time.perf_counter() - t0
    same = (np.array_equal(out.cpu().numpy(), lab) and np.array_equal(np.asarray(r[0]), lab)
            and st["adjusted_flow"] == ost["adjusted_flow"] == int(r[1]))
    return {"config": "holed icosphere, 500k-point proxy at res 256, Qhull Delaunay (Morton cell "
                      "order), lambda_fill=10",
            "n_tets": g.n_tets, "free_nodes": int(st["free_n"]), "flow": int(st["adjusted_flow"]),
            "ms": round(ms, 3), "tets_per_s": round(g.n_tets / (ms * 1e-3), 1),
            "solve_device_ms": round(st["solve_device_ms"], 3),
            "dropin_host_arrays_ms": round(1e3 * float(np.median(walls)), 3),
            "identical_to_oracle": bool(same),
            "cpu_baseline": {"value": round(g.n_tets / cpu_s, 1), "unit": "tets/s", "cores": 1,
                             "kind": "port", "sample": "the whole graph: reduction + BK + scatter, "
                                                       "oracle/wtivo_oracle.c"}}


def run_bottom_up_ab(args, local, bench_inputs):
    """Direction-optimizing relabels, A/B: median device solve time of the
    benchmark cut and of a 3M-tet holed-torus cut, relabels top-down only and
    with bottom-up steps (switch when the unlabelled candidates number at most
    ratio x the frontier; ratios 1 and 8), 5 alternating cuts per setting;
    every setting's labels compared with the top-down cut's."""
    import torch

    import gpupr_capi
    import synth

    dev = torch.device("cuda", local)
    tg = synth.config3_graph(1, 3_000_000, args.seed)
    torus = tuple(torch.from_numpy(np.ascontiguousarray(tg[k])).to(dev)
                  for k in ("vertices", "tets", "neighbors", "labels"))
    settings = {"top_down": None,
                "bottom_up_r1": gpupr_capi.options(bfs_bottom_up=1, bfs_bottom_up_ratio=1.0),
                "bottom_up_r8": gpupr_capi.options(bfs_bottom_up=1, bfs_bottom_up_ratio=8.0)}
    out = {}
    for name, (V, T, Nb, L) in (("benchmark", bench_inputs), ("torus_3M", torus)):
        lab = torch.empty(int(T.shape[0]), dtype=torch.uint8, device=dev)
        ref = None
        times = {k: [] for k in settings}
        steps = {}
        same = True
        for rep in range(6):
            for k, o in settings.items():
                _, st = gpupr_capi.graph_cut(V, T, Nb, L, 10.0, out=lab, opts=o)
                if rep:
                    times[k].append(st["solve_device_ms"])
                steps[k] = int(st["bottom_up_steps"])
                if ref is None:
                    ref = lab.clone()
                else:
                    same = same and bool(torch.equal(lab, ref))
        out[name] = {"n_tets": int(T.shape[0]), "identical_cuts": same,
                     **{k: {"solve_ms": round(float(np.median(v)), 3), "bottom_up_steps": steps[k]}
                        for k, v in times.items()}}
    return out


def run_noalloc(args, local):
    """The allocation-free solve beside the allocating one on the same reduced
    graph (a holed-torus lattice of 1M tets, under the 1,048,576-node limit of
    the static scratch array): median wall time of 5 alternating calls each,
    the graph's residuals restored before every call; results compared."""
    import torch

    import gpupr_capi
    import synth

    dev = torch.device("cuda", local)
    g = synth.config3_graph(1, 1_000_000, args.seed)
    tets, nbrs = (torch.from_numpy(np.ascontiguousarray(g[k])).to(dev) for k in ("tets", "neighbors"))
    b = gpupr_capi.build_reduced(g["vertices"], tets, nbrs, g["labels"], 10.0)
    n = len(b["nbr"])
    if n > 1 << 20:
        return {"skipped": f"{n} free nodes exceed the static scratch limit"}
    scratch = gpupr_capi.noalloc_prepare()
    nbr = torch.from_numpy(np.ascontiguousarray(b["nbr"])).to(dev)
    res0 = torch.from_numpy(np.ascontiguousarray(b["res"]).view(np.int32)).to(dev)
    term0 = torch.from_numpy(np.ascontiguousarray(b["term"])).to(dev)
    res, term = res0.clone(), term0.clone()
    part = torch.empty(n, dtype=torch.uint8, device=dev)
    t_alloc, t_na = [], []
    for rep in range(6):
        for which in (0, 1):
            res.copy_(res0)
            term.copy_(term0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            if which == 0:
                pa, sa, _ = gpupr_capi.solve_reduced(nbr, res, term)
            else:
                sn = gpupr_capi.solve_reduced_noalloc(nbr, res, term, part)
            torch.cuda.synchronize()
            if rep:
                (t_alloc if which == 0 else t_na).append(time.perf_counter() - t0)
    same = sa["raw_flow"] == sn["raw_flow"] and np.array_equal(part.cpu().numpy(), pa)
    return {"config": "holed-torus Kuhn lattice, 1M tets, reduced graph in HBM",
            "free_nodes": n, "scratch_bytes": scratch,
            "solve_reduced_ms": round(1e3 * float(np.median(t_alloc)), 3),
            "solve_reduced_engine": int(sa["engine"]),
            "noalloc_ms": round(1e3 * float(np.median(t_na)), 3), "noalloc_engine": 1,
            "identical": bool(same)}


def _audit_case(dF, F, dev):
    """Device time of gpupr_edge_audit on device faces, its roofline, and the
    oracle's sort-and-count (1 core) on the same faces."""
    import torch

    import gpupr_capi
    from oracle import oracle as orc

    stream = torch.cuda.current_stream(dev)
    for _ in range(3):
        bad, nbytes = gpupr_capi.edge_audit(dF)
    ms = cuda_ms(lambda: gpupr_capi.edge_audit(dF), 5, stream)
    t0 = time.perf_counter()
    ref = orc.edge_audit(F)
    cpu_s = time.perf_counter() - t0
    nf = len(F)
    slots = nbytes // 8
    # faces 12 B; each of the 3 edge updates reads and writes its 8-byte slot;
    # the table is cleared (8 B a slot) and scanned (8 B a slot)
    alg = nf * 12 + 3 * nf * 16 + slots * 16
    pk, pk_kind = peaks()
    gbs = alg / (ms * 1e-3) / 1e9
    return {"faces": int(nf), "bad_edge_groups": int(bad), "identical_to_oracle": bool(bad == ref),
            "faces_per_s": round(nf / (ms * 1e-3), 1), "ms": round(ms, 3), "table_bytes": int(nbytes),
            "roofline": {"bound": "hbm", "kernel": "k_edge_count + k_edge_bad (+ table clear)",
                         "achieved": round(gbs, 1), "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": round(gbs / pk["hbm_gbs"], 4), "peak_source": pk_kind,
                         "algorithmic_bytes": int(alg)},
            "cpu_baseline": {"value": round(nf / cpu_s, 1), "unit": "faces/s", "cores": 1, "kind": "port",
                             "sample": "all faces, oracle/wtivo_oracle.c (qsort of 3F edge keys)"}}


def run_audit(args, local, g, labels_dev, tets, nbrs):
    """Edge-degree watertight audit: of the benchmark cut's surface (device
    faces; its 631k faces and table fit in L2) and of a closed 5.24M-face
    icosphere (subdivision 9, table larger than L2); CPU baseline: the
    oracle's sort-and-count, 1 core."""
    import torch

    import synth
    import wtivo_gpupr

    dev = torch.device("cuda", local)
    Vs, F = wtivo_gpupr.surface_extraction_topology_cuda(labels_dev.cpu().numpy(), g["vertices"], tets, nbrs)
    out = {"config": "cut surface of the benchmark graph, faces in HBM",
           **_audit_case(torch.from_numpy(np.ascontiguousarray(F)).to(dev), F, dev)}
    _, SF = synth.icosphere(9, 0.4)
    SF = np.ascontiguousarray(SF, np.int32)
    out["sphere"] = {"config": "closed icosphere, subdivision 9, faces in HBM",
                     **_audit_case(torch.from_numpy(SF).to(dev), SF, dev)}
    return out


def run_batch(args, local):
    """Config 3: 64 uneven graphs (tets log-uniform 50k..4M) cut as one batch
    (one segmented solve; graphs retire as they finish) vs the same 64 graphs
    cut one after the other, inputs in HBM, for two seeded batches.  Each batch
    is timed with the built-in batch rule, then the batch autotuner is run on
    the seed+1 batch and both batches are timed again with the table entry of
    their size bucket (free nodes per graph); labels and flows compared with
    the one-by-one cuts."""
    import torch

    import gpupr_capi
    import synth

    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)

    def load(seed):
        sizes = synth.config3_sizes(seed, 64)
        graphs = [synth.config3_graph(i, int(n), seed) for i, n in enumerate(sizes)]
        toff, voff, V, T, Nb, L = gpupr_capi.pack_batch(graphs)
        packed = (toff, voff) + tuple(torch.from_numpy(x).to(dev) for x in (V, T, Nb, L))
        singles = [tuple(torch.from_numpy(np.ascontiguousarray(g[k])).to(dev)
                         for k in ("tets", "neighbors", "vertices", "labels")) for g in graphs]
        return packed, singles

    def time_batch(packed, out, reps=3):
        toff, voff, v, t, nb, l = packed
        gpupr_capi.graph_cut_batch(toff, voff, v, t, nb, l, 10.0, out=out)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with no_gc():
            a.record(stream)
            for _ in range(reps):
                _, items, bst = gpupr_capi.graph_cut_batch(toff, voff, v, t, nb, l, 10.0, out=out)
            b.record(stream)
            torch.cuda.synchronize()
        return a.elapsed_time(b) / reps, items, bst

    old = gpupr_capi.batch_tune_table()
    gpupr_capi.set_batch_tune_table([])
    seeds = {}
    data = {}
    for seed in (args.seed, args.seed + 1):
        packed, singles = load(seed)
        data[seed] = (packed, singles)
        out = torch.empty(int(packed[0][-1]), dtype=torch.uint8, device=dev)
        rule_ms, items, bst = time_batch(packed, out)
        outs = [torch.empty(int(s[0].shape[0]), dtype=torch.uint8, device=dev) for s in singles]
        for (gt, gn, gv, gl), o in zip(singles, outs):
            gpupr_capi.graph_cut(gv, gt, gn, gl, 10.0, out=o)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with no_gc():
            a.record(stream)
            seq = [gpupr_capi.graph_cut(gv, gt, gn, gl, 10.0, out=o)[1]
                   for (gt, gn, gv, gl), o in zip(singles, outs)]
            b.record(stream)
            torch.cuda.synchronize()
        seq_ms = a.elapsed_time(b)
        toff = packed[0]
        ob = out.cpu().numpy()
        same = all(items[k]["adjusted_flow"] == seq[k]["adjusted_flow"] and
                   np.array_equal(ob[int(toff[k]):int(toff[k + 1])], outs[k].cpu().numpy())
                   for k in range(len(singles)))
        seeds[seed] = {"tets": int(toff[-1]), "free_nodes": int(bst["free_n"]), "sequential_ms": round(seq_ms, 3),
                       "rule": {"batch_ms": round(rule_ms, 3), "graphs_retired": int(bst["graphs_retired"]),
                                "global_relabels": int(bst["global_relabels"]),
                                "blocks_per_sm": int(bst["solve_blocks_per_sm"]),
                                "chain_hops": int(bst["chain_hops"])},
                       "identical_to_sequential": bool(same)}
        del outs, out
    # tune on the seed+1 batch; its entry serves the bucket of both batches
    p1 = data[args.seed + 1][0]
    t0 = time.perf_counter()
    entry = gpupr_capi.autotune_batch(*p1[:2], *p1[2:], 10.0, reps=3)
    tune_s = time.perf_counter() - t0
    for seed in seeds:
        packed = data[seed][0]
        out = torch.empty(int(packed[0][-1]), dtype=torch.uint8, device=dev)
        ms, items, bst = time_batch(packed, out)
        r = seeds[seed]
        r["tuned"] = {"batch_ms": round(ms, 3), "bucket": int(int(bst["free_n"] // 64).bit_length() - 1),
                      "blocks_per_sm": int(bst["solve_blocks_per_sm"]),
                      "relabel_work_factor": float(bst["relabel_work_factor"]),
                      "chain_hops": int(bst["chain_hops"]), "chain_max_active": int(bst["chain_max_active"])}
        r["speedup_rule"] = round(r["sequential_ms"] / r["rule"]["batch_ms"], 2)
        r["speedup_tuned"] = round(r["sequential_ms"] / ms, 2)
    table = gpupr_capi.batch_tune_table()
    gpupr_capi.set_batch_tune_table(old)
    s0 = seeds[args.seed]
    best = min(s0["rule"]["batch_ms"], s0["tuned"]["batch_ms"])
    return {"config": "64 graphs, tets log-uniform 50k..4M (holed icosphere / holed torus / "
                      "open rounded box, Kuhn lattices), lambda_fill=10, inputs in HBM",
            "graphs": 64, "tets": s0["tets"], "batch_ms": round(best, 3),
            "sequential_ms": s0["sequential_ms"], "speedup": round(s0["sequential_ms"] / best, 2),
            "batched_cuts_per_s": round(64 / (best * 1e-3), 1),
            "sequential_cuts_per_s": round(64 / (s0["sequential_ms"] * 1e-3), 1),
            "identical_to_sequential": all(v["identical_to_sequential"] for v in seeds.values()),
            "seeds": {str(k): v for k, v in seeds.items()},
            "tuned_on": f"seed {args.seed + 1} batch", "tuning_s": round(tune_s, 2),
            "batch_tune_table": [{k: (round(v, 3) if isinstance(v, float) else v) for k, v in e.items()}
                                 for e in table]}


def run_serve(args):
    """Config 5: Poisson arrivals, tets log-uniform 100k..20M (a pool of 12
    seeded graphs), 160 GiB admission budget, host arrays in and out.  At 20
    req/s (the config's rate) and at 100 req/s (a load where requests queue),
    the same arrival trace goes through the server with its two lanes (small
    requests below 2M tets solve beside large ones, or on the large lane while
    it is idle and the small lane busy), through one lane
    (continuous batching, one solve at a time), and through one lane one
    request at a time (max_batch 1); the 20 req/s trace is also replayed
    against one-at-a-time service times measured alone (the naive FIFO).
    Latency p50/p99 overall and p99 per size bucket."""
    import threading

    import torch

    import gpupr_capi
    import synth

    rng = np.random.default_rng(args.seed + 5)
    pool_sizes = np.exp(rng.uniform(np.log(1e5), np.log(2e7), size=12)).astype(np.int64)
    pool = [synth.config3_graph(i, int(n), args.seed + 5) for i, n in enumerate(pool_sizes)]
    split = 2_000_000

    # service time of each pool graph alone: host topology -> device, cut, labels out
    service = []
    for g in pool:
        for rep in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tt = torch.from_numpy(g["tets"]).cuda()
            nn = torch.from_numpy(g["neighbors"]).cuda()
            gpupr_capi.graph_cut(g["vertices"], tt, nn, g["labels"], 10.0)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            del tt, nn
        service.append(dt)

    def make_trace(rate, seconds):
        r = np.random.default_rng(args.seed + 7 + int(rate))
        n = int(rate * seconds)
        return np.cumsum(r.exponential(1 / rate, size=n)), r.integers(len(pool), size=n)

    def run(arrivals, picks, max_batch, split_tets):
        n_req = len(arrivals)
        results = {}
        with gpupr_capi.Server(hbm_budget_bytes=160 << 30, max_batch=max_batch, split_tets=split_tets) as sv:
            for g0 in (pool[0], pool[int(np.argmax(pool_sizes))]):
                sv.wait(sv.submit(g0["vertices"], g0["tets"], g0["neighbors"], g0["labels"]))
            ids = []
            t_start = time.perf_counter()

            def submitter():
                for k in range(n_req):
                    delay = arrivals[k] - (time.perf_counter() - t_start)
                    if delay > 0:
                        time.sleep(delay)
                    g = pool[picks[k]]
                    ids.append((k, sv.submit(g["vertices"], g["tets"], g["neighbors"], g["labels"])))

            th = threading.Thread(target=submitter)
            th.start()
            done = 0
            while done < n_req:
                while len(ids) <= done:
                    time.sleep(0.0005)
                k, rid = ids[done]
                results[k] = sv.wait(rid)[1]
                done += 1
            th.join()
            wall = time.perf_counter() - t_start
        lat = np.array([results[k]["latency_ms"] for k in range(n_req)])
        bs = np.array([results[k]["batch_size"] for k in range(n_req)])
        small = np.array([len(pool[picks[k]]["labels"]) < split for k in range(n_req)])

        def p99(m):
            return round(float(np.percentile(lat[m], 99)), 2) if m.any() else None

        return {"p50_ms": round(float(np.percentile(lat, 50)), 2),
                "p99_ms": round(float(np.percentile(lat, 99)), 2),
                "p99_small_ms": p99(small), "p99_large_ms": p99(~small),
                "p50_small_ms": round(float(np.percentile(lat[small], 50)), 2) if small.any() else None,
                "cuts_per_s": round(n_req / wall, 2), "mean_batch": round(float(bs.mean()), 2),
                "max_batch": int(bs.max())}

    out = {"config": "Poisson arrivals, tets log-uniform 100k..20M (pool of 12 seeded graphs), "
                     "160 GiB budget, host arrays in and out; small = under 2M tets",
           "lane_split_tets": split}
    for rate, seconds in ((20.0, args.serve_seconds), (100.0, args.serve_seconds / 2)):
        arrivals, picks = make_trace(rate, seconds)
        leg = {"requests": len(arrivals),
               "mean_tets_per_request": int(np.mean([len(pool[p]["labels"]) for p in picks])),
               "two_lanes": run(arrivals, picks, 0, None),
               "one_lane": run(arrivals, picks, 0, 0),
               "one_lane_max_batch_1": run(arrivals, picks, 1, 0)}
        if rate == 20.0:
            free_at, seq_lat = 0.0, []
            for k in range(len(arrivals)):
                start = max(arrivals[k], free_at)
                free_at = start + service[picks[k]]
                seq_lat.append(1e3 * (free_at - arrivals[k]))
            seq_lat = np.array(seq_lat)
            leg["naive_fifo"] = {"p50_ms": round(float(np.percentile(seq_lat, 50)), 2),
                                 "p99_ms": round(float(np.percentile(seq_lat, 99)), 2),
                                 "mean_service_ms": round(1e3 * float(np.mean([service[p] for p in picks])), 2)}
        out[f"rate_{int(rate)}"] = leg
    return out


def run_reference(args, world, rank, local):
    """The reference's own module on the same graph (oracle/_ref)."""
    if rank != 0:
        return None
    import torch

    from oracle.build_ref import built_module, load_reference

    if built_module() is None:
        return {"impl": "reference", "unavailable": "reference module not built in oracle/_ref"}
    ref = load_reference()
    dev = torch.device("cuda", local)
    g = make_graph(args.n_tets, args.seed)
    N = g.n_tets
    tets = torch.from_numpy(g["tets"]).to(dev)
    nbrs = torch.from_numpy(g["neighbors"]).to(dev)
    threads = os.cpu_count() or 1

    def step():
        with quiet_stdout():
            return ref.graph_cut_fast(g["vertices"], tets, nbrs, g["labels"], 10.0, threads, 1024,
                                      2000000, 8)

    for _ in range(args.warmup):
        r = step()
    torch.cuda.synchronize()
    times, solve_s = [], []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            r = step()
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
            solve_s.append(float(r[16]))
    ms = 1e3 * float(np.mean(times))
    v = N / (ms * 1e-3)
    free_n = N - int(r[7]) - int(r[8])      # tets neither fixed source nor fixed sink
    return {
        "impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": "tets/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32/int64 (exact integer flow; FP64 capacities)",
        "data": "synthetic (seeded generator; no CGAL/OpenVDB in the image)",
        "config": bench_config(N, free_n, g, args, world),
        "solve_only": {"ms": round(1e3 * float(np.median(solve_s)), 3),
                       "what": "median of the reference's own solve_seconds per cut (its CUDA "
                               "push-relabel with global relabels and final BFS; host build excluded)"},
        "flow": int(r[1]), "solve": {"rounds": int(r[11]), "global_relabels": int(r[12]),
                                     "build_seconds": float(r[14]), "solve_seconds": float(r[16]),
                                     "native_total_seconds": float(r[17])},
        "cpu_baseline": {"value": round(v, 1), "unit": "tets/s", "cores": threads,
                         "kind": "reference",
                         "sample": "full workload: reference graph_cut_fast (host build on all "
                                   "host threads + its CUDA solver on this GPU), oracle/_ref",
                         "host": host_cpu()},
        "e2e": {"value": round(v, 1), "unit": "tets/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "clocks": clk.summary(),
    }


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            line = run_reference(args, world, rank, local)
        else:
            line = run_ours(args, world, rank, local)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
