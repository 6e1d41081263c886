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
* ``batch`` / ``serve`` / ``labels`` / ``audit`` / ``raw`` / ``autotune``: the
  batched cut of 64 uneven graphs, the serving loop under Poisson arrivals,
  the tet-centroid label sampler, the watertight audit of the cut surface, a
  raw integer graph through gpupr_solve_ell, and the autotuner's choice
  (tuned on another graph of the same generator).
* ``cpu_baseline``: the CPU oracle (single-threaded Boykov-Kolmogorov, with
  the reference's graph reduction) on a bounded sample of the same workload.
* ``--impl reference``: the reference's own module (compiled from its
  sources into oracle/_ref) on the same graph: its host graph build on all
  host threads and its CUDA push-relabel on this GPU.

Multi-GPU: a single cut does not shard (every round and BFS level would
need a boundary exchange), so N GPUs run N independent replicas (weak
scaling, no collective on the data path); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import contextlib
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
# two excess updates 16 = 24 B; a BFS frontier expansion reads nbr 16 + rev 1
# + 4 heights 16 + 4 reverse residuals 16 and writes height+queue 8 = 57 B.
B_VISIT, B_PUSH, B_BFS = 73, 24, 57


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
    return ap.parse_args()


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


def make_graph(n_tets, seed):
    import synth

    return synth.config2(seed, n_tets=int(n_tets))


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
    if not args.no_autotune:
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
    with Clocks(local) as clk:
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
        nbytes = B_VISIT * visits + B_PUSH * pushes + B_BFS * bfsv
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
                                      "build": round(sum(s["build_device_ms"] for s in stats) / args.steps, 3)}}
    if rank == 0:
        rs = random_sector_rate(dev)
        roofline["random_sector_gbs"] = round(rs, 1)
        if isinstance(traffic, (int, float)) and kms > 0:
            dram = traffic / (kms / max(launches, 1) * 1e-3) / 1e9
            roofline["traffic_gbs"] = round(dram, 1)
            roofline["traffic_frac_of_random_sector_rate"] = round(dram / rs, 4)

    # e2e through the drop-in module: pinned host topology, host V/labels
    e2e = None
    if not args.no_e2e:
        pt = torch.from_numpy(g["tets"]).pin_memory()
        pn = torch.from_numpy(g["neighbors"]).pin_memory()
        hV = np.ascontiguousarray(g["vertices"])
        hL = np.ascontiguousarray(g["labels"])
        # double-buffered topology: step k+1's upload runs on a copy stream
        # while step k cuts (every step still copies its own inputs in).
        # Both are non-default streams: work on the legacy default stream
        # would wait for every other stream and serialise the two.
        bufs = [(torch.empty_like(tets), torch.empty_like(nbrs)) for _ in range(2)]
        copy_stream = torch.cuda.Stream(dev)
        cut_stream = torch.cuda.Stream(dev)
        ready = [torch.cuda.Event(), torch.cuda.Event()]

        def upload(k):
            """Step k's topology, in 64 MiB pieces with at most one piece in
            the copy queue, so the cut's own host copies are never queued
            behind gigabytes of it (runs on a host thread during the cut)."""
            dt_, dn_ = bufs[k % 2]
            copy_stream.wait_stream(cut_stream)
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
                return wtivo_gpupr.graph_cut_fast(hV, dt_, dn_, hL, 10.0)

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
        a.record(cut_stream)
        upload(0)
        for k in range(args.steps):
            th = None
            if k + 1 < args.steps:
                th = threading.Thread(target=upload, args=(k + 1,))
                th.start()
            r = cut(k)
            if th is not None:
                th.join()
        b.record(cut_stream)
        torch.cuda.synchronize()
        ems, evalue = whole_job(N, a.elapsed_time(b) / args.steps, world)
        serial_ms = max_over_ranks(serial_ms, world)
        h2d = pt.numel() * 4 + pn.numel() * 4 + hV.nbytes + hL.nbytes
        e2e = {"value": round(evalue, 1), "unit": "tets/s",
               "ms_per_step": round(ems, 3), "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(N),
               "serial_ms_per_step": round(serial_ms, 3),
               "api": "wtivo_gpupr.graph_cut_fast with host vertices/labels and labels returned to "
                      "numpy; each step's tets/neighbors copied from pinned memory, step k+1's copy "
                      "on a second stream while step k cuts (serial_ms_per_step: no overlap)"}
        assert np.array_equal(np.asarray(r[0]), out.cpu().numpy()), "e2e labels differ"

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, args.seed)
    batch = run_batch(args, local) if rank == 0 and not args.no_batch else None
    serve = run_serve(args) if rank == 0 and not args.no_serve else None
    labels = run_labels(args, local, g) if rank == 0 and not args.no_labels else None
    audit = run_audit(args, local, g, out, tets, nbrs) if rank == 0 and not args.no_audit else None
    raw = run_raw(args, local) if rank == 0 and not args.no_raw else None

    s0 = stats[-1]
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "tets/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_max, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32/int64 (exact integer flow; FP64 capacities)",
        "data": "synthetic (seeded generator; no CGAL/OpenVDB in the image)",
        "config": {"workload": WORKLOAD, "n_tets": N, "free_nodes": int(s0["free_n"]),
                   "lattice": list(g["shape"]), "lambda_fill": 10.0, "seed": args.seed,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2_flush": "none needed: inputs (2.6 GB topology) exceed the 126 MB L2"},
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
        "batch": batch, "serve": serve, "labels": labels, "audit": audit, "raw": raw, "autotune": tune,
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


def run_raw(args, local):
    """Config 4: a raw integer graph (all nodes free, given integer n-links
    and t-links; gpupr_solve_ell) of 11.7M nodes (125^3-cube Kuhn lattice over
    uniform space, area-proportional n-links, noisy sphere-SDF t-links),
    inputs in HBM; checked by the max-flow = min-cut identity; CPU baseline:
    the BK oracle, 1 core, on the 1.4M-node graph of the same generator."""
    import torch

    import gpupr_capi
    import synth
    from oracle import oracle as orc

    dev = torch.device("cuda", local)
    g = synth.config4(args.seed, n_points=2_000_000, use_delaunay=False)
    nbr, cap, s, k = (torch.from_numpy(np.ascontiguousarray(x)).to(dev)
                      for x in (g["nbr"], g["cap"].view(np.int32), g["src"].view(np.int32),
                                g["snk"].view(np.int32)))
    n = int(nbr.shape[0])
    stream = torch.cuda.current_stream(dev)
    for _ in range(3):
        flow, part, st = gpupr_capi.solve_ell(nbr, cap, s, k)
    ms = cuda_ms(lambda: gpupr_capi.solve_ell(nbr, cap, s, k), 5, stream)
    # certificate: capacity of the returned cut in the input graph
    p = part.long()
    valid = nbr >= 0
    pu = torch.where(valid, p[nbr.long().clamp_min(0)], torch.zeros_like(nbr).long())
    nl = (cap.long() * (valid & (p[:, None] == 0) & (pu == 1))).sum()
    src, snk = s.long(), k.long()
    cut = int((nl + torch.where(p == 0, snk, torch.zeros_like(snk)).sum()
               + torch.where(p == 1, src, torch.zeros_like(src)).sum()).item())
    gs = synth.config4(args.seed, n_points=250_000, use_delaunay=False)
    term = (gs["src"].astype(np.int64) - gs["snk"].astype(np.int64)).astype(np.int32)
    t0 = time.perf_counter()
    orc.maxflow_bk(gs["nbr"], gs["cap"], term)
    cpu_s = time.perf_counter() - t0
    return {"config": "raw integer graph, 125^3-cube Kuhn lattice (11.7M nodes), integer n-links "
                      "round(1e4 area/mean), sphere-SDF t-links, inputs in HBM",
            "nodes": n, "flow": int(flow), "cut_capacity_equals_flow": bool(cut == flow),
            "ms": round(ms, 3), "nodes_per_s": round(n / (ms * 1e-3), 1),
            "solve_device_ms": round(st["solve_device_ms"], 3), "rounds": int(st["rounds"]),
            "global_relabels": int(st["global_relabels"]),
            "cpu_baseline": {"value": round(len(gs["nbr"]) / cpu_s, 1), "unit": "nodes/s", "cores": 1,
                             "kind": "port", "sample": f"{len(gs['nbr'])}-node graph of the same "
                                                       "generator, BK max flow, oracle/wtivo_oracle.c"}}


def run_audit(args, local, g, labels_dev, tets, nbrs):
    """Edge-degree watertight audit of the benchmark cut's surface (device
    faces); CPU baseline: the oracle's sort-and-count, 1 core."""
    import torch

    import gpupr_capi
    import wtivo_gpupr
    from oracle import oracle as orc

    dev = torch.device("cuda", local)
    Vs, F = wtivo_gpupr.surface_extraction_topology_cuda(labels_dev.cpu().numpy(), g["vertices"], tets, nbrs)
    dF = torch.from_numpy(np.ascontiguousarray(F)).to(dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(3):
        bad, nbytes = gpupr_capi.edge_audit(dF)
    ms = cuda_ms(lambda: gpupr_capi.edge_audit(dF), 5, stream)
    t0 = time.perf_counter()
    ref = orc.edge_audit(F)
    cpu_s = time.perf_counter() - t0
    nf = len(F)
    cap = nbytes // 12
    alg = nf * 12 + 3 * nf * 12 + cap * 12 * 2      # faces, 3 edge updates, table clear + scan
    pk, pk_kind = peaks()
    gbs = alg / (ms * 1e-3) / 1e9
    return {"config": "cut surface of the benchmark graph, faces in HBM", "faces": int(nf),
            "bad_edge_groups": int(bad), "identical_to_oracle": bool(bad == ref),
            "faces_per_s": round(nf / (ms * 1e-3), 1), "ms": round(ms, 3),
            "roofline": {"bound": "hbm", "kernel": "k_edge_count + k_edge_bad", "achieved": round(gbs, 1),
                         "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": round(gbs / pk["hbm_gbs"], 4),
                         "peak_source": pk_kind, "algorithmic_bytes": int(alg)},
            "cpu_baseline": {"value": round(nf / cpu_s, 1), "unit": "faces/s", "cores": 1, "kind": "port",
                             "sample": "all faces, oracle/wtivo_oracle.c (qsort of 3F edge keys)"}}


def run_batch(args, local):
    """Config 3: 64 uneven graphs (tets log-uniform 50k..4M) cut as one batch
    vs the same 64 graphs cut one after the other, inputs in HBM."""
    import torch

    import gpupr_capi
    import synth

    dev = torch.device("cuda", local)
    sizes = synth.config3_sizes(args.seed, 64)
    graphs = [synth.config3_graph(i, int(n), args.seed) for i, n in enumerate(sizes)]
    toff, voff, V, T, Nb, L = gpupr_capi.pack_batch(graphs)
    t, nb, v, l = (torch.from_numpy(x).to(dev) for x in (T, Nb, V, L))
    out = torch.empty(len(L), dtype=torch.uint8, device=dev)
    singles = [tuple(torch.from_numpy(np.ascontiguousarray(g[k])).to(dev)
                     for k in ("tets", "neighbors", "vertices", "labels")) for g in graphs]
    outs = [torch.empty(len(g["labels"]), dtype=torch.uint8, device=dev) for g in graphs]
    stream = torch.cuda.current_stream(dev)
    gpupr_capi.graph_cut_batch(toff, voff, v, t, nb, l, 10.0, out=out)
    for (gt, gn, gv, gl), o in zip(singles, outs):
        gpupr_capi.graph_cut(gv, gt, gn, gl, 10.0, out=o)
    torch.cuda.synchronize()
    reps = 3
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        _, items, bst = gpupr_capi.graph_cut_batch(toff, voff, v, t, nb, l, 10.0, out=out)
    b.record(stream)
    torch.cuda.synchronize()
    batch_ms = a.elapsed_time(b) / reps
    a.record(stream)
    seq = []
    for (gt, gn, gv, gl), o in zip(singles, outs):
        _, st = gpupr_capi.graph_cut(gv, gt, gn, gl, 10.0, out=o)
        seq.append(st)
    b.record(stream)
    torch.cuda.synchronize()
    seq_ms = a.elapsed_time(b)
    same = all(items[k]["adjusted_flow"] == seq[k]["adjusted_flow"] for k in range(len(graphs)))
    ob = out.cpu().numpy()
    same = same and all(np.array_equal(ob[int(toff[k]):int(toff[k + 1])], outs[k].cpu().numpy())
                        for k in range(len(graphs)))
    return {"config": "64 graphs, tets log-uniform 50k..4M (holed icosphere / holed torus / "
                      "open rounded box, Kuhn lattices), lambda_fill=10, inputs in HBM",
            "graphs": len(graphs), "tets": int(toff[-1]), "batch_ms": round(batch_ms, 3),
            "sequential_ms": round(seq_ms, 3), "speedup": round(seq_ms / batch_ms, 2),
            "batched_cuts_per_s": round(len(graphs) / (batch_ms * 1e-3), 1),
            "sequential_cuts_per_s": round(len(graphs) / (seq_ms * 1e-3), 1),
            "identical_to_sequential": bool(same), "engine": int(bst["engine"]),
            "rounds": int(bst["rounds"]), "global_relabels": int(bst["global_relabels"])}


def run_serve(args):
    """Config 5: Poisson arrivals at 20 req/s, tets log-uniform 100k..20M,
    160 GiB admission budget.  The same arrival trace goes through the
    continuous-batching server, through the same server one request at a time
    (max_batch 1: FIFO, uploads still overlapping the previous cut), and is
    replayed against one-at-a-time service times measured alone (host arrays
    copied in, cut, labels copied out: the naive FIFO)."""
    import threading

    import torch

    import gpupr_capi
    import synth

    rng = np.random.default_rng(args.seed + 5)
    pool_sizes = np.exp(rng.uniform(np.log(1e5), np.log(2e7), size=12)).astype(np.int64)
    pool = [synth.config3_graph(i, int(n), args.seed + 5) for i, n in enumerate(pool_sizes)]
    n_req = int(20 * args.serve_seconds)
    arrivals = np.cumsum(rng.exponential(1 / 20.0, size=n_req))
    picks = rng.integers(len(pool), size=n_req)

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

    def trace(max_batch):
        results = {}
        with gpupr_capi.Server(hbm_budget_bytes=160 << 30, max_batch=max_batch) as sv:
            g0 = pool[0]
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
        up = np.array([results[k]["upload_ms"] for k in range(n_req)])
        sv_ms = np.array([results[k]["solve_ms"] for k in range(n_req)])
        return {"p50_ms": round(float(np.percentile(lat, 50)), 2),
                "p99_ms": round(float(np.percentile(lat, 99)), 2),
                "cuts_per_s": round(n_req / wall, 2), "mean_batch": round(float(bs.mean()), 2),
                "max_batch": int(bs.max()), "mean_upload_ms": round(float(up.mean()), 2),
                "mean_solve_ms": round(float(sv_ms.mean()), 2)}

    batched = trace(0)
    one_at_a_time = trace(1)
    free_at, seq_lat = 0.0, []
    for k in range(n_req):
        start = max(arrivals[k], free_at)
        free_at = start + service[picks[k]]
        seq_lat.append(1e3 * (free_at - arrivals[k]))
    seq_lat = np.array(seq_lat)
    return {"config": "Poisson 20 req/s for %.0f s, tets log-uniform 100k..20M (pool of 12 "
                      "seeded graphs), 160 GiB budget, host arrays in and out" % args.serve_seconds,
            "requests": n_req, "mean_tets_per_request": int(np.mean([len(pool[p]["labels"]) for p in picks])),
            **batched,
            "server_max_batch_1": one_at_a_time,
            "naive_fifo": {"p50_ms": round(float(np.percentile(seq_lat, 50)), 2),
                           "p99_ms": round(float(np.percentile(seq_lat, 99)), 2),
                           "mean_service_ms": round(1e3 * float(np.mean([service[p] for p in picks])), 2)}}


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
    times = []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            r = step()
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
    ms = 1e3 * float(np.mean(times))
    v = N / (ms * 1e-3)
    return {
        "impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": "tets/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32/int64 (reference: FP64 host capacities, int CUDA push-relabel)",
        "data": "synthetic (seeded generator; no CGAL/OpenVDB in the image)",
        "config": {"workload": WORKLOAD, "n_tets": N, "lattice": list(g["shape"]),
                   "lambda_fill": 10.0, "seed": args.seed, "parallelism": "single GPU"},
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
