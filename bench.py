#!/usr/bin/env python
"""Benchmark of the SIGMo hot path on B200: query x molecule pairs/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sigmo|reference]

A step is one pass of the whole hot path (signatures for iterations 1..R,
label filter + R refinements, GMCR mapping, join with per-pair uint64 counts)
over one batch.  The default workload is 100,000 seeded synthetic molecules
(10-60 heavy atoms) x 600 queries (3-30 atoms, 70% in 6-15), 6 refinement
iterations, find-all, REF_PTX semantics.

value: pairs/s of the batched form with the graphs resident in HBM (device
time from CUDA events on the library's stream, max over ranks).  e2e: the same
metric through the C ABI from pinned host buffers (graph upload + match +
per-pair count read-back every step).  plain_form: the stage-per-launch form
(reference driver order, host sync after every stage).  cpu_baseline: the
CPU oracle (the reference's algorithm restated; the SYCL reference cannot be
built here) on a bounded sample, all host threads.

--impl reference times that CPU implementation alone (rank 0; other ranks
exit 0) and prints the same JSON line with "impl": "reference".

Multi-GPU (torchrun): data graphs are independent, so every rank runs its own
replica of the workload (weak scaling, no data-path collective); the timing
is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "query×molecule pairs/s (bit-exact) on 1 B200 vs plain form; p50/p99 batch latency"

WORKLOADS = {
    "drug100k": dict(
        desc="100,000 synthetic molecules (10-60 atoms) x 600 queries (3-30 atoms, skewed 6-15), 6 refinement iterations",
        mols=100_000, min_atoms=10, max_atoms=60, kind=0, median=22.0, queries=600, qmin=3, qmax=30, skew=(6, 15),
        qkind=0, R=6, seed_d=20251, seed_q=20252),
    "uneven1m": dict(
        desc="1,000,000 synthetic molecules (6-120 atoms, lognormal median 22, 5% macrocycles / fused systems) x 2,000 "
             "queries (3-40 atoms), 6 refinement iterations",
        mols=1_000_000, min_atoms=6, max_atoms=120, kind=1, median=22.0, queries=2000, qmin=3, qmax=40, skew=(0, 0),
        qkind=0, R=6, seed_d=30301, seed_q=30302),
    "symmetry2m": dict(
        desc="2,000,000 ring-rich synthetic molecules (2-6 fused aromatic 6-cycles, carbon chains up to 20) x 300 highly "
             "automorphic queries (6-cycles, fused bi/tri-cycles, carbon chains 4-12, branched stars), 6 refinement iterations",
        mols=2_000_000, min_atoms=10, max_atoms=64, kind=2, median=22.0, queries=300, qmin=4, qmax=14, skew=(0, 0),
        qkind=3, R=6, seed_d=50501, seed_q=50502),
    "drug1k": dict(
        desc="1,000 synthetic molecules (10-40 atoms) x 20 queries (4-12 atoms), 6 refinement iterations",
        mols=1_000, min_atoms=10, max_atoms=40, kind=0, median=22.0, queries=20, qmin=4, qmax=12, skew=(0, 0),
        qkind=0, R=6, seed_d=1001, seed_q=1002),
}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["sigmo", "reference"], default="sigmo")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="drug100k")
    ap.add_argument("--mode", choices=["find-all", "find-first"], default="find-all")
    ap.add_argument("--profile", choices=["ref-ptx", "exact"], default="ref-ptx")
    ap.add_argument("--plain-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-sample", type=int, default=30_000,
                    help="molecules in the CPU-baseline sample (also the GPU/oracle parity sample)")
    ap.add_argument("--ref-step-mols", type=int, default=0,
                    help="reference arm: molecules per step (0: the workload split over warm-up + timed steps, "
                         "1,000-10,000 per step)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mols", type=int, default=0, help="override the workload's molecule count (profiling runs)")
    ap.add_argument("--serve-seconds", type=float, default=3.0, help="length of the serving run (0: skip it)")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="mean request arrivals per second (Poisson)")
    ap.add_argument("--serve-mols", type=int, default=5_000_000,
                    help="serving database size (molecules of 10-40 atoms; 0: the workload's molecules)")
    ap.add_argument("--serve-rates-low", default="20,40,60,80",
                    help="further serving runs at these arrival rates (comma list; empty: none): where p99 <= 50 ms holds")
    ap.add_argument("--serve-inflight", type=int, default=2)
    ap.add_argument("--serve-batch-queries", type=int, default=64, help="most query graphs batched together")
    ap.add_argument("--no-graph", action="store_true", help="time ordinary calls instead of CUDA-graph replays")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default join launch shape")
    ap.add_argument("--join-kernel", type=int, choices=[0, 1, 2], default=None,
                    help="force the join kernel (2: per-lane DFS with CTA-local slot regions, the default; 0: per-lane DFS "
                         "with one work cursor; 1: warp-cooperative frontier) after any autotuning")
    ap.add_argument("--serving-only", action="store_true", help="run only the serving measurement (prints its JSON)")
    ap.add_argument("--shard", action="store_true",
                    help="N>1: split one workload's molecules over the ranks (strong scaling, global ids kept) instead of "
                         "running a replica per rank")
    return ap.parse_args()


# ---- distributed plumbing ----------------------------------------------------------
def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def init_dist(world, backend):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist

    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def max_over_ranks(dist, value: float, device=None) -> float:
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- workload ----------------------------------------------------------------------
def make_workload(wl, rank=0):
    import sigmo_b200 as sb

    d = sb.generate_molecules(wl["mols"], wl["min_atoms"], wl["max_atoms"], seed=wl["seed_d"] + 7919 * rank, kind=wl["kind"],
                              median=wl["median"])
    q = sb.generate_queries(wl["queries"], wl["qmin"], wl["qmax"], seed=wl["seed_q"], kind=wl["qkind"],
                            skew_lo=wl["skew"][0], skew_hi=wl["skew"][1])
    return q, d


def use_all_host_threads():
    """The oracle's OpenMP thread count = the host threads this process may
    run on (torchrun sets OMP_NUM_THREADS=1 for its workers)."""
    import oracle

    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    oracle.lib().orc_set_num_threads(max(1, n))


def cpu_baseline(q, d, wl, sample_mols, find_first, profile):
    """The oracle (CPU restatement of the reference) on the first
    `sample_mols` molecules x all queries, every host thread.  The first
    molecules keep their global vertex ids, so the oracle's GMCR and per-pair
    counts for them are the full batch's (returned for the parity check)."""
    import oracle

    use_all_host_threads()
    ds = d.slice(0, min(sample_mols, d.num_graphs))
    prof = {"ref-ptx": oracle.REF_PTX, "exact": oracle.EXACT}[profile]
    t0 = time.perf_counter()
    out = oracle.run_pipeline(q, ds, wl["R"], prof, find_first)
    dt = time.perf_counter() - t0
    pairs = q.num_graphs * ds.num_graphs
    return {
        "value": pairs / dt,
        "unit": "pairs/s",
        "cores": int(oracle.lib().orc_num_threads()),
        "kind": "port",
        "sample": f"first {ds.num_graphs} molecules x {q.num_graphs} queries of the workload, full pipeline "
                  f"({'find-first' if find_first else 'find-all'}, {wl['R']} iterations), {dt:.2f} s",
        "matches": int(out["total"]),
        "seconds": dt,
    }, out, ds.num_graphs


def parity_sample(ref, n_graphs, offsets, indices, counts):
    """The GPU's GMCR and per-pair counts of the first n_graphs molecules
    against the oracle's for the same molecules (bit-exact comparison)."""
    n_slots = int(offsets[n_graphs])
    same = (np.array_equal(np.asarray(offsets[: n_graphs + 1], dtype=np.int64), ref["offsets"].astype(np.int64))
            and np.array_equal(np.asarray(indices[:n_slots]), ref["indices"])
            and np.array_equal(np.asarray(counts[:n_slots]), ref["per_pair"]))
    return {"molecules": n_graphs, "admitted_pairs": n_slots, "matches": int(ref["total"]),
            "compared": "GMCR offsets and indices, per-pair uint64 counts", "identical": bool(same)}


def out_of_domain(q, d, offsets=None, indices=None):
    """Pairs outside the reference's defined domain: queries of >= 30 vertices
    (its DFS stack holds 30 frames, isomorphism.hpp:288,322) and molecules of
    > 64 atoms (its 64-bit BFS / visited sets, utils.hpp:71-73,
    signature.hpp:353-385).  The oracle defines their results."""
    qs = np.diff(np.asarray(q.graph_offsets, dtype=np.int64))
    ds = np.diff(np.asarray(d.graph_offsets, dtype=np.int64))
    bq, bd = qs >= 30, ds > 64
    nq, nd = int(bq.sum()), int(bd.sum())
    out = {"queries_30_plus": nq, "molecules_over_64": nd,
           "pairs": nq * len(ds) + nd * len(qs) - nq * nd,
           "semantics": "defined by the oracle (dynamic DFS depth; BFS and visited sets over local ids < 64 under ref-ptx)"}
    if offsets is not None:
        g = np.repeat(np.arange(len(ds)), np.diff(np.asarray(offsets, dtype=np.int64)))
        out["admitted_pairs"] = int((bq[np.asarray(indices, dtype=np.int64)] | bd[g]).sum())
    return out


def workload_config(args, wl, q, d, world, shard):
    """The config object of the JSON line; both arms print the same one."""
    R = wl["R"]
    return {"workload": args.workload + ": " + wl["desc"], "molecules": d.num_graphs, "queries": q.num_graphs,
            "data_vertices": d.total_nodes, "query_vertices": q.total_nodes, "iterations": R, "mode": args.mode,
            "profile": args.profile, "pairs_per_step_per_gpu": q.num_graphs * d.num_graphs,
            "l2": "inputs larger than L2: every step writes and re-reads %.0f MB of data-graph signatures "
                  "(iterations 1..%d) plus the candidate planes" % (8 * R * d.total_nodes / 1e6, R),
            "parallelism": (f"shards{world}" if shard else f"replicas{world}") if world > 1 else "single"}


# ---- clocks --------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        # raw samples (the JSON line carries their summary); SIGMO_CLOCKS_DIR keeps them
        out_dir = Path(os.environ.get("SIGMO_CLOCKS_DIR") or tempfile.gettempdir())
        self.path = out_dir / f"sigmo_clocks_rank{index}_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
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
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---- roofline -----------------------------------------------------------------------
def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        j = json.loads(p.read_text())
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


JOIN_KERNELS = {0: "k_join_masks", 1: "k_join_frontier", 2: "k_join_lanes"}  # sigmo_tuning.join_kernel


def traffic_for(kernel: str, workload: str, key: str = "bytes_per_launch"):
    """A per-launch figure of one ncu capture summarised under profiles/."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    j = json.loads(p.read_text())
    e = j.get(f"{kernel}@{workload}")
    return None if e is None else e.get(key)


def join_bytes(q, d, offsets, indices):
    """Algorithmic bytes of one batched join: per admitted pair its slot
    (query id + data graph, 8 B) and count (8 B), one graph-local candidate
    mask per query vertex and one adjacency row per data vertex
    (8 B x words per local set each)."""
    sizes_q = np.diff(np.asarray(q.graph_offsets, dtype=np.int64))
    sizes_d = np.diff(np.asarray(d.graph_offsets, dtype=np.int64))
    aw = max(1, (int(sizes_d.max()) + 63) // 64) if len(sizes_d) else 1
    graph_of_slot = np.repeat(np.arange(len(sizes_d)), np.diff(offsets.astype(np.int64)))
    nq = sizes_q[indices.astype(np.int64)]
    ng = sizes_d[graph_of_slot]
    return int((16 + 8 * aw * (nq + ng)).sum())


def refine_bytes(Qn, N):
    """Algorithmic bytes of one plain refinement pass: the bitset read and
    written once (4 B per 32 (query vertex, data vertex) pairs each way), the
    data and query signatures read once (8 B per vertex)."""
    W = (N + 31) // 32
    return 8 * Qn * W + 8 * N + 8 * Qn


def fused_filter_bytes(Qn, N, R):
    """Algorithmic HBM bytes of one fused filter launch: the final bitset
    written once (4 B per 32 (query vertex, data vertex) pairs, rows padded
    to 128 B), data labels read once, bit-sliced data signatures read once
    (16 labels x 4 planes x 4 B per 32 data vertices per iteration) and the
    query signatures / labels read once."""
    W = (N + 31) // 32
    Wp = (W + 31) // 32 * 32
    return 4 * Qn * Wp + N + R * 16 * 16 * Wp + 8 * R * Qn + Qn


# ---- serving loop ---------------------------------------------------------------------
def run_serving(args, d, wl, local):
    """The serving loop against a resident database (default 5,000,000
    molecules of 10-40 atoms, ~125M vertices): Poisson arrivals of requests of
    1-64 query graphs (3-30 atoms, skewed 6-15), find-first, continuous
    batching; latency = submit -> per-query results on the host, measured
    inside the library.  Runs at `--serve-rate` (the target rate, 200/s) and at
    each of `--serve-rates-low`, each for `--serve-seconds` of arrivals, on one
    server."""
    import threading

    import sigmo_b200 as sb

    if args.serve_mols and args.serve_mols != d.num_graphs:
        # the serving database shape: molecules of 10-40 heavy atoms (5M molecules ~ 125M vertices)
        d = sb.generate_molecules(args.serve_mols, 10, 40, seed=wl["seed_d"] + 17, kind=0)
    hbm, _ = peaks()
    t_setup = time.perf_counter()
    srv = sb.Server(d, device=local, iterations=wl["R"], find_first=True, max_inflight=args.serve_inflight,
                    max_batch_queries=args.serve_batch_queries)
    setup_s = time.perf_counter() - t_setup
    warm = [sb.generate_queries(k, 3, 30, seed=690_000 + k, skew_lo=6, skew_hi=15) for k in (1, 16, 64, 40)]
    # warm-up: requests before the timed arrivals, some at once so that every
    # worker has run (and the memory pool holds) concurrent batches
    for _ in range(2):
        for t in [srv.submit(warm[i % len(warm)]) for i in range(2 * args.serve_inflight)]:
            srv.wait(t)
            srv.release(t)

    def one_rate(rate, seed):
        rng = np.random.default_rng(seed)
        n_req = max(1, int(round(rate * args.serve_seconds)))
        sizes = rng.integers(1, 65, n_req)
        reqs = [sb.generate_queries(int(k), 3, 30, seed=seed * 1000 + i, skew_lo=6, skew_hi=15) for i, k in enumerate(sizes)]
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
        tickets = [None] * n_req

        def submitter():
            t0 = time.perf_counter()
            for i in range(n_req):
                delay = arrivals[i] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                tickets[i] = srv.submit(reqs[i])

        st0 = srv.stats()
        with ClockSampler(local) as clk:
            t0 = time.perf_counter()
            th = threading.Thread(target=submitter)
            th.start()
            th.join()
            results = [srv.wait(t) for t in tickets]
            wall = time.perf_counter() - t0
        st1 = srv.stats()
        for t in tickets:
            srv.release(t)
        lat = np.array([r["ms_latency"] for r in results])
        qms = np.array([r["ms_queue"] for r in results])
        pairs = sum(r["pairs"] for r in results)
        big = [r["ms_latency"] for r, k in zip(results, sizes) if k == 64 or r["batch_queries"] >= 48]
        # admission: the resident plane rows each batch gathers / its filter-stage time
        by_batch = {}
        for r in results:
            by_batch[r["batch_id"]] = r
        adm = [b["gathered_plane_bytes"] / (b["ms_filter"] / 1e3) / 1e9 for b in by_batch.values()
               if b["gathered_plane_bytes"] and b["ms_filter"] > 0]
        p99 = float(np.percentile(lat, 99))

        def stage_medians(batches):
            if not batches:
                return None
            return {k: round(float(np.median([b[f] for b in batches])), 3)
                    for k, f in (("device", "ms_device"), ("filter", "ms_filter"), ("mapping", "ms_mapping"),
                                 ("join", "ms_join"), ("queries", "batch_queries"))} | {"batches": len(batches)}

        return {
            "requests": n_req, "arrival_rate_per_s": rate, "queries_per_request": "uniform 1-64",
            "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3), "p95": round(float(np.percentile(lat, 95)), 3),
                           "p99": round(p99, 3), "max": round(float(lat.max()), 3)},
            "target_p99_ms": 50.0, "meets_target": bool(p99 <= 50.0), "p99_over_target": round(p99 / 50.0, 2),
            "latency_ms_full_batches_p99": round(float(np.percentile(big, 99)), 3) if big else None,
            "queue_ms_p50": round(float(np.percentile(qms, 50)), 3),
            "pairs_per_s": round(pairs / wall, 1),
            "wall_s": round(wall, 3),
            "batches": st1["batches"] - st0["batches"],
            "mean_requests_per_batch": round((st1["requests_completed"] - st0["requests_completed"]) /
                                             max(1, st1["batches"] - st0["batches"]), 2),
            "batch_stages_ms_median": {"all": stage_medians(list(by_batch.values())),
                                       "batches_of_48_plus_queries": stage_medians(
                                           [b for b in by_batch.values() if b["batch_queries"] >= 48])},
            "admission_gather_gbs_median": round(float(np.median(adm)), 1) if adm else None,
            "admission_gather_frac_of_hbm": round(float(np.median(adm)) / hbm, 4) if adm else None,
            "clocks": clk.summary(),
        }

    runs = {"target_rate": one_rate(args.serve_rate, 4242)}
    lows = [float(x) for x in args.serve_rates_low.split(",") if x.strip()]
    if lows:
        runs["lower_rates"] = [one_rate(rate, 4343 + i) for i, rate in enumerate(lows)]
        held = [r["arrival_rate_per_s"] for r in runs["lower_rates"] if r["meets_target"]]
        runs["highest_rate_meeting_target"] = max(held) if held else None
    st = srv.stats()
    srv.close()
    return {
        "database": {"molecules": d.num_graphs, "vertices": d.total_nodes, "directed_edges": d.total_edges,
                     "resident_bytes": st["resident_bytes"], "setup_s": round(setup_s, 2)},
        "mode": "find-first", "max_inflight": args.serve_inflight, "max_batch_queries": args.serve_batch_queries,
        "max_batches_in_flight": st["max_batches_in_flight"], "peak_reserved_bytes": st["peak_reserved_bytes"],
        "admission_note": "gathered plane rows (8 B x 32 graphs x words per vertex set, per plane and 32-graph tile) "
                          "over the batch's filter-stage time (query signatures + admission), against the measured "
                          "HBM copy bandwidth",
        **runs,
    }


# ---- the sigmo arm -------------------------------------------------------------------
def run_sigmo(args, rank, world, local):
    import torch

    import sigmo_b200 as sb

    wl = dict(WORKLOADS[args.workload])
    if args.mols:
        wl["mols"] = args.mols
    torch.cuda.set_device(local)
    dist = init_dist(world, "nccl")
    ff = args.mode == "find-first"
    shard = args.shard and world > 1
    q, d = make_workload(wl, 0 if shard else rank)
    R = wl["R"]
    pairs = q.num_graphs * d.num_graphs
    if args.serving_only:
        if rank == 0:
            print(json.dumps({"serving": run_serving(args, d, wl, local)}))
        return

    queue = sb.Queue(local, profile=args.profile)
    qg = sb.createDeviceCSRGraph(queue, q)
    if shard:  # this rank's contiguous range of molecules; the job's pairs are counted once
        first, count, _ = sb.shard_plan(d, world)[rank]
        dg = sb.createDeviceShard(queue, d, first, count)
    else:
        dg = sb.createDeviceCSRGraph(queue, d)
    gm = sb.GMCR(queue)
    stream = torch.cuda.ExternalStream(queue.stream, device=local)

    tuning = None
    if not args.no_autotune:
        tuning = sb.autotune(queue, qg, dg, R, ff, reps=2)
    if args.join_kernel is not None:
        queue.set_tuning(join_kernel=args.join_kernel)
        if tuning is not None:
            tuning["join_kernel"] = args.join_kernel
    graph = not args.no_graph
    for _ in range(max(args.warmup, 0)):
        res = sb.match_batched(queue, qg, dg, R, ff, None, gm)
    queue.wait()

    # ---- per-stage device times: ordinary calls (CUDA events per stage) ----
    stage = []
    for _ in range(args.steps):
        stage.append(sb.match_batched(queue, qg, dg, R, ff, None, gm))
    if graph:  # capture, then warm the replay
        for _ in range(max(args.warmup, 1)):
            sb.match_batched(queue, qg, dg, R, ff, None, gm, graph=True)
    queue.wait()

    # ---- timed region: K steps, device-resident inputs ----
    step_ms = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = queue.launch_count()
    with ClockSampler(local) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            res = sb.match_batched(queue, qg, dg, R, ff, None, gm, graph=graph)
            step_ms.append(res["ms_total"])
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    launches = queue.launch_count() - launches0
    elapsed_ms = ev0.elapsed_time(ev1)
    elapsed_ms = max_over_ranks(dist, elapsed_ms, device=f"cuda:{local}")
    ms_per_step = elapsed_ms / args.steps
    value = (1 if shard else world) * pairs / (ms_per_step / 1e3)
    total_matches = res["total_matches"]
    if shard:  # the exchange step of a sharded job: the sum of the shards' counts
        t = torch.tensor([total_matches], dtype=torch.int64, device=f"cuda:{local}")
        dist.all_reduce(t)
        total_matches = int(t.item())
    admitted = res["admitted_pairs"]

    # ---- per-stage device times (timed steps) and the dominant kernel's roofline ----
    med = lambda k: statistics.median(s[k] for s in stage)  # noqa: E731
    stages = {k: round(med(k), 4) for k in ("ms_signatures", "ms_filter", "ms_mapping", "ms_join", "ms_total")}
    hbm, peak_kind = peaks()
    offsets, indices = gm.getGMCR()
    jb = join_bytes(q, d, offsets, indices)
    join_ms = med("ms_join")
    achieved = jb / (join_ms / 1e3) / 1e9
    jk = JOIN_KERNELS.get(queue.get_tuning()["join_kernel"], "k_join_lanes")
    jkey = f"join:{jk}"
    l1, l2 = traffic_for(jkey, args.workload, "l1_hit_rate"), traffic_for(jkey, args.workload, "l2_hit_rate")
    roof = {"kernel": f"join stage: k_pair_masks + {jk} (side stream: k_join_fast for queries over 16 vertices, "
                      "k_join_literal_small for the data graphs starting below vertex 256)",
            "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
            "frac": round(achieved / hbm, 4), "traffic": traffic_for(jkey, args.workload),
            "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs, burst copy)" if peak_kind == "measured" else peak_kind,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of k_pair_masks and the phase-B kernel "
                              "on a 20,000-molecule slice of this workload, scaled to this batch by admitted pairs "
                              "(profiles/traffic.json); the phase-B counters below come from the same capture",
            "algorithmic_bytes_per_launch": jb, "ms_per_launch": round(join_ms, 4),
            "warp_execution_efficiency": traffic_for(jkey, args.workload, "warp_execution_efficiency"),
            "active_warps_of_peak": traffic_for(jkey, args.workload, "active_warps_of_peak"),
            "issue_active_of_peak": traffic_for(jkey, args.workload, "issue_active_of_peak"),
            "note": "DFS over admitted pairs: latency- and issue-bound, no bandwidth roofline applies (ncu: threads "
                    "per instruction / 32, active warps and issue-active fraction above"
                    + (f"; L1 hit rate {l1:.0%}, L2 hit rate {l2:.0%}" if l1 is not None and l2 is not None else "")
                    + f"); the stage is {100 * join_ms / stages['ms_total']:.0f}% of the step"}

    # ---- the plain stage-per-launch form (same results, reference order) ----
    plain = None
    if args.plain_steps > 0 and not shard:
        def plain_step(check=False):
            sig = sb.Signature(queue, dg.total_nodes, qg.total_nodes)
            c2 = sb.Candidates(queue, qg.total_nodes, dg.total_nodes)
            sig.generateDataSignatures(dg)
            sig.generateQuerySignatures(qg)
            sb.filterCandidates(queue, qg, dg, sig, c2)
            queue.wait()
            for r in range(1, R + 1):
                sig.refineDataSignatures(dg, r)
                queue.wait()
                sig.refineQuerySignatures(qg, r)
                queue.wait()
                ev = sb.refineCandidates(queue, qg, dg, sig, c2)
                queue.wait()
                refine_ms.append(ev.getProfilingInfo() * 1e3)
            g2 = sb.GMCR(queue)
            gev = g2.generateGMCR(qg, dg, c2)
            gmcr_ms.append(gev.getProfilingInfo() * 1e3)
            nm = np.zeros(1, np.uint64)
            sb.joinCandidates(queue, qg, dg, c2, g2, nm, ff)
            queue.wait()
            dig = c2.digest() if check else None
            adm = g2.total_query_indices
            sig.close()
            c2.close()
            g2.close()
            return int(nm[0]), dig, adm

        refine_ms, gmcr_ms = [], []
        plain_step()  # warm-up
        refine_ms.clear()
        gmcr_ms.clear()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.plain_steps):
            p_total, _, p_adm = plain_step()
        torch.cuda.synchronize()
        p_ms = (time.perf_counter() - t0) * 1e3 / args.plain_steps
        refine_ms_timed = list(refine_ms)
        _, p_digest, _ = plain_step(check=True)  # final-bitset digest, outside the timed region
        refine_ms[:] = refine_ms_timed
        rb = refine_bytes(qg.total_nodes, dg.total_nodes)
        r_ms = statistics.median(refine_ms)
        r_ach = rb / (r_ms / 1e3) / 1e9
        gb = 4 * qg.total_nodes * ((dg.total_nodes + 31) // 32) + 8 * dg.num_graphs
        g_ms = statistics.median(gmcr_ms)
        g_ach = gb / (g_ms / 1e3) / 1e9
        plain = {"value": pairs / (p_ms / 1e3), "unit": "pairs/s", "ms_per_step": round(p_ms, 3),
                 "batched_over_plain": round((pairs / (ms_per_step / 1e3)) / (pairs / (p_ms / 1e3)), 3),
                 "identical_results": bool(p_total == total_matches and p_adm == admitted),
                 "roofline_refine": {"kernel": "k_sig_planes + k_refine (one refinement pass)", "bound": "hbm",
                                     "achieved": round(r_ach, 1), "peak": hbm, "unit": "GB/s", "frac": round(r_ach / hbm, 4),
                                     "traffic": traffic_for("k_refine", args.workload),
                                     "algorithmic_bytes_per_launch": rb, "ms_per_launch": round(r_ms, 4)},
                 "roofline_gmcr": {"kernel": "GMCR stage (k_gmcr_ne's one read of the final bitset, admission, scan, "
                                             "fill; stage events, so the fraction is a lower bound for k_gmcr_ne)",
                                   "bound": "hbm", "achieved": round(g_ach, 1), "peak": hbm, "unit": "GB/s",
                                   "frac": round(g_ach / hbm, 4), "algorithmic_bytes_per_launch": gb,
                                   "ms_per_launch": round(g_ms, 4)}}

    # ---- e2e through the C ABI from pinned host buffers ----
    e2e = None
    if args.e2e_steps > 0 and not shard:
        import ctypes

        from sigmo_b200 import _lib as L

        def pinned_copy(h):
            arrs = {}
            for f, dt in (("graph_offsets", torch.int32), ("row_offsets", torch.int32), ("column_indices", torch.int32),
                          ("node_labels", torch.uint8), ("edge_labels", torch.uint8)):
                a = np.asarray(getattr(h, f))
                t = torch.empty(max(a.size, 1), dtype=dt, pin_memory=True)
                t.numpy()[: a.size] = a.view(np.int32) if dt == torch.int32 else a
                arrs[f] = t
            raw = L.HostGraphsC(h.num_graphs, h.total_nodes, h.total_edges, arrs["graph_offsets"].data_ptr(),
                                arrs["row_offsets"].data_ptr(), arrs["column_indices"].data_ptr(),
                                arrs["node_labels"].data_ptr(), arrs["edge_labels"].data_ptr())
            nbytes = sum(int(np.asarray(getattr(h, f)).nbytes) for f in arrs)
            return raw, arrs, nbytes

        qraw, qkeep, qbytes = pinned_copy(q)
        draw, dkeep, dbytes = pinned_copy(d)
        counts_host = torch.empty(max(admitted, 1), dtype=torch.int64, pin_memory=True)
        lib = L.lib()

        def e2e_step(per_pair):
            hq, hd = ctypes.c_void_p(), ctypes.c_void_p()
            L.check(lib.sigmo_graph_create(queue._h, ctypes.byref(qraw), ctypes.byref(hq)))
            L.check(lib.sigmo_graph_create(queue._h, ctypes.byref(draw), ctypes.byref(hd)))
            r = L.MatchResultC()  # the call reads back the admitted and matched totals (8 B each)
            L.check(lib.sigmo_match_batched(queue._h, hq, hd, R, int(ff), 0, None, gm._h, ctypes.byref(r)))
            if per_pair:
                L.check(lib.sigmo_match_download_counts(gm._h, ctypes.c_void_p(counts_host.data_ptr()), counts_host.numel()))
            lib.sigmo_graph_destroy(hq)
            lib.sigmo_graph_destroy(hd)
            return r.total_matches, r.admitted_pairs

        def e2e_time(per_pair):
            e2e_step(per_pair)
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.e2e_steps):
                et, ea = e2e_step(per_pair)
            e1.record(stream)
            e1.synchronize()
            e_ms = max_over_ranks(dist, e0.elapsed_time(e1), device=f"cuda:{local}") / args.e2e_steps
            return e_ms, et, ea

        # the result the reference's API returns (joinCandidates' num_matches) ...
        e_ms, et, ea = e2e_time(False)
        e2e = {"value": world * pairs / (e_ms / 1e3), "unit": "pairs/s", "ms_per_step": round(e_ms, 3),
               "h2d_bytes_per_step": qbytes + dbytes, "d2h_bytes_per_step": 16, "result": "match and pair totals",
               "identical_results": bool(et == total_matches and ea == admitted)}
        # ... and with every pair's count downloaded as well
        p_ms, pt, pa = e2e_time(True)
        e2e["with_per_pair_counts"] = {"value": world * pairs / (p_ms / 1e3), "ms_per_step": round(p_ms, 3),
                                       "d2h_bytes_per_step": 8 * pa + 16,
                                       "identical_results": bool(pt == total_matches and pa == admitted)}

    serving = None
    if args.serve_seconds > 0 and world == 1:
        serving = run_serving(args, d, wl, local)

    cpu = parity = None
    ood = out_of_domain(q, d, offsets, indices) if not shard else out_of_domain(q, d)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, cref, n_sample = cpu_baseline(q, d, wl, args.cpu_sample, ff, args.profile)
        parity = parity_sample(cref, n_sample, offsets, indices, gm.getPairCounts())
        del cref

    if dist:
        torch.cuda.synchronize()
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    out = {
        "metric": METRIC,
        "value": round(value, 1),
        "unit": "pairs/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True,
        "scaling": "strong" if shard else "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded generator; SIGMo's SMARTS/ZINC sets are not available)",
        "config": workload_config(args, wl, q, d, world, shard),
        "value_scope": "value times CUDA-graph replays of the batched form with both graph batches resident; the query "
                       "batch's plane program (its signatures and the host-side class program) is built once per query "
                       "batch and cached on the query handle, so replays skip it; e2e creates both graphs every step "
                       "and so rebuilds it",
        "latency_ms": {"p50": round(float(np.percentile(step_ms, 50)), 3), "p99": round(float(np.percentile(step_ms, 99)), 3)},
        "stages_ms": stages,
        "admitted_pairs": admitted,
        "total_matches": total_matches,
        "roofline": roof,
        "parity_sample": parity,
        "out_of_domain": ood,
        "plain_form": plain,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
        "cuda_graph": graph,
        "tuning": tuning,
        "serving": serving,
    }
    print(json.dumps(out))


# ---- the reference arm ------------------------------------------------------------------
def run_reference(args, rank, world, local):
    """The reference's algorithm on the host cores: the oracle (its CPU
    restatement, REF_PTX semantics, -O3 and OpenMP) on the same workload and
    config as the sigmo arm.  No SYCL compiler is installed; the reference's
    own source runs on the host only through the SYCL stand-in under
    oracle/ (one work-group at a time, -O0), which computes the REF_X86
    semantics and serves as the oracle's checker, not as a timed baseline.  Inputs come from the host-only
    workload library (oracle/libsigmo_workload.so, the same seeded
    generator), so this arm never maps the product's CUDA library.  Each step
    runs the full pipeline on the next contiguous slice of the workload's
    molecules (ids re-based to 0) x all queries, so the warm-up and timed
    steps together walk the whole workload."""
    if rank != 0:
        return
    import oracle
    from oracle import workload

    wl = WORKLOADS[args.workload]
    ff = args.mode == "find-first"
    d = workload.generate_molecules(wl["mols"], wl["min_atoms"], wl["max_atoms"], seed=wl["seed_d"], kind=wl["kind"],
                                    median=wl["median"])
    q = workload.generate_queries(wl["queries"], wl["qmin"], wl["qmax"], seed=wl["seed_q"], kind=wl["qkind"],
                                  skew_lo=wl["skew"][0], skew_hi=wl["skew"][1])
    prof = {"ref-ptx": oracle.REF_PTX, "exact": oracle.EXACT}[args.profile]
    total_steps = max(args.warmup, 0) + max(args.steps, 1)
    per_step = args.ref_step_mols or min(10_000, max(1_000, -(-d.num_graphs // total_steps)))
    per_step = max(1, min(per_step, d.num_graphs))
    use_all_host_threads()
    cursor = 0

    def step():
        nonlocal cursor
        if cursor >= d.num_graphs:
            cursor = 0
        ds = workload.slice_graphs(d, cursor, per_step)
        cursor += ds.num_graphs
        t0 = time.perf_counter()
        out = oracle.run_pipeline(q, ds, wl["R"], prof, ff)
        return time.perf_counter() - t0, q.num_graphs * ds.num_graphs, int(out["total"])

    for _ in range(max(args.warmup, 0)):
        step()
    times, pairs, matches = [], 0, 0
    for _ in range(args.steps):
        dt, p, m = step()
        times.append(dt)
        pairs += p
        matches += m
    v = pairs / sum(times)
    sample = (f"{args.steps} timed steps, each the full pipeline on the next {per_step} molecules of the workload (ids "
              f"re-based to 0) x all {q.num_graphs} queries ({'find-first' if ff else 'find-all'}, {wl['R']} "
              f"iterations); no SYCL compiler is installed (the reference's own source builds for the host only "
              f"through a one-work-group-at-a-time SYCL stand-in at -O0 with REF_X86 semantics, used as the "
              f"oracle's checker), so its CPU restatement runs, on all host threads")
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(v, 1),
        "unit": "pairs/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(sum(times) / len(times) * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded generator; SIGMo's SMARTS/ZINC sets are not available)",
        "config": workload_config(args, wl, q, d, 1, False),
        "latency_ms": {"p50": round(float(np.percentile(times, 50)) * 1e3, 3),
                       "p99": round(float(np.percentile(times, 99)) * 1e3, 3)},
        "cpu_baseline": {"value": round(v, 1), "unit": "pairs/s", "cores": int(oracle.lib().orc_num_threads()),
                         "kind": "port", "sample": sample},
        "e2e": {"value": round(v, 1), "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "total_matches_timed_steps": matches,
    }
    print(json.dumps(line))


def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world, local)
    else:
        run_sigmo(args, rank, world, local)


if __name__ == "__main__":
    main()
