"""The bench's multi-rank plumbing on CPU: two gloo ranks, each with its own
replica of the workload (weak scaling, no data-path collective), the timing
reduced as the max over ranks and the per-rank results checked against the
same replicas computed in one process.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import bench

WL = dict(desc="tiny", mols=40, min_atoms=8, max_atoms=20, kind=0, median=14.0, queries=6, qmin=3, qmax=7, skew=(0, 0),
          qkind=0, R=2, seed_d=77, seed_q=78)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import torch

    import oracle

    dist = bench.init_dist(world, "gloo")
    q, d = bench.make_workload(WL, rank)
    res = oracle.run_pipeline(q, d, WL["R"], oracle.REF_PTX, False)
    # each rank reports its own device-style time; the bench keeps the max
    mx = bench.max_over_ranks(dist, float(10 + rank), device=None)
    tot = torch.tensor([res["total"]], dtype=torch.float64)
    dist.all_reduce(tot)
    out[rank] = (int(res["total"]), int(d.graph_offsets[-1]), mx, float(tot.item()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_run_independent_replicas():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        got = dict(out)
    import oracle

    want = []
    for r in range(world):
        q, d = bench.make_workload(WL, r)
        want.append((int(oracle.run_pipeline(q, d, WL["R"], oracle.REF_PTX, False)["total"]), int(d.graph_offsets[-1])))
    assert got[0][0] == want[0][0] and got[1][0] == want[1][0]
    assert got[0][1] != got[1][1] or got[0][0] != got[1][0], "ranks were given the same replica"
    assert got[0][2] == got[1][2] == 11.0  # max over ranks
    assert got[0][3] == got[1][3] == float(want[0][0] + want[1][0])
    assert np.isfinite(got[0][3])


def _shard_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import torch

    import oracle
    import sigmo_b200 as sb

    dist = bench.init_dist(world, "gloo")
    q, d = bench.make_workload(WL, 0)
    full = oracle.run_pipeline(q, d, WL["R"], oracle.REF_PTX, False)  # stands in for the shard's device run
    first, count, base = sb.shard_plan(d, world)[rank]
    off = full["offsets"].astype(np.int64)
    mine = full["per_pair"][off[first]:off[first + count]].astype(np.int64)
    # the exchange step: a sum of the counts and a gather of the per-pair lists
    tot = torch.tensor([int(mine.sum())], dtype=torch.int64)
    dist.all_reduce(tot)
    parts = [None] * world
    dist.all_gather_object(parts, mine.tolist())
    out[rank] = (int(tot.item()), [x for p in parts for x in p], int(full["total"]), full["per_pair"].astype(np.int64).tolist())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_merge_shards_into_the_unsharded_result():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_shard_main, args=(world, _free_port(), out), nprocs=world, join=True)
        got = dict(out)
    for r in range(world):
        tot, merged, want_tot, want_per = got[r]
        assert tot == want_tot and merged == want_per


@pytest.mark.timeout(300)
def test_reference_arm_under_torchrun_prints_one_line_on_all_host_threads():
    """`bench.py --impl reference` launched as two ranks: rank 0 alone runs
    the oracle, on every host thread it may use (not torchrun's
    OMP_NUM_THREADS=1), and prints one JSON line; the other rank exits 0."""
    import json
    import subprocess
    import sys

    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "0", "--workload", "drug1k", "--cpu-sample", "50"]
    res = subprocess.run(cmd, cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))), capture_output=True,
                         text=True, timeout=280)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [json.loads(x) for x in res.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["cores"] == len(os.sched_getaffinity(0))
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
