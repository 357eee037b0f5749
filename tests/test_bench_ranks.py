"""CPU tests (gloo, world_size 2) of bench.py's multi-rank path: one
independent replica system per rank, the timed region's max over ranks, the
whole-job throughput, and the reference arm running on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT

sys.path.insert(0, ROOT)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime
    import numpy as np
    import torch.distributed as dist
    import bench
    from stokesdt_b200 import workloads as wl
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    # replica systems are independent: different seeds, different positions
    seed = bench.replica_seed(11, rank)
    pos = wl.rsa_positions(200, wl.box_for(200, 0.2), seed)
    local_ms = 100.0 * (rank + 1)            # rank 1 is the slow one
    t = bench.max_over_ranks(dist, local_ms, "cpu")
    rate = bench.aggregate_rate(world, 16 * 3, t)
    out[rank] = (seed, float(pos[0, 0]), t, rate)
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_max_over_ranks_and_aggregate_rate():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    (s0, x0, t0, r0), (s1, x1, t1, r1) = out[0], out[1]
    assert s0 != s1 and x0 != x1
    assert t0 == t1 == 200.0
    assert r0 == r1 == pytest.approx(2 * 48 / 0.2)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    res = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--gpus", "2", "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, env=env, timeout=120)
    assert res.returncode == 0
    assert res.stdout.strip() == ""


def _batch_worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    import bench
    from stokesdt_b200 import workloads as wl
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    systems = wl.batch_systems(nsys=32, seed=5)
    mine, total = bench.batch_units(systems, world, rank)
    cost = sum(wl.system_cost(systems[i]) for i in mine)
    t = bench.max_over_ranks(dist, 10.0 + rank, "cpu")
    out[rank] = (sorted(mine), total, cost, t)
    dist.barrier()
    dist.destroy_process_group()


def test_batch_systems_shard_over_ranks():
    """Config 4 over 2 ranks: disjoint shards covering every system, the job
    total counted once, timed by the slowest rank."""
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    mp.spawn(_batch_worker, args=(2, port, out), nprocs=2, join=True)
    (m0, n0, c0, t0), (m1, n1, c1, t1) = out[0], out[1]
    assert n0 == n1 == 32
    assert not set(m0) & set(m1) and sorted(m0 + m1) == list(range(32))
    assert t0 == t1 == 11.0
    assert max(c0, c1) < 0.6 * (c0 + c1) + 1e-3


def _serve_worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    import bench
    from stokesdt_b200 import workloads as wl
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    systems = bench.serve_systems(world)
    mine = wl.shard_systems(systems, world, rank)
    reqs = bench.serve_requests(len(systems), 60, 40.0, seed=3)
    share = bench.rank_share(reqs, mine)
    lat = bench.gather_all(dist, [float(i) for i in range(len(share))], world)
    span = bench.max_over_ranks(dist, 1.0 + rank, "cpu")
    out[rank] = (sorted(mine), len(systems), [tuple(r) for r in share], len(lat), span)
    dist.barrier()
    dist.destroy_process_group()


def test_serve_stream_shards_over_ranks():
    """Config 5 over 2 ranks: 12 systems per rank, disjoint shards, every
    request of the stream served by exactly one rank (the one owning its
    system), latencies gathered over the whole job, span of the slowest."""
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    mp.spawn(_serve_worker, args=(2, port, out), nprocs=2, join=True)
    (m0, n0, q0, l0, t0), (m1, n1, q1, l1, t1) = out[0], out[1]
    assert n0 == n1 == 24
    assert not set(m0) & set(m1) and sorted(m0 + m1) == list(range(24))
    assert len(q0) + len(q1) == 60 and not set(q0) & set(q1)
    assert all(r[1] in m0 for r in q0) and all(r[1] in m1 for r in q1)
    assert l0 == l1 == 60
    assert t0 == t1 == 2.0
