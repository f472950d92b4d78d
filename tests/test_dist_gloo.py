"""Multi-process (world size 2, gloo, CPU) checks of the N>1 host logic:
sharding covers every problem once, the job time is the maximum over ranks,
and diagnostics gather on rank 0; the work-balanced sharding of the batched
solve, computed independently on each rank from the same batch, partitions it
and its per-rank records merge on rank 0."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from similie_b200 import dist as sd


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        problems = list(range(64))
        mine = sd.shard(problems, *sd.env()[:2])
        t = sd.max_over_ranks(1.0 + rank)          # rank r "took" 1 + r seconds
        got = sd.gather_to_rank0({"rank": rank, "problems": mine})
        q.put((rank, mine, t, got))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_max_time():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    covered = sorted(x for _, mine, _, _ in res for x in mine)
    assert covered == list(range(64))
    assert all(t == 2.0 for _, _, t, _ in res)
    gathered = res[0][3]
    assert [g["rank"] for g in gathered] == [0, 1] and res[1][3] is None


def test_shard_by_work_balances_the_slowest_rank():
    costs = [1024 ** 2] * 5 + [128 ** 2] * 20 + [512 ** 2] * 7
    parts = sd.shard_by_work(costs, 4)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= sum(costs) / 4 + max(costs)
    with pytest.raises(ZeroDivisionError):
        sd.shard([1], 0, 0)


def _work_worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    import similie_b200.magnetostatics as mag
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        allp = mag.synthetic_batch(seed=7, count=64)   # the batch of the solve workload, on every rank
        parts = sd.shard_by_work([p.nx * p.ny for p in allp], world)
        mine = parts[rank]
        nodes = sum(allp[i].nx * allp[i].ny for i in mine)
        # a per-rank record as the solve workload makes one (a converged count, a worst residual)
        rec = {"cg": {"converged": len(mine), "max_rel_residual_oracle": 1e-11 * (rank + 1), "nodes": nodes,
                      "total_iterations": 10 * len(mine), "max_iterations": 100 + rank}}
        got = sd.gather_to_rank0(rec)
        merged = sd.merge_records(got, ("converged", "total_iterations"), ("max_rel_residual_oracle",
                                                                            "max_iterations")) if rank == 0 else None
        q.put((rank, parts, mine, nodes, merged))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_shard_by_work_partitions_the_solve_batch():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_work_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == res[1][1]                        # both ranks computed the same partition
    mine = [r[2] for r in res]
    assert sorted(mine[0] + mine[1]) == list(range(64))  # every problem on exactly one rank
    loads = [r[3] for r in res]
    assert max(loads) - min(loads) <= 1024 * 1024        # balanced to within one of the largest problems
    merged = res[0][4]["cg"]
    assert merged["converged"] == 64 and merged["total_iterations"] == 640
    assert merged["max_rel_residual_oracle"] == 2e-11 and merged["max_iterations"] == 101
