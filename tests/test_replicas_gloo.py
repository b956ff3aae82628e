"""Multi-rank host logic on CPU: two gloo ranks split the batched heat set and reduce their timings.

No GPU: the ranks run the oracle on their shard (as the checker), agree on the assignment without exchanging it, and
the max / sum reductions give the job's time and unit count.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _sizes(count=24, seed=11):
    s = seed
    out = []
    for _ in range(count):  # side N ~ U{8..24} from the uint32 LCG
        s = (s * 1664525 + 1013904223) & 0xFFFFFFFF
        out.append(8 + (s >> 16) % 17)
    return out


def _rank_main(rank, world, port, outdir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import oracle as O
    import workloads as W

    dist = replicas.init("gloo", timeout_s=60)
    info = replicas.RankInfo.from_env()
    sizes = _sizes()
    costs = [float(N) ** 3 for N in sizes]
    mine = replicas.shard_batch(costs, info.world)[info.rank]
    worst = 0.0
    for i in mine:
        w = W.heat2d_lognormal(sizes[i], 100 + i, 2)
        sym = O.analyze(w.pat)
        ok, Lx, *_ = O.factor(sym, w.values)
        assert ok
        for b in w.rhs:
            x = O.solve_chol(sym, Lx, b)
            r = O.matvec(w.pat, w.values, x) - b
            worst = max(worst, float(np.linalg.norm(r) / np.linalg.norm(b)))
    t_job = replicas.max_over_ranks(float(rank + 1))
    units = replicas.sum_over_ranks(float(len(mine)))
    worst_all = replicas.max_over_ranks(worst)
    np.save(os.path.join(outdir, f"r{rank}.npy"), np.array([t_job, units, worst_all] + mine, dtype=np.float64))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_batch_partitions_and_balances():
    costs = [float(N) ** 3 for N in _sizes(256, 7)]
    for world in (1, 2, 3, 8):
        parts = replicas.shard_batch(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)  # LPT bound
        assert parts == replicas.shard_batch(costs, world)  # deterministic


@pytest.mark.timeout(300)
def test_two_gloo_ranks_split_the_batch(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(240)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = [np.load(os.path.join(tmp_path, f"r{r}.npy")) for r in range(world)]
    for r in res:
        assert r[0] == 2.0  # max over ranks of (rank + 1)
        assert r[1] == 24.0  # every problem solved exactly once
        assert r[2] < 1e-12  # worst relative residual over the batch
    shards = [set(r[3:].astype(int).tolist()) for r in res]
    assert shards[0].isdisjoint(shards[1]) and shards[0] | shards[1] == set(range(24))
