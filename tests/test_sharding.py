"""Sharding of independent worlds across ranks: the LPT partition and the
end-of-run gather, on world_size 2 over gloo (CPU).  The per-rank runner here
is the oracle, standing in for the per-GPU batched engine."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from autoverse_b200 import sharding, workloads as wl


def test_lpt_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    costs = list(rng.uniform(1, 100, 200))
    for n in (1, 2, 3, 8):
        parts = sharding.lpt_partition(costs, n)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(200))
        loads = [sum(costs[i] for i in p) for p in parts]
        lower = max(sum(costs) / n, max(costs))
        assert max(loads) <= 4.0 / 3.0 * lower + 1e-9


def test_lpt_is_deterministic_and_handles_empty():
    costs = [5.0, 5.0, 5.0, 1.0]
    assert sharding.lpt_partition(costs, 2) == sharding.lpt_partition(costs, 2)
    assert sharding.lpt_partition([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        sharding.lpt_partition(costs, 0)


def test_world_cost_grows_with_size_and_kernels():
    small, _ = wl.single_blob(64)
    big, _ = wl.single_blob(256)
    multi, _ = wl.multispecies(64, channels=2, R=8)
    assert sharding.world_cost(big) > 10 * sharding.world_cost(small)
    assert sharding.world_cost(multi) > sharding.world_cost(small)


def oracle_runner(worlds, steps):
    from oracle import oracle as O
    out = []
    for cfg, seed in worlds:
        st = O.OraclePropagator(cfg).run(O.seed_generate(seed, cfg), steps)
        out.append(float(st.astype(np.float64).sum()))
    return out


def _rank_main(rank, world_size, port, worlds, steps, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        res = sharding.run_sharded(worlds, steps, rank, world_size, runner=oracle_runner)
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_run_sharded_two_ranks_matches_single_process():
    worlds = wl.batched_worlds(6, sides=(64, 96), seed=21)
    steps = 2
    expected = oracle_runner(worlds, steps)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, worlds, steps, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results[0] == results[1] == expected
