"""Scenario sharding over ranks (hydrob200.shard), CPU.

The multi-GPU ensemble runs one process per GPU, each stepping its share of
the scenarios with no data-path exchange, and gathers results on rank 0.  The
share assignment and the gathering are host logic, tested here with two gloo
ranks on the CPU.  The stepper is the CPU oracle (one OracleDeck per
scenario), so the gathered states must equal a single-process run bit for bit.
"""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from hydrob200.shard import ShardedRun, lpt_shards

NAMES = ["stress_a", "f1", "stress_b", "probe"]
STEPS = 10


def test_lpt_assigns_each_scenario_once_and_balances():
    rng = np.random.default_rng(3)
    for n, ranks in ((64, 8), (13, 4), (5, 8), (1, 2)):
        sizes = np.exp(rng.uniform(np.log(5e3), np.log(2e5), n)).astype(int)
        shards = lpt_shards(sizes, ranks)
        assert sorted(i for s in shards for i in s) == list(range(n))
        loads = [int(sum(sizes[i] for i in s)) for s in shards]
        bound = max(int(sizes.max()), int(np.ceil(sizes.sum() / ranks)))
        assert max(loads) <= 4 * bound / 3
        assert shards == lpt_shards(sizes, ranks)   # deterministic


class OracleStepper:
    def __init__(self, roots):
        from oracle.oracle import OracleDeck
        self.decks = [OracleDeck(r) for r in roots]

    def step(self, n):
        for d in self.decks:
            d.run(n)

    def get_state(self, k):
        return self.decks[k].dump()


def _rank_main(rank, world, port, roots, sizes, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        run = ShardedRun(sizes, lambda idx: OracleStepper([roots[i] for i in idx]), rank, world)
        run.step(STEPS)
        got = run.gather("H")
        worst = run.max_over_ranks(float(rank + 1))
        q.put((rank, run.mine, got, worst))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_gather_what_one_process_computes(deck_dir):
    from oracle.oracle import OracleDeck
    import hydrob200 as hb
    roots = [deck_dir[n] for n in NAMES]
    sizes = [hb.Deck(r).cells for r in roots]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, roots, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        rank, mine, got, worst = q.get(timeout=300)
        res[rank] = (mine, got, worst)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(res[0][0] + res[1][0]) == list(range(len(NAMES)))
    assert res[0][2] == res[1][2] == 2.0          # max over ranks
    assert res[1][1] is None
    gathered = res[0][1]
    assert sorted(gathered) == list(range(len(NAMES)))
    for i, r in enumerate(roots):
        o = OracleDeck(r)
        o.run(STEPS)
        np.testing.assert_array_equal(gathered[i], o.dump()["H"], err_msg=NAMES[i])
