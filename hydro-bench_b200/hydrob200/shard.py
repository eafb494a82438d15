"""Sharding a batch of independent scenarios over ranks (one process per GPU).

Scenarios never exchange data, so a rank steps its share as one batch
(``hydrob200.Batch``) with no collective on the data path.  Shares are chosen
by longest-processing-time first: scenarios in decreasing cell count, each to
the rank with the least cells so far (the lower rank on ties), which keeps the
largest load within 4/3 of the optimum.  At the end, per-scenario results are
gathered on rank 0 and the timing is the maximum over ranks.
"""
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np


def lpt_shards(sizes: Sequence[int], nranks: int) -> List[List[int]]:
    """Scenario indices per rank (each list in increasing index order)."""
    if nranks <= 0:
        raise ValueError("nranks must be positive")
    load = [0] * nranks
    shards: List[List[int]] = [[] for _ in range(nranks)]
    for i in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        r = min(range(nranks), key=lambda r: (load[r], r))
        shards[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(s) for s in shards]


class ShardedRun:
    """One rank's share of a scenario batch.

    ``make(indices)`` builds this rank's stepper over the given scenarios;
    the stepper offers ``step(n)`` and ``get_state(k)`` (k = position within
    the share, states in the scenario's reference order).  ``hydrob200.Batch``
    is the GPU stepper; any object with those two methods will do.
    """

    def __init__(self, sizes: Sequence[int], make: Callable[[List[int]], object], rank: int = 0, world: int = 1,
                 group=None):
        self.sizes = [int(s) for s in sizes]
        self.rank, self.world, self.group = rank, world, group
        self.shards = lpt_shards(self.sizes, world)
        self.mine = self.shards[rank]
        self.stepper = make(self.mine) if self.mine else None

    @property
    def cells(self) -> int:
        """Cells stepped by this rank."""
        return sum(self.sizes[i] for i in self.mine)

    def step(self, n: int) -> None:
        if self.stepper is not None:
            self.stepper.step(n)

    def max_over_ranks(self, value: float) -> float:
        if self.world == 1:
            return value
        import torch
        import torch.distributed as dist
        t = torch.tensor([value], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
        return float(t.item())

    def gather(self, field: str = "H") -> Optional[Dict[int, np.ndarray]]:
        """{scenario: state[field]} of every scenario on rank 0 (None elsewhere)."""
        local = {i: np.asarray(self.stepper.get_state(k)[field], dtype=np.float64)
                 for k, i in enumerate(self.mine)} if self.stepper is not None else {}
        if self.world == 1:
            return local
        import torch.distributed as dist
        parts = [None] * self.world if self.rank == 0 else None
        dist.gather_object(local, parts, dst=0, group=self.group)
        if self.rank != 0:
            return None
        out: Dict[int, np.ndarray] = {}
        for p in parts:
            out.update(p)
        return out
