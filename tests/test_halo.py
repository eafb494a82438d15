"""A mesh split into parts with a one-ring halo (hydrob200.halo), CPU.

The plan (parts, halos, send and receive lists) is checked for its
properties; then the parts are stepped by the oracle over the sub-meshes that
plan cuts, with the halo exchanged after every step, in one process (three
parts) and across two gloo ranks (one part each).  Every owned cell must equal
the whole-mesh oracle run bit for bit: an owned cell sees the same neighbours,
geometry and tables as in the whole mesh.  The stress decks carry every
boundary code (KLAS 1, 3, 4, 5, 6, 7, 10).
"""
import ctypes as C
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from hydrob200 import halo

STEPS = 12
STATE = "huvz"


def _oracle_arrays(root):
    from oracle.oracle import OracleDeck
    d = OracleDeck(root)
    names = halo.SLOT_ARRAYS + halo.CELL_ARRAYS + halo.DAY_ARRAYS + ("zw", "qw", "nhq1") + tuple(STATE) + \
        ("w", "f0", "f1", "f2", "f3")
    return {k: d.arr(k).copy() for k in names}, d.scalars


class OracleStepper:
    """One part stepped by the oracle over its sub-mesh arrays (no deck files)."""

    def __init__(self, part, sub, scalars):
        from oracle import oracle as O
        import torch
        self.O, self.part = O, part
        self.sub = {k: np.ascontiguousarray(v) for k, v in sub.items()}
        self.sub["nhq1"] = np.ascontiguousarray(self.sub["nhq1"], dtype=np.int32)
        d = O._Deck()
        d.cells = len(self.sub["zbc"])
        d.ndays, d.mdt, d.nhq = int(scalars["ndays"]), int(scalars["mdt"]), int(scalars["nhq"])
        d.dt, d.hm1, d.hm2, d.jl = scalars["dt"], scalars["hm1"], scalars["hm2"], scalars["jl"]
        for k, v in self.sub.items():
            if k != "nhq1":
                setattr(d, k, v.ctypes.data_as(O._dp))
        d.nhq1 = self.sub["nhq1"].ctypes.data_as(O._ip)
        self.d, self.t = d, 0
        self.rbuf = {q: torch.zeros((len(i), 4), dtype=torch.float64) for q, i in part.recv.items()}

    def step(self, n):
        assert self.O.lib().orc_run(C.byref(self.d), self.O.VARIANT_H, self.t, n) == n
        self.t += n

    def pack(self, q):
        import torch
        idx = self.part.send[q]
        return torch.from_numpy(np.stack([self.sub[k][idx] for k in STATE], axis=1).copy())

    def recv_buffer(self, q):
        return self.rbuf[q]

    def unpack(self, q, records):
        a = records.numpy()
        for i, k in enumerate(STATE):
            self.sub[k][self.part.recv[q]] = a[:, i]

    def owned_state(self):
        return {k.upper(): self.sub[k][self.part.owned_local].copy() for k in STATE}


def _whole(root):
    from oracle.oracle import OracleDeck
    d = OracleDeck(root)
    assert d.run(STEPS) == STEPS
    return {k.upper(): d.arr(k).copy() for k in STATE}


@pytest.mark.parametrize("nparts", [2, 3, 5])
def test_plan_covers_every_cell_once_with_a_one_ring_halo(deck_dir, nparts):
    arrays, _ = _oracle_arrays(deck_dir["f1"])
    nb = arrays["nac"].reshape(-1, 4).astype(np.int64) - 1
    parts = halo.plan(arrays["nac"], nparts)
    owned = np.concatenate([p.owned for p in parts])
    assert np.array_equal(np.sort(owned), np.arange(nb.shape[0]))
    sizes = [len(p.owned) for p in parts]
    assert max(sizes) - min(sizes) <= 1
    for p in parts:
        ring = nb[p.owned].reshape(-1)
        ring = np.setdiff1d(ring[ring >= 0], p.owned)
        assert np.array_equal(np.sort(p.halo), ring)
        assert np.array_equal(np.sort(np.concatenate([p.cells[i] for i in p.recv.values()])), np.sort(p.halo))
        for q, idx in p.recv.items():
            # the records q sends are those p receives, cell for cell
            assert np.array_equal(parts[q].cells[parts[q].send[p.index]], p.cells[idx])
            assert np.all(np.isin(parts[q].cells[parts[q].send[p.index]], parts[q].owned))


def test_sub_mesh_walls_only_the_cut_slots(deck_dir):
    arrays, sc = _oracle_arrays(deck_dir["stress_a"])
    C_ = len(arrays["zbc"])
    for p in halo.plan(arrays["nac"], 3):
        sub = halo.sub_arrays(arrays, C_, sc["ndays"], sc["nhq"], p)
        g = arrays["nac"].reshape(-1, 4)[p.cells].astype(np.int64) - 1
        loc = sub["nac"].reshape(-1, 4).astype(np.int64) - 1
        kl = sub["klas"].reshape(-1, 4)
        inside = np.isin(g, p.cells)
        assert np.array_equal(loc >= 0, (g >= 0) & inside)
        assert np.array_equal(p.cells[loc[loc >= 0]], g[loc >= 0])
        assert np.all(kl[(g >= 0) & ~inside] == halo.KLAS_WALL)
        assert np.array_equal(kl[(g < 0) | inside], arrays["klas"].reshape(-1, 4)[p.cells][(g < 0) | inside])
        # owned cells keep every neighbour
        assert np.all(inside[np.searchsorted(p.cells, p.owned)] | (g[np.searchsorted(p.cells, p.owned)] < 0))


@pytest.mark.parametrize("name,nparts", [("f1", 3), ("stress_a", 3), ("stress_b", 2)])
def test_split_run_equals_whole_mesh(deck_dir, name, nparts):
    arrays, sc = _oracle_arrays(deck_dir[name])
    run = halo.HaloRun(arrays, sc, nparts, lambda part, sub: OracleStepper(part, sub, sc))
    run.step(STEPS)
    got = run.gather()
    want = _whole(deck_dir[name])
    for k in "HUVZ":
        np.testing.assert_array_equal(got[k], want[k], err_msg=f"{name} {k}")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, root, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        arrays, sc = _oracle_arrays(root)
        run = halo.HaloRun(arrays, sc, world, lambda part, sub: OracleStepper(part, sub, sc), rank, world)
        run.step(STEPS)
        q.put((rank, run.gather()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_equal_whole_mesh(deck_dir):
    root = deck_dir["stress_a"]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, root, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[1] is None
    want = _whole(root)
    for k in "HUVZ":
        np.testing.assert_array_equal(res[0][k], want[k], err_msg=k)
