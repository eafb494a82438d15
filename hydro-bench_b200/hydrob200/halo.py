"""One mesh split into parts with a one-ring halo, exchanged after every step.

For meshes larger than one GPU holds.  The cells are ordered by reverse
Cuthill-McKee over the neighbour graph and cut into contiguous, equally sized
ranges (on a channel these are slabs across it, with a short cut).  Each part
is stepped by its own handle over its owned cells plus the halo: every cell
outside the part that shares a slot with an owned cell.  A halo slot that
leads out of the part becomes a wall (KLAS 4); what the halo cells compute
with it is overwritten, because after every step each halo cell takes the
state its owner computed (``hb_halo_pack`` / ``hb_halo_unpack`` on the
device, and between GPUs a ``torch.distributed`` send/receive of the packed
records).

An owned cell's fluxes need only its own state and its neighbours' (one
ring), so every owned cell computes the same operations on the same inputs as
in the whole mesh: the split run is bit-identical to the single-handle run.

The reference steps one mesh on one GPU and has no counterpart of this.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Callable, Dict, List, Optional

import numpy as np

from . import _lib
from ._lib import check, lib

CELL_ARRAYS = ("zbc", "zb1", "area", "fnc", "bfeat")
SLOT_ARRAYS = ("nac", "klas", "side", "cosf", "sinf", "slcos", "slsin")
DAY_ARRAYS = ("qt", "dqt", "zt", "dzt")
KLAS_WALL = 4.0


def rcm_order(nac: np.ndarray) -> np.ndarray:
    """Reverse Cuthill-McKee order of the cells (``nac`` [4C], 1-based, 0 = none)."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    nb = np.asarray(nac).reshape(-1, 4).astype(np.int64) - 1
    C_ = nb.shape[0]
    rows = np.repeat(np.arange(C_), 4)
    cols = nb.reshape(-1)
    keep = cols >= 0
    g = csr_matrix((np.ones(int(keep.sum()), dtype=np.int8), (rows[keep], cols[keep])), shape=(C_, C_))
    return np.asarray(reverse_cuthill_mckee(g, symmetric_mode=True), dtype=np.int64)


@dataclasses.dataclass
class Part:
    """One part: its cells in the whole mesh's (reference) numbering.

    ``cells`` is the part's local numbering (owned and halo cells in
    increasing global order).  ``send[q]`` / ``recv[q]``: local indices of the
    owned cells that are halo cells of part q, and of this part's halo cells
    that part q owns, both in increasing global order, so that records sent
    by one part land on the matching cells of the other.
    """
    index: int
    owned: np.ndarray
    halo: np.ndarray
    cells: np.ndarray
    owned_local: np.ndarray
    send: Dict[int, np.ndarray]
    recv: Dict[int, np.ndarray]


def plan(nac: np.ndarray, nparts: int, order: Optional[np.ndarray] = None) -> List[Part]:
    """Split the cells into `nparts` parts of equal size (contiguous in `order`)."""
    nb = np.asarray(nac).reshape(-1, 4).astype(np.int64) - 1
    ncell = nb.shape[0]
    if nparts < 1 or nparts > ncell:
        raise ValueError(f"nparts must lie in 1..{ncell}")
    order = rcm_order(nac) if order is None else np.asarray(order, dtype=np.int64)
    owner = np.empty(ncell, dtype=np.int64)
    bounds = np.linspace(0, ncell, nparts + 1).round().astype(np.int64)
    for p in range(nparts):
        owner[order[bounds[p]:bounds[p + 1]]] = p
    parts = []
    for p in range(nparts):
        owned = np.sort(np.nonzero(owner == p)[0])
        ring = nb[owned].reshape(-1)
        ring = np.unique(ring[ring >= 0])
        halo = ring[owner[ring] != p]
        cells = np.union1d(owned, halo)
        local = np.searchsorted(cells, owned)
        recv = {}
        for q in np.unique(owner[halo]):
            recv[int(q)] = np.searchsorted(cells, halo[owner[halo] == q])
        parts.append(Part(p, owned, halo, cells, local, {}, recv))
    for p in parts:
        for q, idx in list(p.recv.items()):
            # what q sends to p: q's owned cells among p's halo, in global order
            g = p.cells[idx]
            parts[q].send[p.index] = np.searchsorted(parts[q].cells, g)
    return parts


def sub_arrays(arrays: Dict[str, np.ndarray], ncell: int, ndays: int, nhq: int, part: Part) -> Dict[str, np.ndarray]:
    """The part's mesh arrays (local numbering) from the whole mesh's.

    Slots that lead out of the part (halo cells only) become walls."""
    cells = part.cells
    n = len(cells)
    out: Dict[str, np.ndarray] = {}
    slots = (4 * cells[:, None] + np.arange(4)[None, :]).reshape(-1)
    for k in SLOT_ARRAYS:
        if k in arrays:
            out[k] = np.ascontiguousarray(np.asarray(arrays[k], dtype=np.float64)[slots])
    g = out["nac"].astype(np.int64) - 1
    pos = np.searchsorted(cells, np.where(g >= 0, g, 0))
    inside = (g >= 0) & (pos < n) & (cells[np.minimum(pos, n - 1)] == np.where(g >= 0, g, -1))
    out["nac"] = np.where(inside, pos + 1, 0).astype(np.float64)
    cut = (g >= 0) & ~inside
    out["klas"] = np.where(cut, KLAS_WALL, out["klas"])
    for k in CELL_ARRAYS + ("h", "u", "v", "z", "w"):
        if k in arrays:
            out[k] = np.ascontiguousarray(np.asarray(arrays[k])[cells])
    if "nhq1" in arrays:
        out["nhq1"] = np.ascontiguousarray(np.asarray(arrays["nhq1"], dtype=np.int32)[cells])
    for k in DAY_ARRAYS:
        if k in arrays:
            a = np.asarray(arrays[k], dtype=np.float64).reshape(ndays, ncell)
            out[k] = np.ascontiguousarray(a[:, cells].reshape(-1))
    for k in ("zw", "qw"):
        if k in arrays:
            a = np.asarray(arrays[k], dtype=np.float64).reshape(ncell, max(nhq, 0))
            out[k] = np.ascontiguousarray(a[cells].reshape(-1))
    for k in ("f0", "f1", "f2", "f3"):
        if k in arrays:
            out[k] = np.ascontiguousarray(np.asarray(arrays[k], dtype=np.float64)[slots])
    return out


def deck_arrays(deck) -> Dict[str, np.ndarray]:
    """Copies of every mesh array of a ``hydrob200.Deck``, with its initial state."""
    names = SLOT_ARRAYS + CELL_ARRAYS + DAY_ARRAYS + ("zw", "qw", "nhq1")
    out = {k: np.array(deck.array(k)) for k in names}
    st = deck.state()
    for k in "HUVZW":
        out[k.lower()] = st[k].copy()
    return out


class SubDeck:
    """A part's mesh in the form ``hydrob200.Solver`` takes (``mesh``, ``cells``, ``state()``)."""

    def __init__(self, whole_mesh: _lib.MeshDesc, arrays: Dict[str, np.ndarray]):
        self._arrays = arrays
        m = _lib.MeshDesc()
        for f in ("ndays", "nhq", "steps_per_day", "dt", "hm1", "hm2", "jl"):
            setattr(m, f, getattr(whole_mesh, f))
        m.cells = len(arrays["zbc"])
        for k in SLOT_ARRAYS + CELL_ARRAYS + DAY_ARRAYS + ("zw", "qw"):
            setattr(m, k, arrays[k].ctypes.data_as(_lib._dp))
        m.nhq1 = arrays["nhq1"].ctypes.data_as(_lib._ip)
        self.mesh = m
        self.cells = m.cells

    def state(self) -> Dict[str, np.ndarray]:
        return {k: self._arrays[k.lower()] for k in "HUVZW"}


class PartSolver:
    """A part on one GPU: a ``hydrob200.Solver`` over the part's mesh and its
    halo lists.  ``pack(q)`` returns the records part q's halo needs from
    this part (a CUDA tensor); ``unpack(q, records)`` writes q's records into
    this part's halo."""

    def __init__(self, part: Part, sub: SubDeck, device: int = 0, **solver_kw):
        import torch
        from .solver import Solver
        self.part = part
        self.solver = Solver(sub, device=device, **solver_kw)
        self.device = torch.device("cuda", device)
        rb = C.c_int32()
        check(lib().hb_state_record_bytes(self.solver._h, C.byref(rb)))
        self.dtype = torch.float64 if rb.value == 32 else torch.float32
        self._ids: Dict[str, int] = {}
        self._buf: Dict[str, "torch.Tensor"] = {}
        for kind, lists in (("send", part.send), ("recv", part.recv)):
            for q, idx in lists.items():
                cells = np.ascontiguousarray(idx, dtype=np.int32)
                lid = C.c_int32()
                check(lib().hb_halo_define(self.solver._h, cells.ctypes.data_as(_lib._ip), len(cells), C.byref(lid)))
                self._ids[f"{kind}{q}"] = lid.value
                self._buf[f"{kind}{q}"] = torch.empty((max(len(cells), 1), 4), dtype=self.dtype, device=self.device)

    def _stream(self):
        import torch
        return torch.cuda.current_stream(self.device).cuda_stream

    def step(self, n: int) -> None:
        self.solver.step(n, self._stream())

    def pack(self, q: int):
        key = f"send{q}"
        buf = self._buf[key]
        check(lib().hb_halo_pack(self.solver._h, self._ids[key], C.c_void_p(buf.data_ptr()), C.c_void_p(self._stream())))
        return buf[: len(self.part.send[q])]

    def recv_buffer(self, q: int):
        return self._buf[f"recv{q}"][: len(self.part.recv[q])]

    def unpack(self, q: int, records) -> None:
        key = f"recv{q}"
        if records.data_ptr() % 16:
            records = records.clone()
        check(lib().hb_halo_unpack(self.solver._h, self._ids[key], C.c_void_p(records.data_ptr()),
                                   C.c_void_p(self._stream())))

    def owned_state(self) -> Dict[str, np.ndarray]:
        st = self.solver.get_state()
        return {k: st[k][self.part.owned_local] for k in "HUVZ"}

    def close(self) -> None:
        self.solver.close()


class HaloRun:
    """A mesh split into `nparts` parts, stepped with a halo exchange after every step.

    world = 1: every part in this process (on `device`), the exchange a
    device-to-device copy.  world = nparts: part r on rank r, the exchange a
    ``torch.distributed`` send/receive per neighbouring part (NCCL for CUDA
    records, gloo for CPU ones).  ``make(part, arrays)`` builds a part's
    stepper (default: ``PartSolver`` on the GPU); a stepper offers step(n),
    pack(q), recv_buffer(q), unpack(q, records) and owned_state().
    """

    def __init__(self, arrays: Dict[str, np.ndarray], scalars: Dict[str, int], nparts: int,
                 make: Callable[[Part, Dict[str, np.ndarray]], object], rank: int = 0, world: int = 1, group=None,
                 order: Optional[np.ndarray] = None):
        if world not in (1, nparts):
            raise ValueError("world must be 1 (all parts here) or nparts (one part per rank)")
        self.ncell = len(arrays["zbc"])
        self.parts = plan(arrays["nac"], nparts, order)
        self.rank, self.world, self.group = rank, world, group
        self.mine = list(range(nparts)) if world == 1 else [rank]
        self.steppers = {p: make(self.parts[p], sub_arrays(arrays, self.ncell, scalars["ndays"], scalars["nhq"],
                                                           self.parts[p]))
                         for p in self.mine}

    def step(self, n: int = 1) -> None:
        for _ in range(n):
            for p in self.mine:
                self.steppers[p].step(1)
            self.exchange()

    def exchange(self) -> None:
        if self.world == 1:
            # every part packs first, then every part unpacks (packs read owned
            # cells, unpacks write halo cells: the order does not matter)
            out = {(p, q): self.steppers[p].pack(q) for p in self.mine for q in self.parts[p].send}
            for (p, q), rec in out.items():
                self.steppers[q].unpack(p, rec)
            return
        import torch.distributed as dist
        p = self.rank
        st = self.steppers[p]
        ops = []
        for q in sorted(set(self.parts[p].send) | set(self.parts[p].recv)):
            if q in self.parts[p].send:
                ops.append(dist.P2POp(dist.isend, st.pack(q), q, self.group))
            if q in self.parts[p].recv:
                ops.append(dist.P2POp(dist.irecv, st.recv_buffer(q), q, self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for q in sorted(self.parts[p].recv):
            st.unpack(q, st.recv_buffer(q))

    def gather(self) -> Optional[Dict[str, np.ndarray]]:
        """The whole mesh's state {H, U, V, Z} (reference order) on rank 0, None elsewhere."""
        local = {p: (self.parts[p].owned, self.steppers[p].owned_state()) for p in self.mine}
        if self.world > 1:
            import torch.distributed as dist
            got = [None] * self.world if self.rank == 0 else None
            dist.gather_object(local, got, dst=0, group=self.group)
            if self.rank != 0:
                return None
            local = {k: v for d in got for k, v in d.items()}
        out = {k: np.empty(self.ncell) for k in "HUVZ"}
        for owned, st in local.values():
            for k in "HUVZ":
                out[k][owned] = st[k]
        return out

    def close(self) -> None:
        for s in self.steppers.values():
            if hasattr(s, "close"):
                s.close()


def split_deck(deck, nparts: int, rank: int = 0, world: int = 1, group=None, device: int = 0,
               **solver_kw) -> HaloRun:
    """A ``hydrob200.Deck`` split into `nparts` GPU parts (``PartSolver``)."""
    arrays = deck_arrays(deck)
    m = deck.mesh

    def make(part, sub):
        return PartSolver(part, SubDeck(m, sub), device=device, **solver_kw)

    return HaloRun(arrays, {"ndays": m.ndays, "nhq": m.nhq}, nparts, make, rank, world, group)
