"""Seeded synthetic hydro-cal decks.

Builds unstructured channel meshes and writes them in the reference's text
deck layout, so the reference binaries and this library read byte-identical
inputs.

Deck layout (native reader, ``cuda_native_impl/hydro-cal-src/src/mesh.cpp:5-38``)::

    BINFOR/{TIME,GIRD,DEPTH,BOUNDARY,CALTIME,JL,INITIALLEVEL,INITIALU1,INITIALV1,CV}.DAT
    SOURCES/{PNAC,PNAP,PKLAS,PZBC,PXY,MBZ,MBQ,MBW,MBZQ}.DAT
    BOUNDE/{NZ/NZ%04d,NQ/NQ%04d,NZQ/NZQ%04d}.DAT

The CPU solver (``hydro-cal-fortan/calculate.cpp:1135-1160``,
``read_data.hh:37-51``) reads the same files with the BINFOR files at the deck
root; :func:`write_cpu_solver_deck` writes that variant.

Mesh conventions follow ``mesh.cpp:297-337``: cell nodes counter-clockwise,
slot ``j`` is the edge from node ``j`` to node ``j+1`` (outward normal
``(COSF, SINF) = (dy, -dx)/L``), a triangle stores ``NAP[3] = 0`` and its
fourth slot is a zero-length edge with ``NAC = KLAS = 0``.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

KLAS_WALL = 4
KLAS_INFLOW = 10      # given discharge (functors.cu:204-232)
KLAS_LEVEL = 1        # given water level (functors.cu:371-392)
KLAS_RATING = 3       # rating curve (functors.cu:320-369)
KLAS_OPEN = 5         # open boundary (functors.cu:551-557)
KLAS_WEIR = 6         # weir overflow (functors.cu:258-318)
KLAS_BREACH = 7       # levee breach (functors.cu:234-256)


@dataclasses.dataclass
class Series:
    """One boundary time series file: ``N`` then ``N`` lines ``time value``."""
    times: np.ndarray
    values: np.ndarray


@dataclasses.dataclass
class Deck:
    """Everything a hydro-cal deck holds, in the reference's (1-based) terms."""
    name: str
    xy: np.ndarray                 # [NOD, 2] node coordinates
    nap: np.ndarray                # [CELL, 4] 1-based node ids, 0 for the missing 4th node
    nac: np.ndarray                # [CELL, 4] 1-based neighbour ids, 0 = none
    klas: np.ndarray               # [CELL, 4] boundary codes
    zbc: np.ndarray                # [CELL] bed elevation
    z0: np.ndarray                 # [CELL] initial water level (INITIALLEVEL)
    u0: np.ndarray                 # [CELL]
    v0: np.ndarray                 # [CELL]
    manning: np.ndarray            # [CELL] Manning n (CV.DAT)
    mdt: int = 3600                # seconds per boundary-table interval ("day")
    ndays: int = 1
    ntoutput: int = 1
    dt: float = 1.0
    hm1: float = 0.001
    hm2: float = 0.01
    jl: float = 0.0
    nhq: int = 5
    ndi: int = 0
    # boundary groups: lists of (cell 1-based, group 1-based)
    mbq: List[Tuple[int, int]] = dataclasses.field(default_factory=list)
    mbz: List[Tuple[int, int]] = dataclasses.field(default_factory=list)
    mbzq: List[Tuple[int, int]] = dataclasses.field(default_factory=list)
    mbw: List[Tuple[int, float]] = dataclasses.field(default_factory=list)
    nq_series: List[Series] = dataclasses.field(default_factory=list)
    nz_series: List[Series] = dataclasses.field(default_factory=list)
    nzq_tables: List[Series] = dataclasses.field(default_factory=list)  # (Z, Q) pairs
    meta: Dict[str, object] = dataclasses.field(default_factory=dict)

    @property
    def cells(self) -> int:
        return int(self.nap.shape[0])

    @property
    def nodes(self) -> int:
        return int(self.xy.shape[0])

    @property
    def steps_per_day(self) -> int:
        return int(self.mdt / self.dt)


# ---------------------------------------------------------------------------
# topology
# ---------------------------------------------------------------------------

def orient_ccw(xy: np.ndarray, tris: np.ndarray) -> np.ndarray:
    """Return triangles with counter-clockwise node order."""
    p0, p1, p2 = xy[tris[:, 0]], xy[tris[:, 1]], xy[tris[:, 2]]
    cross = (p1[:, 0] - p0[:, 0]) * (p2[:, 1] - p0[:, 1]) - (p1[:, 1] - p0[:, 1]) * (p2[:, 0] - p0[:, 0])
    out = tris.copy()
    cw = cross < 0
    out[cw, 1], out[cw, 2] = tris[cw, 2], tris[cw, 1]
    return out


def build_neighbours(nap0: np.ndarray) -> np.ndarray:
    """Neighbour across each slot for 0-based node lists ``nap0`` [CELL,4] (-1 = no 4th node).

    Returns 1-based ``NAC`` (0 = boundary / degenerate slot), matching how the
    reference decks store it (``mesh.cpp:40-58``).
    """
    ncell = nap0.shape[0]
    nv = np.where(nap0[:, 3] < 0, 3, 4)
    a_list, b_list, cell_list, slot_list = [], [], [], []
    for j in range(4):
        valid = j < nv
        a = nap0[:, j]
        b = np.where(nv == 3, nap0[:, (j + 1) % 3], nap0[:, (j + 1) % 4])
        idx = np.nonzero(valid)[0]
        a_list.append(a[idx]); b_list.append(b[idx])
        cell_list.append(idx); slot_list.append(np.full(idx.shape, j))
    a = np.concatenate(a_list); b = np.concatenate(b_list)
    cell = np.concatenate(cell_list); slot = np.concatenate(slot_list)
    lo = np.minimum(a, b).astype(np.int64); hi = np.maximum(a, b).astype(np.int64)
    key = lo * (int(hi.max()) + 1) + hi
    order = np.argsort(key, kind="stable")
    ks = key[order]
    nac = np.zeros((ncell, 4), dtype=np.int64)
    same = np.nonzero(ks[1:] == ks[:-1])[0]
    if same.size:
        # each interior edge appears exactly twice
        triple = np.nonzero((ks[2:] == ks[:-2]))[0]
        if triple.size:
            raise ValueError("non-manifold mesh: an edge is shared by more than two cells")
        i0 = order[same]; i1 = order[same + 1]
        nac[cell[i0], slot[i0]] = cell[i1] + 1
        nac[cell[i1], slot[i1]] = cell[i0] + 1
    return nac


def _grid_counts(ncells: int, lx: float, ly: float) -> Tuple[int, int]:
    """Quad counts (mx, my) with 2*mx*my >= ncells and mx/my close to lx/ly."""
    half = ncells / 2.0
    my = max(2, int(round(math.sqrt(half * ly / lx))))
    mx = int(math.ceil(half / my))
    return mx, my


def delaunay_channel(ncells: int, lx: float, ly: float, seed: int, jitter: float = 0.3):
    """Delaunay triangulation of seeded jittered points on an ``lx`` x ``ly`` rectangle.

    Points start on a regular (mx+1) x (my+1) lattice; interior points are
    jittered in both directions, boundary points only along their side. The
    triangle count of a planar point set is ``2N - B - 2`` (N points, B on the
    hull), so the lattice is trimmed to the exact count: one boundary point
    is dropped when the surplus is odd, then surplus/2 interior points.
    """
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    mx, my = _grid_counts(ncells, lx, ly)
    hx, hy = lx / mx, ly / my
    ii, jj = np.meshgrid(np.arange(mx + 1), np.arange(my + 1), indexing="ij")
    ii = ii.ravel(); jj = jj.ravel()
    x = ii * hx; y = jj * hy
    on_x = (ii == 0) | (ii == mx)
    on_y = (jj == 0) | (jj == my)
    interior = ~(on_x | on_y)
    jx = rng.uniform(-jitter, jitter, x.shape) * hx
    jy = rng.uniform(-jitter, jitter, y.shape) * hy
    x = x + np.where(interior | (on_y & ~on_x), jx, 0.0)
    y = y + np.where(interior | (on_x & ~on_y), jy, 0.0)
    keep = np.ones(x.shape, dtype=bool)
    surplus = 2 * mx * my - ncells
    if surplus < 0:
        raise ValueError("lattice too small")
    if surplus % 2 == 1:
        # drop one non-corner point of the y = 0 side
        cand = np.nonzero((jj == 0) & (ii > 0) & (ii < mx))[0]
        keep[cand[len(cand) // 2]] = False
        surplus -= 1
    if surplus:
        cand = np.nonzero(interior)[0]
        # spread the removed points out: never two lattice neighbours
        chosen: List[int] = []
        taken = set()
        perm = rng.permutation(cand)
        for p in perm:
            pi, pj = int(ii[p]), int(jj[p])
            if any((pi + di, pj + dj) in taken for di in (-1, 0, 1) for dj in (-1, 0, 1)):
                continue
            chosen.append(int(p)); taken.add((pi, pj))
            if len(chosen) == surplus // 2:
                break
        if len(chosen) != surplus // 2:
            raise ValueError("could not trim lattice to the requested cell count")
        keep[np.array(chosen)] = False
    xy = np.stack([x[keep], y[keep]], axis=1)
    tri = Delaunay(xy)
    tris = tri.simplices.astype(np.int64)
    if tris.shape[0] != ncells:
        raise ValueError(f"Delaunay gave {tris.shape[0]} triangles, wanted {ncells}")
    if np.unique(tris).size != xy.shape[0]:
        raise ValueError("Delaunay dropped input points")
    tris = orient_ccw(xy, tris)
    # a column sweep numbering, like a mesh generator's front order
    cen = xy[tris].mean(axis=1)
    col = np.floor(cen[:, 0] / hx).astype(np.int64)
    order = np.lexsort((cen[:, 1], col))
    tris = tris[order]
    return xy, tris, (hx, hy)


def _bed_bumps(cx, cy, centres, amp, width):
    z = np.zeros_like(cx)
    for (bx, by) in centres:
        r2 = (cx - bx) ** 2 + (cy - by) ** 2
        z += amp * np.exp(-r2 / (2.0 * width * width))
    return z


def _assemble(name, xy, cells_nodes, nv3):
    """cells_nodes: [C,4] 0-based (col 3 = -1 for triangles)."""
    nac = build_neighbours(cells_nodes)
    nap = cells_nodes + 1
    nap[nv3, 3] = 0
    return nap, nac


def _boundary_slots(nac: np.ndarray, nap: np.ndarray):
    """(cell, slot) of every real slot without a neighbour (0-based)."""
    nv = np.where(nap[:, 3] == 0, 3, 4)
    cells, slots = np.nonzero(nac == 0)
    real = slots < nv[cells]
    return cells[real], slots[real]


def _slot_midpoints(xy, nap, cells, slots):
    nv = np.where(nap[:, 3] == 0, 3, 4)
    a = nap[cells, slots] - 1
    b = nap[cells, (slots + 1) % nv[cells]] - 1
    return 0.5 * (xy[a] + xy[b])


def channel_deck(name: str, ncells: int, lx: float, ly: float, seed: int, *,
                 slope: float = 1e-4, z0: float = 0.05, depth: float = 2.0,
                 bump_amp: float = 0.5, bump_width: float = 300.0, nbumps: int = 3,
                 q_in: float = 100.0, hydrograph: Optional[Tuple[float, float, float]] = None,
                 n_manning: float = 0.025, n_field: Optional[np.ndarray] = None,
                 dt: float = 1.0, steps: int = 100, mdt: Optional[int] = None,
                 hm1: float = 0.001, hm2: float = 0.01, zero_q_edges: int = 8) -> Deck:
    """The channel scenario family of the benchmark configurations.

    Bed ``ZBC = z0 + slope*(lx - x) + sum of Gaussian bumps`` at cell
    centroids. The initial level is ``depth`` above the inclined datum plane
    ``z0 + slope*(lx - x)``; the reference sets ``H = max(level - ZBC, HM1)``
    (``mesh.cpp:350-361``). Long sides are walls (KLAS 4), the x = 0 side is a
    KLAS 10 discharge inflow (constant ``q_in`` or a Gaussian hydrograph
    ``(peak, t_peak_s, sigma_s)``), the x = lx side a KLAS 1 fixed level, and
    ``zero_q_edges`` wall edges become KLAS 10 edges with zero discharge.
    """
    rng = np.random.default_rng(seed + 1_000_003)
    xy, tris, (hx, hy) = delaunay_channel(ncells, lx, ly, seed)
    nodes4 = np.concatenate([tris, -np.ones((tris.shape[0], 1), dtype=np.int64)], axis=1)
    nv3 = np.ones(tris.shape[0], dtype=bool)
    nap, nac = _assemble(name, xy, nodes4, nv3)
    cen = xy[tris].mean(axis=1)
    centres = [(rng.uniform(0.2 * lx, 0.8 * lx), rng.uniform(0.25 * ly, 0.75 * ly)) for _ in range(nbumps)]
    plane = z0 + slope * (lx - cen[:, 0])
    zbc = plane + _bed_bumps(cen[:, 0], cen[:, 1], centres, bump_amp, bump_width)
    level = plane + depth
    klas = np.zeros_like(nac)
    bc, bs = _boundary_slots(nac, nap)
    mid = _slot_midpoints(xy, nap, bc, bs)
    tol = 1e-6 * max(lx, ly)
    at_in = mid[:, 0] < tol
    at_out = mid[:, 0] > lx - tol
    klas[bc, bs] = KLAS_WALL
    klas[bc[at_in], bs[at_in]] = KLAS_INFLOW
    klas[bc[at_out], bs[at_out]] = KLAS_LEVEL
    # one boundary slot per cell for the zero-discharge edges
    wall_idx = np.nonzero(~at_in & ~at_out)[0]
    nb_per_cell = np.bincount(bc, minlength=nac.shape[0])
    wall_idx = wall_idx[nb_per_cell[bc[wall_idx]] == 1]
    zq = rng.choice(wall_idx, size=min(zero_q_edges, wall_idx.size), replace=False)
    zq = np.sort(zq)
    klas[bc[zq], bs[zq]] = KLAS_INFLOW

    if mdt is None:
        mdt = int(round(3600 * dt)) if dt >= 1 else 3600
    spd = int(mdt / dt)
    ndays = max(1, int(math.ceil(steps / max(1, spd - 1))) + 1)
    t_unit = mdt / 86400.0               # one table interval, in BOUNDRYinterp time units
    t_end = (ndays + 1) * t_unit * 2.0 + 1.0
    in_cells = sorted(set((bc[at_in] + 1).tolist()))
    zq_cells = sorted(set((bc[zq] + 1).tolist()))
    out_cells = sorted(set((bc[at_out] + 1).tolist()))
    mbq = [(c, 1) for c in in_cells] + [(c, 2) for c in zq_cells]
    mbz = [(c, 1) for c in out_cells]
    if hydrograph is None:
        q_series = Series(np.array([0.0, t_end]), np.array([q_in, q_in]))
    else:
        peak, t_peak, sigma = hydrograph
        ts = np.linspace(0.0, t_end, 257)
        secs = ts / t_unit * mdt
        base = 0.1 * peak
        q_series = Series(ts, base + (peak - base) * np.exp(-0.5 * ((secs - t_peak) / sigma) ** 2))
    zero_series = Series(np.array([0.0, t_end]), np.array([0.0, 0.0]))
    z_out = z0 + depth
    z_series = Series(np.array([0.0, t_end]), np.array([z_out, z_out]))
    manning = np.full(nac.shape[0], n_manning) if n_field is None else np.asarray(n_field, dtype=np.float64)
    deck = Deck(name=name, xy=xy, nap=nap, nac=nac, klas=klas, zbc=zbc, z0=level,
                u0=np.zeros(nac.shape[0]), v0=np.zeros(nac.shape[0]), manning=manning,
                mdt=mdt, ndays=ndays, dt=dt, hm1=hm1, hm2=hm2,
                mbq=mbq, mbz=mbz, nq_series=[q_series, zero_series], nz_series=[z_series],
                meta=dict(seed=seed, ncells=ncells, lx=lx, ly=ly, hx=hx, hy=hy, bumps=centres,
                          steps=steps))
    return deck


def stress_deck(name: str, mx: int, my: int, seed: int, *, dt: float = 1.0, steps: int = 50,
                mdt: int = 60, hm1: float = 0.001, hm2: float = 0.01, jl: float = 0.3,
                with_breach: bool = False, with_unknown: bool = True) -> Deck:
    """A small mixed quad/triangle deck that reaches every branch of the flux chain.

    A jittered ``mx`` x ``my`` lattice; a seeded half of the quads is split
    into two triangles. The bed is rough with a dry ridge, a shallow shelf and
    a fast jet, so dry, shallow, supercritical and Osher branches all occur.
    Boundary slots cycle through KLAS 4, 10, 1, 3, 5 (and the unknown code 13
    that only writes FLUX2); an interior weir (KLAS 6 on both sides), an
    interior code 9 pair (mirror Osher from the lower-numbered side) and,
    optionally, breach edges (KLAS 7) are placed inside.
    """
    rng = np.random.default_rng(seed)
    lx, ly = 50.0 * mx, 50.0 * my
    hx, hy = lx / mx, ly / my
    ii, jj = np.meshgrid(np.arange(mx + 1), np.arange(my + 1), indexing="ij")
    x = ii * hx; y = jj * hy
    inner = (ii > 0) & (ii < mx) & (jj > 0) & (jj < my)
    x = x + np.where(inner, rng.uniform(-0.2, 0.2, x.shape) * hx, 0.0)
    y = y + np.where(inner, rng.uniform(-0.2, 0.2, y.shape) * hy, 0.0)
    xy = np.stack([x.ravel(), y.ravel()], axis=1)
    nid = lambda i, j: i * (my + 1) + j
    cells = []
    for i in range(mx):
        for j in range(my):
            a, b, c, d = nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)
            if rng.uniform() < 0.5:
                cells.append([a, b, c, d])
            elif rng.uniform() < 0.5:
                cells.append([a, b, c, -1]); cells.append([a, c, d, -1])
            else:
                cells.append([a, b, d, -1]); cells.append([b, c, d, -1])
    nodes4 = np.array(cells, dtype=np.int64)
    perm = rng.permutation(nodes4.shape[0])        # scattered numbering
    nodes4 = nodes4[perm]
    nv3 = nodes4[:, 3] < 0
    nap, nac = _assemble(name, xy, nodes4, nv3)
    nv = np.where(nv3, 3, 4)
    cen = np.array([xy[r[:k]].mean(axis=0) for r, k in zip(nodes4, nv)])
    # rough bed: tilted plane + noise + a ridge that stays dry + a deep pool
    zbc = 1.0 + 0.002 * (lx - cen[:, 0]) + rng.uniform(-0.05, 0.05, cen.shape[0])
    ridge = np.abs(cen[:, 0] - 0.55 * lx) < 0.6 * hx
    zbc = zbc + np.where(ridge & (cen[:, 1] > 0.5 * ly), 3.0, 0.0)
    level = np.full(cen.shape[0], 1.0 + 0.002 * lx * 0.5 + 0.8)
    # left third deeper (dam-break like), a shelf with a few mm of water
    level = np.where(cen[:, 0] < 0.3 * lx, level + 1.5, level)
    shelf = (cen[:, 0] > 0.7 * lx) & (cen[:, 1] < 0.3 * ly)
    level = np.where(shelf, zbc + rng.uniform(0.0, 0.012, cen.shape[0]), level)
    dry = (cen[:, 0] > 0.8 * lx) & (cen[:, 1] > 0.7 * ly)
    level = np.where(dry, zbc - 0.1, level)
    u0 = np.where(cen[:, 0] < 0.3 * lx, 2.5, 0.3) + rng.uniform(-0.2, 0.2, cen.shape[0])
    v0 = rng.uniform(-0.3, 0.3, cen.shape[0])
    jet = (cen[:, 1] > 0.45 * ly) & (cen[:, 1] < 0.55 * ly) & (cen[:, 0] < 0.3 * lx)
    u0 = np.where(jet, 9.0, u0)
    klas = np.zeros_like(nac)
    bc, bs = _boundary_slots(nac, nap)
    mid = _slot_midpoints(xy, nap, bc, bs)
    tol = 1e-6 * lx
    left = mid[:, 0] < tol; right = mid[:, 0] > lx - tol
    bottom = mid[:, 1] < tol; top = mid[:, 1] > ly - tol
    klas[bc, bs] = KLAS_WALL
    klas[bc[left], bs[left]] = KLAS_INFLOW
    # right side: alternate level / rating / open; one cell per boundary slot there
    ridx = np.nonzero(right & ~bottom & ~top)[0]
    ridx = ridx[np.argsort(mid[ridx, 1])]
    codes = [KLAS_LEVEL, KLAS_RATING, KLAS_OPEN]
    for k, r in enumerate(ridx):
        klas[bc[r], bs[r]] = codes[k % 3]
    if with_unknown:
        tidx = np.nonzero(top & ~left & ~right)[0]
        for r in tidx[::5]:
            klas[bc[r], bs[r]] = 13
    # interior special pairs
    nb_cells, nb_slots = np.nonzero((nac > 0))
    def pick_pair(exclude):
        while True:
            k = int(rng.integers(nb_cells.size))
            c, s = int(nb_cells[k]), int(nb_slots[k])
            o = int(nac[c, s]) - 1
            os_ = int(np.nonzero(nac[o] == c + 1)[0][0])
            if klas[c, s] == 0 and klas[o, os_] == 0 and c not in exclude and o not in exclude:
                return c, s, o, os_
    used = set()
    weirs = []
    for _ in range(4):
        c, s, o, os_ = pick_pair(used)
        klas[c, s] = KLAS_WEIR; klas[o, os_] = KLAS_WEIR
        used.update([c, o]); weirs.append((c, o))
    for _ in range(3):
        c, s, o, os_ = pick_pair(used)
        lo_c, lo_s = (c, s) if c < o else (o, os_)
        klas[lo_c, lo_s] = 9          # non-boundary non-zero code
        used.update([c, o])
    if with_breach:
        for _ in range(2):
            c, s, o, os_ = pick_pair(used)
            klas[c, s] = KLAS_BREACH; klas[o, os_] = KLAS_BREACH
            used.update([c, o])
    mbw = []
    for (c, o) in weirs:
        top_w = max(zbc[c], zbc[o]) + rng.uniform(0.2, 1.5)
        mbw.append((c + 1, float(top_w))); mbw.append((o + 1, float(top_w)))
    ndays = int(math.ceil(steps / (int(mdt / dt) - 1))) + 2
    t_unit = mdt / 86400.0
    t_end = (ndays + 1) * t_unit * 2 + 1.0
    ts = np.linspace(0.0, t_end, 33)
    in_cells = sorted(set((bc[left] + 1).tolist()))
    mbq = [(c, 1 + (k % 2)) for k, c in enumerate(in_cells)]
    q1 = Series(ts, 20.0 + 15.0 * np.sin(ts / t_unit * 0.3))
    q2 = Series(ts, 5.0 + 3.0 * np.cos(ts / t_unit * 0.2))
    lvl_cells = sorted(set(int(bc[r]) + 1 for k, r in enumerate(ridx) if k % 3 == 0))
    mbz = [(c, 1) for c in lvl_cells]
    z1 = Series(ts, 2.3 + 0.4 * np.sin(ts / t_unit * 0.25))
    rat_cells = sorted(set(int(bc[r]) + 1 for k, r in enumerate(ridx) if k % 3 == 1))
    mbzq = [(c, 1) for c in rat_cells]
    zq = Series(np.array([1.0, 1.5, 2.0, 2.5, 3.0]), np.array([0.0, 5.0, 20.0, 45.0, 80.0]))
    manning = rng.uniform(0.015, 0.04, nac.shape[0])
    return Deck(name=name, xy=xy, nap=nap, nac=nac, klas=klas, zbc=zbc, z0=level, u0=u0, v0=v0,
                manning=manning, mdt=mdt, ndays=ndays, dt=dt, hm1=hm1, hm2=hm2, jl=jl, nhq=5,
                mbq=mbq, mbz=mbz, mbzq=mbzq, mbw=mbw, nq_series=[q1, q2], nz_series=[z1],
                nzq_tables=[zq], meta=dict(seed=seed, mx=mx, my=my, steps=steps))


def probe_deck(name: str, seed: int = 31, mx: int = 20, my: int = 40, steps: int = 60, mdt: int = 20) -> Deck:
    """A stress deck whose boundary tables jump by orders of magnitude between
    table intervals, so that ``QT + DQT*kt`` and ``ZT + DZT*jt`` (functors.cu:209,
    :376) are dominated by the product term and their rounding becomes visible
    in the fluxes; also more rating-curve (KLAS 3) and weir (KLAS 6) slots."""
    d = stress_deck(name, mx, my, seed, steps=steps, mdt=mdt, jl=0.2)
    rng = np.random.default_rng(seed + 7)
    t_unit = mdt / 86400.0
    nd = d.ndays + 2
    ts = np.arange(nd + 2) * t_unit
    ts[-1] = (d.ndays + 1) * t_unit * 2 + 1.0
    q_lo, q_hi = rng.uniform(0.01, 0.2, ts.size), rng.uniform(20.0, 80.0, ts.size)
    qa = np.where(np.arange(ts.size) % 2 == 0, q_lo, q_hi)
    qb = np.where(np.arange(ts.size) % 2 == 1, q_lo * 3.0, q_hi * 0.7)
    d.nq_series = [Series(ts, qa), Series(ts, qb)]
    zlo = 1.6 + rng.uniform(0.0, 0.1, ts.size)
    zhi = 2.4 + rng.uniform(0.0, 0.6, ts.size)
    d.nz_series = [Series(ts, np.where(np.arange(ts.size) % 2 == 0, zlo, zhi))]
    # every right-side slot alternates 1 / 3 (no open slots), so more rating-curve cells
    nv = np.where(d.nap[:, 3] == 0, 3, 4)
    bc, bs = _boundary_slots(d.nac, d.nap)
    mid = _slot_midpoints(d.xy, d.nap, bc, bs)
    lx = d.xy[:, 0].max()
    right = np.nonzero(mid[:, 0] > lx * (1 - 1e-9))[0]
    right = right[np.argsort(mid[right, 1])]
    lvl, rat = [], []
    for k, r in enumerate(right):
        code = KLAS_LEVEL if k % 2 == 0 else KLAS_RATING
        d.klas[bc[r], bs[r]] = code
        (lvl if code == KLAS_LEVEL else rat).append(int(bc[r]) + 1)
    d.mbz = [(c, 1) for c in sorted(set(lvl))]
    d.mbzq = [(c, 1) for c in sorted(set(rat) - set(lvl))]
    cx = np.array([d.xy[r[:k] - 1].mean(axis=0)[0] for r, k in zip(d.nap, np.where(d.nap[:, 3] == 0, 3, 4))])
    deep = cx > 0.85 * lx            # keep the cells at the level/rating boundary well wet
    d.z0 = np.where(deep, d.zbc + 1.2, d.z0)
    for (c, _) in d.mbzq:            # rating cells flowing outwards
        d.u0[c - 1] = rng.uniform(0.5, 2.0)
        d.v0[c - 1] = rng.uniform(-0.5, 0.5)
    d.nzq_tables = [Series(np.array([1.0, 1.4, 1.8, 2.4, 3.2]), np.array([0.0, 2.0, 9.0, 30.0, 90.0]))]
    del nv
    return d


# ---------------------------------------------------------------------------
# writers
# ---------------------------------------------------------------------------

def _fmt(v: float) -> str:
    return repr(float(v))


def _write_lines(path: str, lines: Sequence[str]) -> None:
    with open(path, "w") as f:
        f.write("\n".join(lines))
        f.write("\n")


def _write_per_cell4(path, arr):
    n = arr.shape[0]
    lines = [f"{n:12d}"]
    lines += [f"{i + 1:12d} {int(r[0]):10d} {int(r[1]):10d} {int(r[2]):10d} {int(r[3]):10d}" for i, r in enumerate(arr)]
    _write_lines(path, lines)


def _write_col(path, header, arr):
    _write_lines(path, [header] + [_fmt(v) for v in arr])


def _write_series(path, s: Series):
    _write_lines(path, [str(len(s.times))] + [f"{_fmt(t)} {_fmt(v)}" for t, v in zip(s.times, s.values)])


def write_deck(deck: Deck, root: str, *, cpu_solver_layout: bool = False) -> str:
    """Write ``deck`` under ``root``; returns ``root``.

    ``cpu_solver_layout`` puts the BINFOR files at the deck root, the layout
    ``hydro-cal-fortan/calculate.cpp:1135-1160`` reads.
    """
    binfor = root if cpu_solver_layout else os.path.join(root, "BINFOR")
    src = os.path.join(root, "SOURCES")
    for d in (binfor, src, os.path.join(root, "BOUNDE", "NQ"), os.path.join(root, "BOUNDE", "NZ"),
              os.path.join(root, "BOUNDE", "NZQ"), os.path.join(root, "OUTPUT")):
        os.makedirs(d, exist_ok=True)
    nz, nq, nzq = len(deck.mbz), len(deck.mbq), len(deck.mbzq)
    _write_lines(os.path.join(binfor, "TIME.DAT"), [f"{deck.mdt}        !PARAMETER (MDT)",
                                                    f"{deck.ndays}          !PARAMETER (NDAYS)",
                                                    f"{deck.ntoutput}"])
    _write_lines(os.path.join(binfor, "GIRD.DAT"), [f"{deck.nodes}        !PARAMETER (NOD)",
                                                    f"{deck.cells}        !PARAMETER (CEL)"])
    _write_lines(os.path.join(binfor, "DEPTH.DAT"), [f"{_fmt(deck.hm1)}        !PARAMETER (HM1)",
                                                     f"{_fmt(deck.hm2)}       !PARAMETER (HM2)"])
    _write_lines(os.path.join(binfor, "BOUNDARY.DAT"), [f"{nz}      !PARAMETER (NZ)",
                                                        f"{nq}        !PARAMETER (NQ)",
                                                        f"{nzq}        !PARAMETER (NZQ)",
                                                        f"{deck.nhq}        !PARAMETER (NHQ)",
                                                        f"{len(deck.mbw)}        !PARAMETER (NWE)",
                                                        f"{deck.ndi}        !PARAMETER (NDI)"])
    dt_txt = str(int(deck.dt)) if float(deck.dt).is_integer() else _fmt(deck.dt)
    _write_lines(os.path.join(binfor, "CALTIME.DAT"), ["0", dt_txt])
    _write_lines(os.path.join(binfor, "JL.DAT"), [_fmt(deck.jl)])
    _write_col(os.path.join(binfor, "INITIALLEVEL.DAT"), "Z1", deck.z0)
    _write_col(os.path.join(binfor, "INITIALU1.DAT"), "u1", deck.u0)
    _write_col(os.path.join(binfor, "INITIALV1.DAT"), "v1", deck.v0)
    _write_col(os.path.join(binfor, "CV.DAT"), "cv", deck.manning)
    _write_per_cell4(os.path.join(src, "PNAC.DAT"), deck.nac)
    _write_per_cell4(os.path.join(src, "PNAP.DAT"), deck.nap)
    _write_per_cell4(os.path.join(src, "PKLAS.DAT"), deck.klas)
    _write_col(os.path.join(src, "PZBC.DAT"), " PZBC", deck.zbc)
    _write_lines(os.path.join(src, "PXY.DAT"), [f"{deck.nodes:12d}"] +
                 [f"{i + 1:10d} {_fmt(p[0])} {_fmt(p[1])}" for i, p in enumerate(deck.xy)])
    _write_lines(os.path.join(src, "MBQ.DAT"), [str(len(deck.nq_series))] +
                 [f"{k + 1}\t{c}\t{g}" for k, (c, g) in enumerate(deck.mbq)])
    _write_lines(os.path.join(src, "MBZ.DAT"), [str(len(deck.nz_series))] +
                 [f"{k + 1}\t{c}\t{g}" for k, (c, g) in enumerate(deck.mbz)])
    _write_lines(os.path.join(src, "MBW.DAT"), [str(len(deck.mbw))] +
                 [f"{k + 1}\t{c}\t{_fmt(t)}" for k, (c, t) in enumerate(deck.mbw)])
    _write_lines(os.path.join(src, "MBZQ.DAT"), [str(len(deck.nzq_tables))] +
                 [f"{k + 1}\t{c}\t{g}" for k, (c, g) in enumerate(deck.mbzq)])
    for k, s in enumerate(deck.nq_series):
        _write_series(os.path.join(root, "BOUNDE", "NQ", f"NQ{k + 1:04d}.DAT"), s)
    for k, s in enumerate(deck.nz_series):
        _write_series(os.path.join(root, "BOUNDE", "NZ", f"NZ{k + 1:04d}.DAT"), s)
    for k, s in enumerate(deck.nzq_tables):
        _write_series(os.path.join(root, "BOUNDE", "NZQ", f"NZQ{k + 1:04d}.DAT"), s)
    return root


def write_cpu_solver_deck(deck: Deck, root: str, steps: int, open_boundaries: bool = False) -> str:
    """Deck for timing ``hydro-cal-fortan/calculate.cpp`` over ``steps`` steps.

    That solver runs every step of every table interval
    (``calculate.cpp:1163-1186``), so the deck is one interval of ``steps``
    steps. Its discharge/level table code is undefined behaviour for NQ > 0
    (``QZSTIME2`` never sized, ``calculate.cpp:1089-1096``) and indexes the
    ZT/QT tables transposed (``calculate.cpp:1165-1175``).  With
    ``open_boundaries`` the deck keeps the mesh's boundary codes and tables,
    for the solver built with the minimal patch of ``oracle/calc_patch.sed``;
    otherwise the open boundaries become walls (same mesh, same per-cell
    work, no tables) for the unpatched solver.
    """
    d = dataclasses.replace(deck)
    d.mdt = int(round(steps * deck.dt))
    d.ndays = 1
    if open_boundaries:
        write_deck(d, root, cpu_solver_layout=True)
        return root
    klas = deck.klas.copy()
    klas[(klas != 0)] = KLAS_WALL
    d.klas = klas
    d.mbq, d.mbz, d.mbzq, d.mbw = [], [], [], []
    d.nq_series, d.nz_series, d.nzq_tables = [], [], []
    d.mdt = int(round(steps * deck.dt))
    d.ndays = 1
    write_deck(d, root, cpu_solver_layout=True)
    return root


# ---------------------------------------------------------------------------
# named configurations
# ---------------------------------------------------------------------------

def config_f1(seed: int = 20240601, steps: int = 100) -> Deck:
    """6,675 Delaunay triangles on a 10 km x 2 km channel, Q = 100 m^3/s, dt = 1 s."""
    return channel_deck("F1_6675", 6675, 10_000.0, 2_000.0, seed, steps=steps)


def config_207k(seed: int = 20240602, steps: int = 900) -> Deck:
    """207,234 triangles on 40 km x 8 km, 1 m bumps, Gaussian hydrograph peaking at 400 m^3/s.

    One boundary-table interval is 60 s, so the hydrograph advances every
    59 steps as in the reference's day/step loop.
    """
    return channel_deck("C207K", 207_234, 40_000.0, 8_000.0, seed, bump_amp=1.0, bump_width=600.0,
                        hydrograph=(400.0, 450.0, 200.0), steps=steps, mdt=60)


def config_24k(seed: int = 20240603, steps: int = 1000, n_field: Optional[np.ndarray] = None) -> Deck:
    """24,020 triangles on 20 km x 4 km (the adjoint configuration)."""
    return channel_deck("C24K", 24_020, 20_000.0, 4_000.0, seed, steps=steps, mdt=60, n_field=n_field)


def ensemble_specs(n: int = 64, seed: int = 20240604, steps: int = 1000, cmin: int = 5_000,
                   cmax: int = 200_000, dt: float = 0.5) -> List[dict]:
    """Parameters of the batched ensemble's scenarios (see config_ensemble),
    one dict of channel_deck arguments per scenario."""
    rng = np.random.default_rng(seed)
    cell_area = 40_000.0 * 8_000.0 / 207_234
    out = []
    for i in range(n):
        c = int(round(math.exp(rng.uniform(math.log(cmin), math.log(cmax)))))
        n_man = float(rng.uniform(0.015, 0.04))
        q_peak = float(rng.uniform(50.0, 500.0))
        ly = math.sqrt(c * cell_area / 5.0)
        lx = 5.0 * ly
        out.append(dict(name=f"E{i:02d}_{c}", ncells=c, lx=lx, ly=ly, seed=seed * 1000 + i, bump_amp=1.0,
                        bump_width=max(150.0, 0.015 * lx), hydrograph=(q_peak, 250.0, 100.0),
                        n_manning=n_man, dt=dt, steps=steps, mdt=60))
    return out


def ensemble_deck(spec: dict) -> Deck:
    return channel_deck(**spec)


def config_ensemble(n: int = 64, seed: int = 20240604, steps: int = 1000, cmin: int = 5_000,
                    cmax: int = 200_000, dt: float = 0.5) -> List[Deck]:
    """The batched ensemble: ``n`` independent channel scenarios, each from its
    own seed.  Cells are log-uniform in [cmin, cmax]; Manning n ~ U(0.015, 0.04);
    a Gaussian inflow hydrograph peaking at Q ~ U(50, 500) m^3/s at t = 250 s
    (sigma 100 s); dt = 0.5 s.  Each domain is 5:1 with the cell area of the
    207,234-cell configuration (40 km x 8 km), bumps of 1 m."""
    return [ensemble_deck(sp) for sp in ensemble_specs(n, seed, steps, cmin, cmax, dt)]


def centroids(deck: Deck) -> np.ndarray:
    """[CELL, 2] centroid of every cell (mean of its nodes)."""
    nap = deck.nap
    nv = np.where(nap[:, 3] > 0, 4, 3)
    pts = deck.xy[np.maximum(nap - 1, 0)]                      # [C, 4, 2]
    pts[nv == 3, 3] = 0.0
    return pts.sum(axis=1) / nv[:, None]


def gaussian_field(xy: np.ndarray, corr_len: float, seed: int, spacing: Optional[float] = None) -> np.ndarray:
    """A seeded smooth Gaussian random field of unit variance at the points xy:
    white noise on a grid (spacing corr_len / 5) smoothed by a Gaussian kernel
    of standard deviation corr_len / sqrt(2), so that its covariance is
    exp(-r^2 / (2 corr_len^2)); bilinear interpolation to the points."""
    from scipy import ndimage
    h = spacing if spacing is not None else corr_len / 5.0
    lo = xy.min(axis=0) - 4 * corr_len
    hi = xy.max(axis=0) + 4 * corr_len
    shape = tuple(int(np.ceil((hi[k] - lo[k]) / h)) + 1 for k in (1, 0))   # (ny, nx)
    rng = np.random.default_rng(seed)
    g = ndimage.gaussian_filter(rng.standard_normal(shape), sigma=corr_len / np.sqrt(2.0) / h, mode="wrap")
    g /= g.std()
    coords = np.stack([(xy[:, 1] - lo[1]) / h, (xy[:, 0] - lo[0]) / h])
    return ndimage.map_coordinates(g, coords, order=1)


def adjoint_case(seed: int = 20240603, steps: int = 1000, ngauges: int = 50, obs_every: int = 10,
                 corr_len: float = 500.0):
    """The adjoint configuration: the 24,020-cell channel (config_24k) with
    uniform n = 0.025, the 'true' field n_true = 0.025 exp(0.2 g) for a seeded
    smooth Gaussian random field g of correlation length 500 m, and 50 seeded
    gauge cells observed every 10 steps.  Returns (deck, n_true, gauges)."""
    d = config_24k(seed=seed, steps=steps)
    g = gaussian_field(centroids(d), corr_len, seed + 17)
    n_true = 0.025 * np.exp(0.2 * g)
    rng = np.random.default_rng(seed + 29)
    gauges = np.sort(rng.choice(d.cells, ngauges, replace=False))
    return d, n_true, gauges


def fractal_surface(xy: np.ndarray, lx: float, ly: float, relief: float, seed: int, slope: float = -2.0,
                    n: int = 512) -> np.ndarray:
    """A seeded random surface with power spectrum ~ |k|^slope (Fourier
    synthesis on an n x n periodic grid over the domain), scaled to span
    [0, relief] and interpolated bilinearly at the points xy."""
    from scipy import ndimage
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(n)[:, None]
    ky = np.fft.fftfreq(n)[None, :]
    k = np.hypot(kx, ky)
    k[0, 0] = np.inf
    amp = k ** (slope / 2.0)
    spec = amp * np.exp(2j * np.pi * rng.uniform(size=(n, n)))
    z = np.real(np.fft.ifft2(spec))
    z = (z - z.min()) / (z.max() - z.min()) * relief
    coords = np.stack([xy[:, 0] / lx * (n - 1), xy[:, 1] / ly * (n - 1)])
    return ndimage.map_coordinates(z, coords, order=1)


def dam_break_deck(ncells: int = 2_000_000, length: float = 20_000.0, seed: int = 20240605, *,
                   relief: float = 5.0, level: float = 5.0, dam_x: float = 10_000.0, n_manning: float = 0.03,
                   dt: float = 0.5, steps: int = 2000, mdt: int = 60, hm1: float = 0.001,
                   hm2: float = 0.01) -> Deck:
    """The wetting/drying configuration: ``ncells`` Delaunay triangles on a
    ``length`` x ``length`` square closed by walls (KLAS 4), bed = a seeded
    fractal surface of spectral slope -2 spanning ``relief`` m, water level
    ``level`` m for x < ``dam_x`` and a dry bed elsewhere (the reference's
    preprocessing then sets H = HM1 where the level is at or below the bed,
    mesh.cpp:350-361), Manning n = 0.03.  No boundary tables are read; NDAYS
    covers ``steps`` steps."""
    xy, tris, (hx, hy) = delaunay_channel(ncells, length, length, seed)
    nodes4 = np.concatenate([tris, -np.ones((tris.shape[0], 1), dtype=np.int64)], axis=1)
    nv3 = np.ones(tris.shape[0], dtype=bool)
    nap, nac = _assemble("DAM", xy, nodes4, nv3)
    cen = xy[tris].mean(axis=1)
    zbc = fractal_surface(cen, length, length, relief, seed + 7)
    z0 = np.where(cen[:, 0] < dam_x, level, zbc - 1.0)
    klas = np.zeros_like(nac)
    bc, bs = _boundary_slots(nac, nap)
    klas[bc, bs] = KLAS_WALL
    spd = int(mdt / dt)
    ndays = int(math.ceil(steps / (spd - 1))) + 1
    return Deck(name=f"DAM_{ncells}", xy=xy, nap=nap, nac=nac, klas=klas, zbc=zbc, z0=z0,
                u0=np.zeros(nac.shape[0]), v0=np.zeros(nac.shape[0]), manning=np.full(nac.shape[0], n_manning),
                mdt=mdt, ndays=ndays, dt=dt, hm1=hm1, hm2=hm2,
                meta=dict(seed=seed, ncells=ncells, length=length, hx=hx, hy=hy, relief=relief, steps=steps))
