"""Python side of the library: deck reading, the handle-based solver and the
reference-layout drop-in, all through the C ABI (``_lib``).

Naming follows the reference: a *deck* is a hydro-cal input directory, a
*slot* is one of the four edge positions of a cell (``4*cell + j``), *KLAS*
the boundary code of a slot, ``kt``/``jt`` the step within a boundary-table
interval and the interval ("day") index of ``cuda_native_impl/benchmark.cu:87-96``.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check, lib, HydroError, VARIANT_H, VARIANT_F, FP64, FP32, SPLIT  # noqa: F401

_VARIANTS = {"H": VARIANT_H, "F": VARIANT_F, VARIANT_H: VARIANT_H, VARIANT_F: VARIANT_F}
_PRECISIONS = {"fp64": FP64, "fp32": FP32, "split": SPLIT, FP64: FP64, FP32: FP32, SPLIT: SPLIT}
_LAYOUTS = {"edge": _lib.LAYOUT_EDGE, "tile": _lib.LAYOUT_TILE, _lib.LAYOUT_EDGE: _lib.LAYOUT_EDGE,
            _lib.LAYOUT_TILE: _lib.LAYOUT_TILE}


def launch_shapes():
    """The compiled launch shapes (hb_launch_shapes): tile_config -> layout, threads, CTAs per SM."""
    n = lib().hb_launch_shapes(None, None, None, 0)
    lay, thr, mb = (C.c_int32 * n)(), (C.c_int32 * n)(), (C.c_int32 * n)()
    lib().hb_launch_shapes(lay, thr, mb, n)
    names = {_lib.LAYOUT_EDGE: "edge", _lib.LAYOUT_TILE: "tile"}
    return {i + 1: dict(layout=names[lay[i]], threads=thr[i], min_blocks=mb[i] // 100, update_min_blocks=mb[i] % 100)
            for i in range(n)}


def _options(variant, precision, device, renumber, tile_config, layout, tile_cells, persistent=False):
    opt = _lib.Options()
    lib().hb_options_default(C.byref(opt))
    opt.variant = _VARIANTS[variant]
    opt.precision = _PRECISIONS[precision]
    opt.device = device
    opt.renumber = 1 if renumber else 0
    opt.tile_config = int(tile_config)
    opt.layout = _LAYOUTS[layout]
    opt.tile_cells = int(tile_cells)
    opt.persistent = 1 if persistent else 0
    return opt

CELL_ARRAYS = ("zbc", "zb1", "area", "fnc", "bfeat")
SLOT_ARRAYS = ("nac", "klas", "side", "cosf", "sinf", "slcos", "slsin")
DAY_ARRAYS = ("qt", "dqt", "zt", "dzt")


def _stream_handle(stream) -> Optional[int]:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)   # torch.cuda.Stream


class Deck:
    """A hydro-cal deck read by the library's reader (``hb_deck_load``)."""

    def __init__(self, root: str):
        self._h = C.c_void_p()
        self._lib = lib()   # held for __del__, which may run after module teardown
        check(self._lib.hb_deck_load(root.encode(), C.byref(self._h)))
        self.root = root
        self.mesh = _lib.MeshDesc()
        check(lib().hb_deck_mesh(self._h, C.byref(self.mesh)))

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            try:
                self._lib.hb_deck_free(self._h)
                self._h = C.c_void_p()
            except TypeError:   # interpreter shutdown: ctypes already torn down, the process frees everything
                pass

    @property
    def cells(self) -> int:
        return self.mesh.cells

    def array(self, name: str) -> np.ndarray:
        """Borrowed numpy view of a mesh array (reference order)."""
        m = self.mesh
        n = {**{k: m.cells for k in CELL_ARRAYS}, **{k: 4 * m.cells for k in SLOT_ARRAYS},
             **{k: m.cells * m.ndays for k in DAY_ARRAYS}, "zw": m.cells * m.nhq, "qw": m.cells * m.nhq,
             "nhq1": m.cells}[name]
        return np.ctypeslib.as_array(getattr(m, name), shape=(n,))

    def state(self) -> Dict[str, np.ndarray]:
        ptrs = [_lib._dp() for _ in range(5)]
        check(lib().hb_deck_state(self._h, *[C.byref(p) for p in ptrs]))
        return {k: np.ctypeslib.as_array(p, shape=(self.cells,)).copy() for k, p in zip("HUVZW", ptrs)}


def _as_dp(a: np.ndarray):
    return a.ctypes.data_as(_lib._dp)


class Solver:
    """The handle-based timestep (``hb_create`` ... ``hb_destroy``).

    State and fluxes cross the boundary in the reference's order; on the
    device the cells are renumbered (``hb_get_permutation``).
    """

    def __init__(self, deck: Deck, variant="H", precision="fp64", device: int = 0, renumber: bool = True,
                 init_state: bool = True, tile_config: int = 0, layout="edge", tile_cells: int = 0,
                 persistent: bool = False):
        self.deck = deck   # keeps the host arrays alive
        opt = _options(variant, precision, device, renumber, tile_config, layout, tile_cells, persistent)
        self.layout = opt.layout
        self.variant = opt.variant
        self.precision = opt.precision
        self._h = C.c_void_p()
        check(lib().hb_create(C.byref(deck.mesh), C.byref(opt), C.byref(self._h)))
        self.cells = deck.cells
        if init_state:
            st = deck.state()
            self.set_state(st["H"], st["U"], st["V"], st["Z"], st["W"])

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().hb_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, H, U, V, Z, W=None):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (H, U, V, Z)]
        w = np.ascontiguousarray(W, dtype=np.float64) if W is not None else None
        for a in arrs:
            if a.shape != (self.cells,):
                raise ValueError("state arrays must have shape (cells,)")
        check(lib().hb_set_state(self._h, *[_as_dp(a) for a in arrs], _as_dp(w) if w is not None else None))

    def get_state(self) -> Dict[str, np.ndarray]:
        out = {k: np.empty(self.cells) for k in "HUVZW"}
        check(lib().hb_get_state(self._h, *[_as_dp(out[k]) for k in "HUVZW"]))
        return out

    def flux(self) -> Dict[str, np.ndarray]:
        out = {k: np.empty(4 * self.cells) for k in ("FLUX0", "FLUX1", "FLUX2", "FLUX3")}
        check(lib().hb_get_flux(self._h, *[_as_dp(out[k]) for k in ("FLUX0", "FLUX1", "FLUX2", "FLUX3")]))
        return out

    def klas(self) -> np.ndarray:
        out = np.empty(4 * self.cells)
        check(lib().hb_get_klas(self._h, _as_dp(out)))
        return out

    def step(self, n: int, stream=None) -> None:
        check(lib().hb_step(self._h, int(n), _stream_handle(stream)))

    def step_host(self, H, U, V, Z, W, n: int = 1, stream=None) -> None:
        """hb_step_host: state in/out through host buffers (numpy arrays or
        page-locked CPU torch tensors, fp64, reference order). Asynchronous."""
        def ptr(a):
            if a is None:
                return None
            if hasattr(a, "data_ptr"):
                return C.cast(C.c_void_p(a.data_ptr()), _lib._dp)
            return _as_dp(a)
        check(lib().hb_step_host(self._h, ptr(H), ptr(U), ptr(V), ptr(Z), ptr(W), int(n), _stream_handle(stream)))

    def sync(self, stream=None) -> None:
        check(lib().hb_sync(self._h, _stream_handle(stream)))

    def checkpoint(self) -> bytes:
        """hb_checkpoint_save: everything needed to continue this run bit for bit."""
        n = C.c_size_t()
        check(lib().hb_checkpoint_size(self._h, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        check(lib().hb_checkpoint_save(self._h, buf, n.value))
        return buf.raw

    def restore(self, blob: bytes) -> None:
        """hb_checkpoint_load: continue from a checkpoint of the same mesh and options."""
        buf = C.create_string_buffer(blob, len(blob))
        check(lib().hb_checkpoint_load(self._h, buf, len(blob)))

    def write_dump(self, path: str, scenario: int = 0, deck: Deck = None) -> None:
        """hb_write_dump: the reference driver's --dump file (benchmark.cu:141-162)."""
        d = deck if deck is not None else (self.deck if hasattr(self, "deck") else self.decks[scenario])
        check(lib().hb_write_dump(self._h, scenario, C.byref(d.mesh), path.encode()))

    def device_errors(self) -> int:
        v = C.c_uint32()
        check(lib().hb_device_errors(self._h, C.byref(v)))
        return v.value

    def set_barrier_limit(self, timeout_ns: int, phantom_arrivals: int = 0) -> None:
        """hb_set_barrier_limit: bound of the persistent kernel's grid-barrier waits."""
        check(lib().hb_set_barrier_limit(self._h, int(timeout_ns), int(phantom_arrivals)))

    @property
    def position(self):
        s, kt, jt = C.c_int64(), C.c_int32(), C.c_int32()
        check(lib().hb_position(self._h, C.byref(s), C.byref(kt), C.byref(jt)))
        return s.value, kt.value, jt.value

    def set_position(self, steps_done: int) -> None:
        check(lib().hb_set_position(self._h, int(steps_done)))

    def capture_graph(self, n: int, stream=None) -> None:
        check(lib().hb_capture_graph(self._h, int(n), _stream_handle(stream)))

    def graph_launch(self, stream=None) -> None:
        check(lib().hb_graph_launch(self._h, _stream_handle(stream)))

    @property
    def tile_config(self) -> int:
        v = C.c_int32()
        check(lib().hb_get_tile_config(self._h, C.byref(v)))
        return v.value

    @tile_config.setter
    def tile_config(self, cfg: int) -> None:
        check(lib().hb_set_tile_config(self._h, int(cfg)))

    def shapes(self):
        """tile_config values of this handle's layout."""
        names = {_lib.LAYOUT_EDGE: "edge", _lib.LAYOUT_TILE: "tile"}
        return [k for k, v in launch_shapes().items() if v["layout"] == names[self.layout]]

    def autotune(self, steps: int = 20, stream=None):
        """hb_autotune: times every launch shape of this handle's layout on its
        mesh(es) and keeps the fastest; returns (best tile_config, ms per step
        by tile_config)."""
        n = lib().hb_tile_configs(None, None, 0)
        ms = (C.c_float * n)()
        best = C.c_int32()
        check(lib().hb_autotune(self._h, int(steps), _stream_handle(stream), ms, n, C.byref(best)))
        return best.value, {k: float(ms[k - 1]) for k in self.shapes()}

    def permutation(self) -> np.ndarray:
        p = np.empty(self.cells, dtype=np.int32)
        check(lib().hb_get_permutation(self._h, p.ctypes.data_as(_lib._ip)))
        return p

    def device_state(self):
        """Zero-copy torch views of the device state (renumbered order): H, U, V,
        Z, W (split precision: H, U, V, H_lo, W)."""
        import torch
        ptrs = [C.c_void_p() for _ in range(5)]
        stride = C.c_int32()
        check(lib().hb_device_state(self._h, *[C.byref(p) for p in ptrs], C.byref(stride)))
        dt = "<f8" if self.precision == FP64 else "<f4"
        item = 8 if self.precision == FP64 else 4

        class _CAI:
            def __init__(self, ptr, n, st):
                self.__cuda_array_interface__ = {"shape": (n,), "typestr": dt, "data": (ptr, False), "version": 3,
                                                 "strides": (st * item,)}

        # split precision keeps no level: its fourth interleaved entry is the depth's low part ("H_lo")
        names = "HUVZW" if self.precision != SPLIT else ("H", "U", "V", "H_lo", "W")
        out = {}
        for k, p in zip(names, ptrs):
            if k == "H_lo":
                p = C.c_void_p(ptrs[0].value + 3 * item)
            out[k] = torch.as_tensor(_CAI(p.value, self.cells, stride.value if k != "W" else 1), device="cuda")
        return out


class Batch(Solver):
    """A batch of independent scenarios stepped together (``hb_create_batch``).

    Every launch covers all scenarios; per-scenario state, fluxes and boundary
    codes are read and written with the ``*_at`` calls (``scenario`` index).
    ``step``, ``sync``, ``capture_graph`` and ``graph_launch`` advance all.
    """

    def __init__(self, decks: Sequence[Deck], variant="H", precision="fp64", device: int = 0,
                 renumber: bool = True, init_state: bool = True, tile_config: int = 0, layout="edge",
                 tile_cells: int = 0, persistent: bool = False):
        self.decks = list(decks)   # keeps the host arrays alive
        opt = _options(variant, precision, device, renumber, tile_config, layout, tile_cells, persistent)
        self.layout = opt.layout
        self.variant = opt.variant
        self.precision = opt.precision
        meshes = (_lib.MeshDesc * len(self.decks))(*[d.mesh for d in self.decks])
        self._h = C.c_void_p()
        check(lib().hb_create_batch(meshes, len(self.decks), C.byref(opt), C.byref(self._h)))
        self.sizes = [d.cells for d in self.decks]
        self.cells = sum(self.sizes)
        if init_state:
            for i, d in enumerate(self.decks):
                st = d.state()
                self.set_state(st["H"], st["U"], st["V"], st["Z"], st["W"], scenario=i)

    def __len__(self):
        return len(self.decks)

    def set_state(self, H, U, V, Z, W=None, scenario: int = 0):
        n = self.sizes[scenario]
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (H, U, V, Z)]
        w = np.ascontiguousarray(W, dtype=np.float64) if W is not None else None
        for a in arrs:
            if a.shape != (n,):
                raise ValueError(f"state arrays of scenario {scenario} must have shape ({n},)")
        check(lib().hb_set_state_at(self._h, scenario, *[_as_dp(a) for a in arrs],
                                    _as_dp(w) if w is not None else None))

    def get_state(self, scenario: int = 0) -> Dict[str, np.ndarray]:
        out = {k: np.empty(self.sizes[scenario]) for k in "HUVZW"}
        check(lib().hb_get_state_at(self._h, scenario, *[_as_dp(out[k]) for k in "HUVZW"]))
        return out

    def flux(self, scenario: int = 0) -> Dict[str, np.ndarray]:
        n = 4 * self.sizes[scenario]
        out = {k: np.empty(n) for k in ("FLUX0", "FLUX1", "FLUX2", "FLUX3")}
        check(lib().hb_get_flux_at(self._h, scenario, *[_as_dp(out[k]) for k in ("FLUX0", "FLUX1", "FLUX2", "FLUX3")]))
        return out

    def klas(self, scenario: int = 0) -> np.ndarray:
        out = np.empty(4 * self.sizes[scenario])
        check(lib().hb_get_klas_at(self._h, scenario, _as_dp(out)))
        return out

    def permutation(self, scenario: int = 0) -> np.ndarray:
        p = np.empty(self.sizes[scenario], dtype=np.int32)
        check(lib().hb_get_permutation_at(self._h, scenario, p.ctypes.data_as(_lib._ip)))
        return p


class RefLayoutMesh:
    """The reference's device arrays (``MeshView``, cell.cpp:11-146, side.cpp:11-52)
    held in torch CUDA tensors, stepped through the drop-in entry points
    ``hb_ref_calculate_flux`` / ``hb_ref_update_cell`` (functors.cu:787-818)."""

    def __init__(self, deck: Deck, variant="H", precision="fp64", device="cuda"):
        import torch
        self.variant = _VARIANTS[variant]
        self.fp32 = _PRECISIONS[precision] == FP32
        dt = torch.float32 if self.fp32 else torch.float64
        m = deck.mesh
        self.cells = m.cells
        self.ndays = m.ndays
        self.steps_per_day = m.steps_per_day
        t = lambda a, d=dt: torch.as_tensor(np.ascontiguousarray(a), device=device).to(d).contiguous()
        st = deck.state()
        self.T = {k: t(st[k]) for k in "HUVZW"}
        for k in CELL_ARRAYS + SLOT_ARRAYS + DAY_ARRAYS + ("zw", "qw"):
            self.T[k] = t(deck.array(k))
        self.T["nhq1"] = t(deck.array("nhq1"), torch.int32)
        for k in ("FLUX0", "FLUX1", "FLUX2", "FLUX3"):
            self.T[k] = torch.zeros(4 * m.cells, dtype=dt, device=device)
        V = _lib.RefMeshViewF32 if self.fp32 else _lib.RefMeshView
        real = C.c_float if self.fp32 else C.c_double
        rp = C.POINTER(real)
        p = lambda k: C.cast(C.c_void_p(self.T[k].data_ptr()), rp)
        v = V()
        v.NHQ, v.NQ, v.NZ, v.NWE, v.NDAYS, v.CELL = m.nhq, 0, 0, 0, m.ndays, m.cells
        v.DT, v.HM1, v.HM2, v.JL = m.dt, m.hm1, m.hm2, m.jl
        c = v.cells
        c.H, c.U, c.V, c.W, c.Z = p("H"), p("U"), p("V"), p("W"), p("Z")
        c.NHQ1 = C.cast(C.c_void_p(self.T["nhq1"].data_ptr()), _lib._ip)
        c.ZBC, c.ZB1, c.AREA, c.FNC, c.BoundaryFeature = p("zbc"), p("zb1"), p("area"), p("fnc"), p("bfeat")
        c.ZW, c.QW, c.QT, c.DQT, c.ZT, c.DZT = p("zw"), p("qw"), p("qt"), p("dqt"), p("zt"), p("dzt")
        s = v.sides
        s.KLAS, s.NAC, s.SIDE, s.COSF, s.SINF = p("klas"), p("nac"), p("side"), p("cosf"), p("sinf")
        s.SLCOS, s.SLSIN = p("slcos"), p("slsin")
        s.FLUX0, s.FLUX1, s.FLUX2, s.FLUX3 = p("FLUX0"), p("FLUX1"), p("FLUX2"), p("FLUX3")
        self.view = v
        self.steps_done = 0

    def calculate_flux(self, kt: int, jt: int, stream=None) -> None:
        f = lib().hb_ref_calculate_flux_f32 if self.fp32 else lib().hb_ref_calculate_flux
        check(f(C.byref(self.view), kt, jt, self.variant, _stream_handle(stream)))

    def update_cell(self, stream=None) -> None:
        f = lib().hb_ref_update_cell_f32 if self.fp32 else lib().hb_ref_update_cell
        check(f(C.byref(self.view), self.variant, _stream_handle(stream)))

    def run(self, n: int, stream=None) -> None:
        """The driver loop of benchmark.cu:87-96, continuing from where it stopped."""
        per_day = self.steps_per_day - 1
        for _ in range(n):
            s = self.steps_done
            jt, kt = s // per_day, 1 + s % per_day
            if jt >= self.ndays:
                raise HydroError(1, "beyond the boundary tables")
            self.calculate_flux(kt, jt, stream)
            self.update_cell(stream)
            self.steps_done += 1

    def dump(self) -> Dict[str, np.ndarray]:
        import torch
        torch.cuda.synchronize()
        m = {"H": "H", "U": "U", "V": "V", "Z": "Z", "W": "W", "FLUX0": "FLUX0", "FLUX1": "FLUX1",
             "FLUX2": "FLUX2", "FLUX3": "FLUX3", "KLAS": "klas"}
        return {k: self.T[v].double().cpu().numpy() for k, v in m.items()}


def take_ref_device_errors() -> int:
    v = C.c_uint32()
    check(lib().hb_ref_take_device_errors(C.byref(v)))
    return v.value
