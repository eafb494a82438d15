"""ctypes front end of the CPU oracle (test infrastructure only).

Loads ``oracle/_build/liboracle.so`` (built by ``oracle/Makefile``), reads a
deck with the oracle's own restatement of the reference reader and steps it
with the oracle's restatement of the reference kernels. Used by the tests,
``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py`` only.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

VARIANT_H = 0
VARIANT_F = 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class _Deck(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("cells", "nod", "ndays", "mdt", "nz", "nq", "nzq", "nhq", "nwe", "ndi", "ntoutput")] + \
               [(n, C.c_double) for n in ("dt", "hm1", "hm2", "jl")] + \
               [(n, _dp) for n in ("nac", "klas", "side", "cosf", "sinf", "slcos", "slsin", "f0", "f1", "f2", "f3",
                                   "h", "u", "v", "z", "w", "zbc", "zb1", "area", "fnc", "bfeat")] + \
               [("nhq1", _ip)] + [(n, _dp) for n in ("zw", "qw", "qt", "dqt", "zt", "dzt")] + [("error", C.c_int)]


def build() -> str:
    """Build the oracle library if it is missing; returns its path."""
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "hydro_oracle.c")):
        subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile")], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        l = C.CDLL(build())
        l.orc_deck_load.argtypes = [C.c_char_p, C.POINTER(_Deck)]
        l.orc_deck_load.restype = C.c_int
        l.orc_deck_free.argtypes = [C.POINTER(_Deck)]
        l.orc_deck_sizeof.restype = C.c_size_t
        l.orc_flux.argtypes = [C.POINTER(_Deck), C.c_int, C.c_int, C.c_int]
        l.orc_update.argtypes = [C.POINTER(_Deck), C.c_int]
        l.orc_run.argtypes = [C.POINTER(_Deck), C.c_int, C.c_int, C.c_int]
        l.orc_run.restype = C.c_int
        l.orc_set_iterations.argtypes = [C.c_int, C.POINTER(C.c_byte)]
        if l.orc_deck_sizeof() != C.sizeof(_Deck):
            raise RuntimeError("oracle struct layout mismatch")
        _lib = l
    return _lib


CELL_FIELDS = ("h", "u", "v", "z", "w", "zbc", "zb1", "area", "fnc", "bfeat")
SLOT_FIELDS = ("nac", "klas", "side", "cosf", "sinf", "slcos", "slsin", "f0", "f1", "f2", "f3")
DAY_FIELDS = ("qt", "dqt", "zt", "dzt")


class OracleDeck:
    """A deck loaded by the oracle; arrays are numpy views of the C memory."""

    def __init__(self, root: str, variant: int = VARIANT_H):
        self._d = _Deck()
        if lib().orc_deck_load(root.encode(), C.byref(self._d)) != 0:
            raise IOError(f"oracle could not read deck {root}")
        self.variant = variant
        self.cells = self._d.cells
        self.step_index = 0

    def __del__(self):
        try:
            lib().orc_deck_free(C.byref(self._d))
        except Exception:
            pass

    def arr(self, name: str) -> np.ndarray:
        d = self._d
        if name in CELL_FIELDS:
            n = d.cells
        elif name in SLOT_FIELDS:
            n = 4 * d.cells
        elif name in DAY_FIELDS:
            n = d.cells * d.ndays
        elif name in ("zw", "qw"):
            n = d.cells * d.nhq
        elif name == "nhq1":
            return np.ctypeslib.as_array(d.nhq1, shape=(d.cells,))
        else:
            raise KeyError(name)
        return np.ctypeslib.as_array(getattr(d, name), shape=(n,))

    @property
    def error(self) -> int:
        return self._d.error

    @property
    def scalars(self) -> Dict[str, float]:
        d = self._d
        return dict(cells=d.cells, ndays=d.ndays, mdt=d.mdt, nhq=d.nhq, dt=d.dt, hm1=d.hm1, hm2=d.hm2, jl=d.jl)

    def flux(self, kt: int, jt: int) -> None:
        lib().orc_flux(C.byref(self._d), self.variant, kt, jt)

    def update(self) -> None:
        lib().orc_update(C.byref(self._d), self.variant)

    def run(self, n: int) -> int:
        done = lib().orc_run(C.byref(self._d), self.variant, self.step_index, n)
        self.step_index += done
        return done

    def gauge_rollout(self, n, zbc, Z0, U0, V0, gauges, obs_every: int, nsteps: int, counts=None,
                      mode: int = 0) -> np.ndarray:
        """The adjoint's rollout restated: from the level Z0 and velocities
        (initial depth as mesh.cpp:350-361: H = Z0 - ZBC where the level is
        above the bed, else H = HM1 and Z = ZBC + HM1), Manning n (FNC = 9.81
        n^2, mesh.cpp:364) and bed ZBC (ZB1 = ZBC + HM1), nsteps steps of the
        driver's loop from step 0; returns the gauge depths after every
        obs_every steps [nobs][ngauges].

        Iteration counts of the boundary fixed points (orc_set_iterations):
        mode 1 records them into counts [nsteps][4*cells] (int8), mode 2
        replays them, mode 0 runs the reference's stopping tests."""
        d = self._d
        hm1 = d.hm1
        zbc = np.asarray(zbc, np.float64)
        Z0 = np.asarray(Z0, np.float64)
        self.arr("fnc")[:] = 9.81 * np.asarray(n, np.float64) * np.asarray(n, np.float64)
        self.arr("zbc")[:] = zbc
        self.arr("zb1")[:] = zbc + hm1
        dry = Z0 <= zbc
        self.arr("h")[:] = np.where(dry, hm1, Z0 - zbc)
        self.arr("z")[:] = np.where(dry, zbc + hm1, Z0)
        self.arr("u")[:] = U0
        self.arr("v")[:] = V0
        for f in ("f0", "f1", "f2", "f3"):
            self.arr(f)[:] = 0.0
        self.step_index = 0
        g = np.asarray(gauges, dtype=np.int64)
        out = []
        h = self.arr("h")
        try:
            for t in range(nsteps):
                if mode:
                    row = np.ascontiguousarray(counts[t])
                    lib().orc_set_iterations(mode, row.ctypes.data_as(C.POINTER(C.c_byte)))
                self.run(1)
                if mode == 1:
                    counts[t] = row
                if (t + 1) % obs_every == 0:
                    out.append(h[g].copy())
        finally:
            lib().orc_set_iterations(0, None)
        return np.array(out)

    def dump(self) -> Dict[str, np.ndarray]:
        """The arrays of a reference ``--dump`` (benchmark.cu:141-162), copied."""
        m = {"H": "h", "U": "u", "V": "v", "Z": "z", "SLCOS": "slcos", "SLSIN": "slsin", "SIDE": "side",
             "FLUX0": "f0", "FLUX1": "f1", "FLUX2": "f2", "FLUX3": "f3"}
        return {k: self.arr(v).copy() for k, v in m.items()}
