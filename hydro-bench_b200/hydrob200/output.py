"""Result files in the reference's text formats (``hb_output_*``).

``run_with_output`` steps a solver through the reference driver's day/step
loop with its output cadence (cuda_native_impl/benchmark.cu:105-124): the
initial frame, then a frame after the last step of every NTOUTPUT-th day and
after the last step.
"""
import ctypes as C
import os
from typing import Optional

import numpy as np

from . import _lib
from ._lib import check, lib
from .solver import Deck


class Output:
    """SIDE.OUT, H2U2V2.OUT, ZUV.OUT, XY-TEC.DAT and TIMELOG.OUT in `directory`."""

    def __init__(self, deck: Deck, directory: str):
        os.makedirs(directory, exist_ok=True)
        self.deck = deck
        self._h = C.c_void_p()
        check(lib().hb_output_open(deck._h, directory.encode(), C.byref(self._h)))

    def frame(self, jt: int, kt: int, state) -> None:
        arrs = [np.ascontiguousarray(state[k], dtype=np.float64) for k in "HUVZ"]
        check(lib().hb_output_frame(self._h, int(jt), int(kt), *[a.ctypes.data_as(_lib._dp) for a in arrs]))

    def close(self) -> None:
        if self._h.value:
            lib().hb_output_close(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ntoutput(deck: Deck) -> int:
    v = C.c_int32()
    check(lib().hb_deck_ntoutput(deck._h, C.byref(v)))
    return v.value


def run_with_output(solver, deck: Deck, directory: str, steps: int, every_days: Optional[int] = None) -> None:
    """Steps `solver` (fresh, at step 0) `steps` steps, writing frames as the
    reference driver's --with-output run does (NTOUTPUT from the deck unless
    `every_days` is given)."""
    every = every_days if every_days is not None else ntoutput(deck)
    if every <= 0:
        every = 1
    per_day = deck.mesh.steps_per_day - 1
    out = Output(deck, directory)
    out.frame(0, 1, solver.get_state())
    done = 0
    day = 0
    while day < deck.mesh.ndays and done < steps:
        n = min(per_day, steps - done)
        solver.step(n)
        done += n
        last_of_day = n == per_day or done == steps
        if last_of_day and ((day + 1) % every == 0 or done == steps):
            solver.sync()
            out.frame(day, n + 1, solver.get_state())
        day += 1
    out.close()
