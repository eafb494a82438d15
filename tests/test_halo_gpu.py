"""A mesh split into parts on the GPU (hydrob200.halo, hb_halo_*), GPU.

The parts run as separate handles on one GPU, in one process: after every
step each part packs the records its neighbours' halos need and the
neighbours unpack them, all in stream order (no kernel waits on another
part).  The owned cells must equal the single-handle run of the whole mesh
bit for bit, in fp64 (edge and tile layouts) and in split precision, on the
channel deck and on a stress deck with every boundary code.
"""
import numpy as np
import pytest

import hydrob200 as hb
from hydrob200 import halo

pytestmark = pytest.mark.gpu

STEPS = 25


@pytest.mark.parametrize("name,nparts,kw", [
    ("f1", 3, {}),
    ("stress_a", 2, {}),
    ("f1", 2, {"precision": "split"}),
    ("stress_b", 3, {"layout": "tile", "tile_cells": 128}),
])
def test_split_run_equals_single_handle(deck_dir, name, nparts, kw):
    deck = hb.Deck(deck_dir[name])
    whole = hb.Solver(deck, **kw)
    whole.step(STEPS)
    want = whole.get_state()
    run = halo.split_deck(deck, nparts, **kw)
    run.step(STEPS)
    got = run.gather()
    for k in "HUVZ":
        np.testing.assert_array_equal(got[k], want[k], err_msg=f"{name} {kw} {k}")
    run.close()
    whole.close()


def test_halo_lists_are_checked(deck_dir):
    import ctypes as C
    from hydrob200 import _lib
    deck = hb.Deck(deck_dir["f1"])
    s = hb.Solver(deck)
    lid = C.c_int32()
    bad = np.array([0, deck.cells], dtype=np.int32)
    with pytest.raises(hb.HydroError):
        _lib.check(_lib.lib().hb_halo_define(s._h, bad.ctypes.data_as(_lib._ip), 2, C.byref(lid)))
    with pytest.raises(hb.HydroError):
        _lib.check(_lib.lib().hb_halo_pack(s._h, 7, C.c_void_p(256), None))
    s.close()
