"""Batches of independent scenarios in one launch (hb_create_batch), GPU.

A batch concatenates its scenarios on the device and gives every CTA one
scenario through segment tables, so each scenario must come out bit for bit
as it does from its own handle: same state, fluxes and boundary codes, in
every precision and variant, whatever the launch shape, through graphs and
the autotuner (which must leave the state as it found it).
"""
import numpy as np
import pytest

import hydrob200 as hb

pytestmark = pytest.mark.gpu

NAMES = ["stress_a", "f1", "breach", "stress_b"]   # different sizes, DT, table intervals and codes


def _bits_equal(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return bool(np.all((a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))))


def _run_single(deck, steps, **kw):
    s = hb.Solver(deck, **kw)
    s.step(steps)
    s.sync()
    return s.get_state(), s.flux(), s.klas()


@pytest.mark.parametrize("layout", ["edge", "tile"])
@pytest.mark.parametrize("precision,variant", [("fp64", "H"), ("fp64", "F"), ("split", "H"), ("fp32", "H")])
def test_batch_equals_single_handles(deck_dir, precision, variant, layout):
    decks = [hb.Deck(deck_dir[n]) for n in NAMES]
    steps = 1   # breach has tables for one step
    b = hb.Batch(decks, precision=precision, variant=variant, layout=layout, tile_cells=64)
    assert len(b) == len(decks)
    b.step(steps)
    b.sync()
    for i, d in enumerate(decks):
        st, fl, kl = _run_single(d, steps, precision=precision, variant=variant)
        bst, bfl, bkl = b.get_state(i), b.flux(i), b.klas(i)
        for k in "HUVZW":
            assert _bits_equal(bst[k], st[k]), f"{NAMES[i]} {k}"
        for k in fl:
            assert _bits_equal(bfl[k], fl[k]), f"{NAMES[i]} {k}"
        np.testing.assert_array_equal(bkl, kl)


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_batch_many_steps_and_shapes(deck_dir, precision):
    """50 steps (stress decks cross table intervals of 19 steps, f1 does not),
    every launch shape, graph replay; each scenario equals its own handle."""
    names = ["stress_a", "f1", "stress_b", "probe"]
    decks = [hb.Deck(deck_dir[n]) for n in names]
    ref = [_run_single(d, 50, precision=precision)[0] for d in decks]
    for cfg, shape in hb.launch_shapes().items():
        b = hb.Batch(decks, precision=precision, tile_config=cfg, layout=shape["layout"], tile_cells=96)
        if cfg % 2:
            b.step(50)
        else:
            b.capture_graph(25)
            b.graph_launch()
            b.graph_launch()
        b.sync()
        for i in range(len(decks)):
            st = b.get_state(i)
            for k in "HUVZ":
                assert _bits_equal(st[k], ref[i][k]), f"tile_config {cfg}: {names[i]} {k}"
        b.close()


@pytest.mark.parametrize("layout", ["edge", "tile"])
def test_autotune_leaves_state_and_picks_a_shape(deck_dir, layout):
    decks = [hb.Deck(deck_dir[n]) for n in ["stress_a", "f1", "stress_b"]]
    a = hb.Batch(decks, precision="split", layout=layout)
    b = hb.Batch(decks, precision="split", layout=layout)
    a.step(5)
    b.step(5)
    best, ms = a.autotune(steps=10)
    assert best == a.tile_config and best in ms and set(ms) == set(a.shapes())
    assert all(v > 0 for v in ms.values())
    assert a.position == b.position
    a.step(20)
    b.step(20)
    a.sync()
    b.sync()
    for i in range(3):
        sa, sb = a.get_state(i), b.get_state(i)
        for k in "HUVZW":
            assert _bits_equal(sa[k], sb[k]), f"scenario {i} {k}"


def test_batch_arguments(deck_dir):
    decks = [hb.Deck(deck_dir[n]) for n in ["stress_a", "f1"]]
    b = hb.Batch(decks)
    out = np.empty(decks[0].cells)
    ptr = out.ctypes.data_as(hb._lib._dp)
    assert hb._lib.lib().hb_get_state_at(b._h, 2, ptr, ptr, ptr, ptr, ptr) == 1   # HB_E_INVALID
    with pytest.raises(hb.HydroError):
        b.step_host(*[np.zeros(decks[0].cells) for _ in range(5)], n=1)
    with pytest.raises(hb.HydroError):
        b.tile_config = 99
    with pytest.raises(hb.HydroError):   # a tile-layout shape on an edge-layout handle
        b.tile_config = next(k for k, v in hb.launch_shapes().items() if v["layout"] == "tile")
