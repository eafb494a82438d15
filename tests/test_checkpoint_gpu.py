"""Checkpoint / resume (hb_checkpoint_*), GPU.

A run interrupted after some steps, saved, restored into a fresh handle and
continued must end exactly where the uninterrupted run ends: state, fluxes
(including the stale ones of codes that leave fluxes unwritten) and boundary
codes, bit for bit, in every precision, both layouts and batches.
"""
import numpy as np
import pytest

import hydrob200 as hb

pytestmark = pytest.mark.gpu


def _same(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return bool(np.all((a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))))


@pytest.mark.parametrize("precision,layout", [("fp64", "edge"), ("fp64", "tile"), ("split", "tile"), ("fp32", "edge")])
def test_resume_is_bit_exact(deck_dir, precision, layout):
    deck = hb.Deck(deck_dir["stress_a"])
    whole = hb.Solver(deck, precision=precision, layout=layout, tile_cells=64)
    whole.step(30)
    whole.sync()
    first = hb.Solver(deck, precision=precision, layout=layout, tile_cells=64)
    first.step(13)
    blob = first.checkpoint()
    first.close()
    second = hb.Solver(deck, precision=precision, layout=layout, tile_cells=64, init_state=False)
    second.restore(blob)
    assert second.position[0] == 13
    second.capture_graph(17)        # a graph replays from the restored position
    second.graph_launch()
    second.sync()
    a, b = whole.get_state(), second.get_state()
    for k in "HUVZW":
        assert _same(a[k], b[k]), k
    fa, fb = whole.flux(), second.flux()
    for k in fa:
        assert _same(fa[k], fb[k]), k
    np.testing.assert_array_equal(whole.klas(), second.klas())


def test_resume_keeps_a_breach(deck_dir):
    deck = hb.Deck(deck_dir["breach"])
    a = hb.Solver(deck)
    a.step(1)
    blob = a.checkpoint()
    b = hb.Solver(deck, init_state=False)
    b.restore(blob)
    np.testing.assert_array_equal(a.klas(), b.klas())
    assert np.any(a.klas() != deck.array("klas"))   # some KLAS 7 slot breached


def test_batch_resume_and_mismatch(deck_dir):
    decks = [hb.Deck(deck_dir[n]) for n in ("stress_a", "f1")]
    whole = hb.Batch(decks, precision="split")
    whole.step(20)
    part = hb.Batch(decks, precision="split")
    part.step(8)
    blob = part.checkpoint()
    again = hb.Batch(decks, precision="split", init_state=False)
    again.restore(blob)
    again.step(12)
    again.sync()
    whole.sync()
    for i in range(2):
        for k in "HUVZ":
            assert _same(whole.get_state(i)[k], again.get_state(i)[k])
    other = hb.Batch(decks, precision="fp64")
    with pytest.raises(hb.HydroError):
        other.restore(blob)
    with pytest.raises(hb.HydroError):
        other.restore(b"not a checkpoint" * 8)
