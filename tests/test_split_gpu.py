"""Split precision (HB_SPLIT) against the fp64 oracle (GPU).

Split precision has no reference counterpart: fluxes, velocities and depths
are fp32, water levels, beds and boundary levels fp64, every level-minus-bed
depth is formed in fp64, and the depth update is Kahan-compensated.  Its
error is measured against the CPU oracle's fp64 run (hydrob200.accuracy):
  * channel deck F1 (6,675 cells), 1000 steps: per-cell relative depth error
    <= 1e-6 on wet cells at every 100th step, mass within 1e-7;
  * the stress decks (every boundary code, wetting and drying), 10 steps:
    per-cell relative depth error <= 5e-6;
and it must beat the plain fp32 tree on the same runs.
"""
import numpy as np
import pytest

import hydrob200 as hb
from hydrob200 import deck as D
from hydrob200.accuracy import depth_error
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def f1_1000(tmp_path_factory):
    d = D.config_f1(steps=1000)
    root = str(tmp_path_factory.mktemp("f1_1000") / "deck")
    D.write_deck(d, root)
    return root


def test_state_round_trip(deck_dir):
    """set_state -> get_state keeps H to fp64 precision (h + h_lo) above the dry
    threshold HM1, to fp32 precision at or below it, and the level everywhere,
    including dry cells whose level lies below the bed (mesh.cpp:350-361 keeps
    such a level while H = HM1)."""
    deck = hb.Deck(deck_dir["stress_a"])
    st0 = deck.state()
    zbc = deck.array("zbc")
    hm1 = deck.mesh.hm1
    dry = np.arange(0, deck.cells, 7)
    st0["Z"][dry] = zbc[dry] - 0.1
    st0["H"][dry] = hm1
    s = hb.Solver(deck, precision="split", init_state=False)
    s.set_state(st0["H"], st0["U"], st0["V"], st0["Z"], st0["W"])
    st = s.get_state()
    rel = np.abs(st["H"] - st0["H"]) / st0["H"]
    above = st0["H"] > np.float32(hm1)
    assert above.any() and (~above).any()
    assert np.max(rel[above]) <= 2.0 ** -44
    assert np.max(rel[~above]) <= 2.0 ** -24
    np.testing.assert_array_equal(st["H"][dry], hm1)
    assert np.max(np.abs(st["Z"] - st0["Z"])) <= 1e-6
    np.testing.assert_array_equal(st["U"], st0["U"].astype(np.float32).astype(np.float64))


def test_f1_1000_steps_against_oracle(f1_1000):
    deck = hb.Deck(f1_1000)
    area = deck.array("area")
    hm2 = deck.mesh.hm2
    o = O.OracleDeck(f1_1000)
    sp = hb.Solver(deck, precision="split")
    f32 = hb.Solver(deck, precision="fp32")
    worst = {"split": 0.0, "fp32": 0.0}
    for k in range(10):
        o.run(100)
        sp.step(100)
        f32.step(100)
        sp.sync()
        f32.sync()
        h_ref = o.dump()["H"]
        e = depth_error(sp.get_state()["H"], h_ref, hm2, area)
        e32 = depth_error(f32.get_state()["H"], h_ref, hm2, area)
        assert e["rel_max"] <= 1e-6, (100 * (k + 1), e)
        assert abs(e["mass_rel"]) <= 1e-7, (100 * (k + 1), e)
        worst["split"] = max(worst["split"], e["rel_max"])
        worst["fp32"] = max(worst["fp32"], e32["rel_max"])
    assert worst["split"] < worst["fp32"], worst


@pytest.mark.parametrize("name", ["stress_a", "stress_b", "probe"])
def test_stress_decks_against_oracle(deck_dir, name):
    """Every boundary code over 10 steps.  Longer runs of these decks are not a
    precision measure: a KLAS 6 weir between two nearly equal levels has a flux
    proportional to (dz/sh)^0.33333 (functors.cu:297-316), whose derivative
    grows without bound as dz -> 0, so any rounding difference there (the
    reference's own fp32 build included) is amplified to 1e-3..1e-1 within
    50 steps."""
    deck = hb.Deck(deck_dir[name])
    o = O.OracleDeck(deck_dir[name])
    sp = hb.Solver(deck, precision="split")
    o.run(10)
    sp.step(10)
    sp.sync()
    e = depth_error(sp.get_state()["H"], o.dump()["H"], deck.mesh.hm2)
    assert e["rel_max"] <= 5e-6, e


def test_host_and_device_entry_points_agree(deck_dir):
    """hb_step_host (state through host buffers) equals hb_step + hb_get_state."""
    deck = hb.Deck(deck_dir["stress_a"])
    a = hb.Solver(deck, precision="split")
    b = hb.Solver(deck, precision="split")
    a.step(10)
    a.sync()
    ref = a.get_state()
    st = deck.state()
    arrs = {k: st[k].copy() for k in "HUVZW"}
    b.step_host(arrs["H"], arrs["U"], arrs["V"], arrs["Z"], arrs["W"], 10)
    b.sync()
    # the host round trip re-encodes the state once, at the start
    for k in "HUVZW":
        np.testing.assert_array_equal(arrs[k], ref[k], err_msg=k)


def test_tile_configs_bit_identical(deck_dir):
    """Every launch shape of both layouts gives the same split-precision bits
    (no atomics in any sum)."""
    deck = hb.Deck(deck_dir["stress_b"])
    ref = None
    for cfg, shape in hb.launch_shapes().items():
        s = hb.Solver(deck, precision="split", tile_config=cfg, layout=shape["layout"], tile_cells=64)
        s.step(20)
        s.sync()
        h = s.get_state()["H"]
        if ref is None:
            ref = h
        else:
            np.testing.assert_array_equal(h, ref, err_msg=f"tile_config {cfg}")
        s.close()


def test_device_state_views(deck_dir):
    """Zero-copy views of the split state: fp32 H, U, V and the depth's low part;
    H + H_lo is the depth hb_get_state reports for wet cells."""
    import torch
    deck = hb.Deck(deck_dir["f1"])
    s = hb.Solver(deck, precision="split")
    s.step(5)
    s.sync()
    v = s.device_state()
    assert set(v) == {"H", "U", "V", "H_lo", "W"}
    assert v["H"].dtype == torch.float32
    perm = s.permutation()
    st = s.get_state()
    depth = v["H"].cpu().numpy().astype(np.float64) + v["H_lo"].cpu().numpy().astype(np.float64)
    np.testing.assert_array_equal(depth, st["H"][perm])
