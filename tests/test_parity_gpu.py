"""Parity of the CUDA paths with the reference (GPU).

Bar (fp64, variants H and F): bit-identical to the reference binary's own
dumps at every recorded step (tests/golden), through both entry points:
  * the handle path (hb_create / hb_step / hb_get_state / hb_get_flux),
  * the drop-in path over reference-layout arrays (hb_ref_calculate_flux /
    hb_ref_update_cell, the CalculateFlux/UpdateCell pair).
fp32: within 1e-5 normwise relative of the reference's fp32 build on H and of
its fp64 build on H.  Inputs beyond the goldens are checked against the CPU
oracle: 1e-14 at step 1, 1e-12 after 50 steps on the channel decks.
"""
import numpy as np
import pytest

import hydrob200 as hb
from conftest import golden
from hydrob200 import deck as D
from hydrob200.golden import DECKS
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FLUX = ("FLUX0", "FLUX1", "FLUX2", "FLUX3")


def normwise(a, b):
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def assert_bits(got, ref, what, mask=None):
    a, b = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    if mask is not None:
        a, b = a[mask], b[mask]
    same = (a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))
    if not same.all():
        idx = np.nonzero(~same)[0]
        raise AssertionError(f"{what}: {idx.size}/{a.size} differ, first {idx[:5]} got {a[idx[:3]]} ref {b[idx[:3]]}")


def _fp64_cases():
    for name, spec in DECKS.items():
        if name == "breach":
            continue
        for b in spec["bins"]:
            if b in ("h64", "f64"):
                yield name, b


@pytest.mark.parametrize("layout,tile_cells", [("edge", 0), ("tile", 0), ("tile", 64)])
@pytest.mark.parametrize("name,binary", list(_fp64_cases()))
def test_handle_path_bit_exact(deck_dir, name, binary, layout, tile_cells):
    deck = hb.Deck(deck_dir[name])
    s = hb.Solver(deck, variant="H" if binary == "h64" else "F", layout=layout, tile_cells=tile_cells)
    done = 0
    for steps in DECKS[name]["steps"]:
        s.step(steps - done)
        s.sync()
        done = steps
        g = golden(name, binary, steps)
        st = s.get_state()
        fl = s.flux() if "FLUX0" in g.files else {}
        for k in g.files:
            if k in ("SIDE", "SLCOS", "SLSIN"):
                continue
            assert_bits(st[k] if k in st else fl[k], g[k], f"{name}/{binary}/s{steps}/{k}")


@pytest.mark.parametrize("name,binary", list(_fp64_cases()))
def test_dropin_path_bit_exact(deck_dir, name, binary):
    deck = hb.Deck(deck_dir[name])
    r = hb.RefLayoutMesh(deck, variant="H" if binary == "h64" else "F")
    done = 0
    for steps in DECKS[name]["steps"]:
        r.run(steps - done)
        done = steps
        g = golden(name, binary, steps)
        d = r.dump()
        for k in g.files:
            if k in ("SIDE", "SLCOS", "SLSIN"):
                continue
            assert_bits(d[k], g[k], f"dropin {name}/{binary}/s{steps}/{k}")
    assert hb.take_ref_device_errors() == 0


def test_breach_masked_bit_exact(deck_dir):
    """KLAS=7: the reference computes FLUX1/FLUX3 from an uninitialised depth; everything else is exact."""
    deck = hb.Deck(deck_dir["breach"])
    k0 = deck.array("klas").copy()
    br = np.nonzero(k0 == 7)[0]
    cells = np.unique(br // 4)
    s = hb.Solver(deck)
    s.step(1)
    g = golden("breach", "h64", 1)
    st, fl = s.get_state(), s.flux()
    keep_slot = np.ones(4 * deck.cells, bool); keep_slot[br] = False
    keep_cell = np.ones(deck.cells, bool); keep_cell[cells] = False
    for k in ("FLUX0", "FLUX2"):
        assert_bits(fl[k], g[k], k)
    for k in ("FLUX1", "FLUX3"):
        assert_bits(fl[k], g[k], k, keep_slot)
    assert_bits(st["H"], g["H"], "H")
    assert_bits(st["Z"], g["Z"], "Z")
    for k in ("U", "V"):
        assert_bits(st[k], g[k], k, keep_cell)
    assert np.all(s.klas()[br] == 0)
    r = hb.RefLayoutMesh(deck)
    r.run(1)
    d = r.dump()
    assert np.all(d["KLAS"][br] == 0)
    assert_bits(d["H"], g["H"], "dropin H")


@pytest.mark.parametrize("variant,binary", [("H", "h32"), ("F", "f32")])
def test_fp32_within_tolerance(deck_dir, variant, binary):
    """fp32: H within 1e-5 (normwise relative) of the reference's fp32 and fp64 builds after 50 steps."""
    deck = hb.Deck(deck_dir["stress_a"])
    s = hb.Solver(deck, variant=variant, precision="fp32")
    r = hb.RefLayoutMesh(deck, variant=variant, precision="fp32")
    s.step(50)
    r.run(50)
    g32 = golden("stress_a", binary, 50)
    g64 = golden("stress_a", "h64" if variant == "H" else "f64", 50)
    for st in (s.get_state(), r.dump()):
        assert normwise(st["H"], g32["H"].astype(np.float64)) <= 1e-5
        assert normwise(st["H"], g64["H"]) <= 1e-5
        for k in ("U", "V"):
            assert normwise(st[k], g64[k]) <= 1e-3


def test_fp32_channel_deck(deck_dir):
    deck = hb.Deck(deck_dir["f1"])
    s = hb.Solver(deck, precision="fp32")
    s.step(100)
    st = s.get_state()
    g64 = golden("f1", "h64", 100)
    assert normwise(st["H"], g64["H"]) <= 1e-5


@pytest.mark.parametrize("seed", [101, 202])
@pytest.mark.parametrize("variant", ["H", "F"])
def test_new_inputs_against_oracle(tmp_path, seed, variant):
    """Seeded stress decks that have no golden: GPU vs the CPU oracle."""
    d = D.stress_deck(f"s{seed}", 18, 9, seed, steps=30, mdt=20)
    root = str(tmp_path / "deck")
    D.write_deck(d, root)
    deck = hb.Deck(root)
    s = hb.Solver(deck, variant=variant)
    r = hb.RefLayoutMesh(deck, variant=variant)
    o = O.OracleDeck(root, O.VARIANT_H if variant == "H" else O.VARIANT_F)
    s.step(1); r.run(1); o.run(1)
    od = o.dump()
    st, fl, rd = s.get_state(), s.flux(), r.dump()
    for k in ("H", "U", "V", "Z"):
        assert normwise(st[k], od[k]) <= 1e-14, k
        assert_bits(rd[k], st[k], f"dropin vs handle {k}")
    for k in FLUX:
        assert normwise(fl[k], od[k]) <= 1e-14, k
        assert_bits(rd[k], fl[k], f"dropin vs handle {k}")
    s.step(29); r.run(29); o.run(29)
    st, rd, od = s.get_state(), r.dump(), o.dump()
    for k in ("H", "U", "V", "Z"):
        assert normwise(st[k], od[k]) <= 1e-11, k
        assert_bits(rd[k], st[k], f"dropin vs handle {k} s30")


def test_graph_replay_advances_time(deck_dir):
    """A captured 10-step graph replayed 5 times equals 50 plain steps and the reference at step 50."""
    deck = hb.Deck(deck_dir["stress_a"])
    a = hb.Solver(deck)
    a.capture_graph(10)
    for _ in range(5):
        a.graph_launch()
    a.sync()
    assert a.position == (50, 1 + 50 % 19, 50 // 19)
    g = golden("stress_a", "h64", 50)
    st, fl = a.get_state(), a.flux()
    for k in ("H", "U", "V", "Z"):
        assert_bits(st[k], g[k], k)
    for k in FLUX:
        assert_bits(fl[k], g[k], k)


def test_renumbering_changes_no_bit(deck_dir):
    deck = hb.Deck(deck_dir["stress_b"])
    a = hb.Solver(deck, renumber=True)
    b = hb.Solver(deck, renumber=False)
    p = a.permutation()
    assert sorted(p.tolist()) == list(range(deck.cells)) and not np.array_equal(p, np.arange(deck.cells))
    a.step(50); b.step(50)
    sa, sb = a.get_state(), b.get_state()
    for k in "HUVZW":
        assert_bits(sa[k], sb[k], k)


def test_state_roundtrip_and_position(deck_dir):
    deck = hb.Deck(deck_dir["stress_a"])
    a = hb.Solver(deck)
    a.step(10)
    st = a.get_state()
    b = hb.Solver(deck)
    b.set_position(10)
    b.set_state(st["H"], st["U"], st["V"], st["Z"], st["W"])
    a.step(40); b.step(40)
    g = golden("stress_a", "h64", 50)
    for s in (a, b):
        x = s.get_state()
        for k in ("H", "U", "V", "Z"):
            assert_bits(x[k], g[k], k)


def test_device_state_views(deck_dir):
    import torch
    deck = hb.Deck(deck_dir["f1"])
    s = hb.Solver(deck)
    s.step(3)
    s.sync()
    v = s.device_state()
    perm = s.permutation()
    st = s.get_state()
    assert v["H"].device.type == "cuda" and v["H"].dtype == torch.float64
    assert np.array_equal(v["H"].cpu().numpy(), st["H"][perm])


def test_errors_are_statuses(deck_dir):
    deck = hb.Deck(deck_dir["stress_a"])
    s = hb.Solver(deck)
    limit = deck.mesh.ndays * (deck.mesh.steps_per_day - 1)
    with pytest.raises(hb.HydroError) as e:
        s.step(limit + 1)
    assert e.value.status == 1
    nac = deck.array("nac")
    saved = nac[5]
    nac[5] = deck.cells + 10     # neighbour out of range
    try:
        with pytest.raises(hb.HydroError) as e:
            hb.Solver(deck)
        assert e.value.status == 2
    finally:
        nac[5] = saved


def test_channel_207k_paths_agree_and_match_oracle(tmp_path):
    """The 207,234-cell benchmark deck: handle path == drop-in path bit for bit after 120 steps
    (crossing two boundary-table intervals); both within 1e-12 of the CPU oracle after 10 steps."""
    d = D.config_207k(steps=120)
    root = str(tmp_path / "c207k")
    D.write_deck(d, root)
    deck = hb.Deck(root)
    s = hb.Solver(deck)
    r = hb.RefLayoutMesh(deck)
    o = O.OracleDeck(root)
    s.step(10); r.run(10); o.run(10)
    od, st = o.dump(), s.get_state()
    for k in ("H", "U", "V", "Z"):
        assert normwise(st[k], od[k]) <= 1e-12, k
    s.step(110); r.run(110)
    st, rd = s.get_state(), r.dump()
    for k in ("H", "U", "V", "Z", "W"):
        assert_bits(st[k], rd[k], k)
    fl = s.flux()
    for k in FLUX:
        assert_bits(fl[k], rd[k], k)
