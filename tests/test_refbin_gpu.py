"""Parity against the reference program itself, run beside this library (GPU).

The golden fixtures pin the small decks; these tests pin the configurations
the measurements run on, and the reference's own shipped decks, by running
the reference's dump driver (cuda_native_impl/benchmark.cu:131-169, built
from the reference sources by oracle/ref.mk into oracle/_ref) on the same
deck files in the same session:

* the 207,234-cell benchmark channel and the 24,020-cell adjoint channel
  (hydrob200.deck.config_207k / config_24k);
* the reference's decks data/F1_text (6,675 quad cells, KLAS 4/10/13) and
  data/F2_24K_text (24,020 cells, KLAS 1/4), packed as tests/golden fixtures.

Bar, fp64 variants H and F: H, U, V, Z and FLUX0..3 bit-identical to the
reference's own fp64 build after step 1 and after step 50, through the
handle path (and the drop-in path for variant H).  fp32: H within 1e-5
(normwise relative) of the reference's fp32 build and of its fp64 build
after 50 steps.  Skipped where the reference programs are not built.
"""
import os
import subprocess

import numpy as np
import pytest

import hydrob200 as hb
from hydrob200 import deck as D
from hydrob200.golden import read_dump

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFBIN = {b: os.path.join(ROOT, "oracle", "_ref", f"ref_{b}") for b in ("h64", "f64", "h32")}
STATE = ("H", "U", "V", "Z")
FLUX = ("FLUX0", "FLUX1", "FLUX2", "FLUX3")
STEPS = (1, 50)

need_ref = pytest.mark.skipif(not all(os.path.exists(p) for p in REFBIN.values()),
                              reason="reference programs not built (oracle/ref.mk)")


def ref_dump(binary: str, root: str, steps: int):
    """The reference driver's --dump after `steps` steps on the deck at `root` (run from root/run)."""
    run = os.path.join(root, "run")
    os.makedirs(run, exist_ok=True)
    out = os.path.join(run, f"{os.path.basename(REFBIN[binary])}_{steps}.bin")
    if not os.path.exists(out):
        r = subprocess.run([REFBIN[binary], str(steps), "1", "--dump", out], cwd=run, capture_output=True,
                           text=True, timeout=900)
        assert r.returncode == 0, r.stdout[-1500:] + r.stderr[-1500:]
    return read_dump(out, np.float32 if binary.endswith("32") else np.float64)


def assert_bits(got, ref, what):
    a, b = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    same = (a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))
    if not same.all():
        idx = np.nonzero(~same)[0]
        rel = float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))
        raise AssertionError(f"{what}: {idx.size}/{a.size} differ (normwise {rel:.3g}), first {idx[:5]} "
                             f"got {a[idx[:3]]} ref {b[idx[:3]]}")


def normwise(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


@pytest.fixture(scope="module")
def decks(tmp_path_factory, ref_deck_dir):
    base = tmp_path_factory.mktemp("refbin")
    out = dict(ref_deck_dir)
    for name, make in (("c207k", lambda: D.config_207k(steps=60)), ("c24k", lambda: D.config_24k(steps=60))):
        root = str(base / name)
        D.write_deck(make(), root)
        out[name] = root
    return out


CASES = [(n, b) for n in ("c207k", "c24k", "ref_f1", "ref_f2_24k") for b in ("h64", "f64")]


@need_ref
@pytest.mark.parametrize("name,binary", CASES)
def test_fp64_bit_exact_against_the_reference_program(decks, name, binary):
    root = decks[name]
    deck = hb.Deck(root)
    s = hb.Solver(deck, variant="H" if binary == "h64" else "F")
    r = hb.RefLayoutMesh(deck) if binary == "h64" else None
    done = 0
    for steps in STEPS:
        s.step(steps - done)
        if r is not None:
            r.run(steps - done)
        done = steps
        g = ref_dump(binary, root, steps)
        st, fl = s.get_state(), s.flux()
        for k in STATE:
            assert_bits(st[k], g[k], f"{name}/{binary}/s{steps}/{k}")
        for k in FLUX:
            assert_bits(fl[k], g[k], f"{name}/{binary}/s{steps}/{k}")
        if r is not None:
            d = r.dump()
            for k in STATE + FLUX:
                assert_bits(d[k], g[k], f"dropin {name}/{binary}/s{steps}/{k}")
    if r is not None:
        assert hb.take_ref_device_errors() == 0


DROPIN = os.path.join(ROOT, "oracle", "_ref", "ref_dropin")


@pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(REFBIN["h64"])),
                    reason="link-level drop-in program not built (oracle/ref.mk)")
@pytest.mark.parametrize("name,steps", [("stress_a", 50), ("f1", 100), ("ref_f1", 50), ("c207k", 50)])
def test_link_level_dropin_program(decks, deck_dir, name, steps):
    """The reference's own driver and host code (benchmark.cu, mesh.cpp,
    cell.cpp, side.cpp) linked against libhydrob200.so in place of
    functors.cu (oracle/ref.mk's ref_dropin): its --dump equals the unmodified
    reference program's bit for bit (state, geometry and fluxes)."""
    root = decks.get(name) or deck_dir[name]
    run = os.path.join(root, "run")
    os.makedirs(run, exist_ok=True)
    out = os.path.join(run, f"dropin_{steps}.bin")
    r = subprocess.run([DROPIN, str(steps), "1", "--dump", out], cwd=run, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0 and "hydrob200:" not in r.stderr, r.stdout[-1500:] + r.stderr[-1500:]
    got = read_dump(out, np.float64)
    ref = ref_dump("h64", root, steps)
    for k in ref:
        assert_bits(got[k], ref[k], f"ref_dropin {name}/s{steps}/{k}")


@need_ref
@pytest.mark.parametrize("name,tile_cells", [("c207k", 0), ("c207k", 512), ("ref_f1", 64)])
def test_tile_layout_bit_exact_against_the_reference_program(decks, name, tile_cells):
    """The tile layout (one kernel per step, slot terms in shared memory)."""
    root = decks[name]
    deck = hb.Deck(root)
    s = hb.Solver(deck, layout="tile", tile_cells=tile_cells)
    done = 0
    for steps in STEPS:
        s.step(steps - done)
        done = steps
        g = ref_dump("h64", root, steps)
        st, fl = s.get_state(), s.flux()
        for k in STATE:
            assert_bits(st[k], g[k], f"tile {name}/s{steps}/{k}")
        for k in FLUX:
            assert_bits(fl[k], g[k], f"tile {name}/s{steps}/{k}")


@need_ref
@pytest.mark.parametrize("name", ["c207k", "ref_f2_24k"])
def test_fp32_against_the_reference_fp32_program(decks, name):
    root = decks[name]
    deck = hb.Deck(root)
    s = hb.Solver(deck, precision="fp32")
    s.step(50)
    st = s.get_state()
    g32, g64 = ref_dump("h32", root, 50), ref_dump("h64", root, 50)
    assert normwise(st["H"], g32["H"]) <= 1e-5
    assert normwise(st["H"], g64["H"]) <= 1e-5
