"""The CPU oracle, pinned against the reference binary's own dumps (CPU only).

The fixtures in tests/golden were produced on a B200 by the reference's
dump driver (cuda_native_impl/benchmark.cu:131-169) built from its own sources
(oracle/ref.mk), on the seeded decks of hydrob200.golden.DECKS
(tests/golden/make_golden.py).
"""
import ctypes

import numpy as np
import pytest

from conftest import golden
from hydrob200.golden import DECKS, deck_digest
from oracle import oracle as O

STATE = ("H", "U", "V", "Z")


def normwise(a, b):
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def test_generator_is_deterministic(deck_dir, manifest):
    """The decks written here are byte-identical to the ones the goldens were made from."""
    for name, path in deck_dir.items():
        assert deck_digest(path) == manifest["decks"][name]["sha256"], name


def test_golden_digests(manifest):
    """Every committed fixture array still hashes to what the generating run recorded."""
    import hashlib
    for key, digests in manifest["dumps"].items():
        name, b, s = key.split("__")
        g = golden(name, b, int(s[1:]))
        for k in g.files:
            assert hashlib.sha256(np.ascontiguousarray(g[k]).tobytes()).hexdigest() == digests[k], (key, k)


@pytest.fixture()
def pattern_guard():
    """Restores the oracle's rounding pattern after a test changes it."""
    lib = O.lib()
    lib.orc_get_pattern.restype = ctypes.c_int
    lib.orc_set_pattern.argtypes = [ctypes.c_int, ctypes.c_int]
    saved = [lib.orc_get_pattern(i) for i in range(lib.orc_pattern_count())]
    yield lib
    for i, m in enumerate(saved):
        lib.orc_set_pattern(i, m)


def _run_cases():
    for name, spec in DECKS.items():
        if name == "breach":
            continue
        for b in spec["bins"]:
            if b in ("h64", "f64"):
                yield name, b


@pytest.mark.parametrize("name,binary", list(_run_cases()))
def test_oracle_matches_reference_fp64(deck_dir, name, binary):
    """Oracle vs reference fp64 build.

    Step 1: normwise relative error <= 1e-14 on every dumped array and at
    least 90 % of all values bit-identical (what differs is CUDA's pow versus
    glibc's, 1-2 ulp). Later steps: H/U/V/Z within 1e-12 on the benchmark's
    channel deck, within 1e-11 on the stress decks, whose dry fronts and
    jets amplify those pow ulps, and 1e-10 on the probe deck, whose boundary
    tables jump by orders of magnitude between intervals.
    """
    o = O.OracleDeck(deck_dir[name], O.VARIANT_H if binary == "h64" else O.VARIANT_F)
    done = 0
    for steps in DECKS[name]["steps"]:
        o.run(steps - done)
        done = steps
        g = golden(name, binary, steps)
        d = o.dump()
        assert o.error == 0
        if steps == 1:
            for k in g.files:
                assert normwise(d[k], g[k]) <= 1e-14, (name, binary, k)
            frac = np.mean([np.mean(d[k] == g[k]) for k in g.files])
            assert frac >= 0.9, frac
        else:
            tol = {"f1": 1e-12, "probe": 1e-10}.get(name, 1e-11)
            for k in STATE:
                assert normwise(d[k], g[k]) <= tol, (name, binary, steps, k)


def test_oracle_geometry_exact(deck_dir):
    """SIDE, SLCOS, SLSIN (host preprocessing, mesh.cpp:280-372) are bit-identical."""
    for name in ("stress_a", "stress_b", "breach"):
        o = O.OracleDeck(deck_dir[name])
        g = golden(name, "h64", 1)
        d = o.dump()
        for k in ("SIDE", "SLCOS", "SLSIN"):
            assert np.array_equal(d[k], g[k]), (name, k)


def test_planted_rounding_mistake_is_caught(deck_dir, pattern_guard):
    """Plant a wrong fusion choice in the oracle: step-1 fluxes stop matching bit for bit."""
    lib = pattern_guard
    name = "stress_a"
    g = golden(name, "h64", 1)
    o = O.OracleDeck(deck_dir[name]); o.run(1)
    good = np.mean(o.dump()["FLUX2"] == g["FLUX2"])
    lib.orc_set_pattern(1, 0)   # P_QL2: round both products instead of fusing
    o2 = O.OracleDeck(deck_dir[name]); o2.run(1)
    bad = np.mean(o2.dump()["FLUX2"] == g["FLUX2"])
    assert good == 1.0 and bad < 0.99, (good, bad)


def test_planted_physics_mistake_is_caught(deck_dir, pattern_guard):
    """Plant a wrong value in the oracle's state: the step-1 comparison fails loudly."""
    name = "f1"
    o = O.OracleDeck(deck_dir[name])
    h = o.arr("h")
    h[123] *= 1.0 + 1e-9
    o.run(1)
    g = golden(name, "h64", 1)
    assert normwise(o.dump()["H"], g["H"]) > 1e-14


def test_fp32_reference_close_to_fp64(deck_dir):
    """The reference's own fp32 build stays within 1e-5 (relative, H) of its fp64 build on the channel deck."""
    for steps in (1, 50, 100):
        g32, g64 = golden("f1", "h32", steps), golden("f1", "h64", steps)
        assert normwise(g32["H"].astype(np.float64), g64["H"]) <= 1e-5


def test_breach_reference_reads_uninitialised_depth(deck_dir):
    """The reference's KLAS=7 branch uses an uninitialised HB (functors.cu:246-247): on the B200
    build its FLUX1/FLUX3 come out NaN. The oracle uses the cell depth instead; everything the
    breach does not touch still matches."""
    o = O.OracleDeck(deck_dir["breach"])
    k0 = o.arr("klas").copy()
    o.run(1)
    g = golden("breach", "h64", 1)
    d = o.dump()
    br = np.nonzero(k0 == 7)[0]
    assert br.size > 0
    assert np.all(np.isnan(g["FLUX1"][br])) and np.all(np.isfinite(d["FLUX1"][br]))
    assert np.all(o.arr("klas")[br] == 0)
    cells = np.unique(br // 4)
    keep = np.ones(o.cells, bool); keep[cells] = False
    for k in ("U", "V"):
        assert normwise(d[k][keep], g[k][keep]) <= 1e-14
    assert normwise(d["H"], g["H"]) <= 1e-14


def test_frozen_iteration_counts_replay_exactly(deck_dir):
    """The oracle's gauge rollout with the boundary fixed points' iteration
    counts recorded (mode 1) and then replayed (mode 2) at the same parameters
    gives the free run's depths bit for bit; the recorded counts are those of
    the KLAS 1 / 10 slots only, within the loops' limits."""
    import hydrob200 as hb
    deck = hb.Deck(deck_dir["f1"])
    o = O.OracleDeck(deck_dir["f1"])
    st = deck.state()
    n = np.sqrt(deck.array("fnc") / 9.81)
    zbc = deck.array("zbc").copy()
    gauges = np.arange(0, deck.cells, 97)
    T = 40
    free = o.gauge_rollout(n, zbc, st["Z"], st["U"], st["V"], gauges, 5, T)
    counts = np.zeros((T, 4 * deck.cells), np.int8)
    rec = o.gauge_rollout(n, zbc, st["Z"], st["U"], st["V"], gauges, 5, T, counts, 1)
    rep = o.gauge_rollout(n, zbc, st["Z"], st["U"], st["V"], gauges, 5, T, counts, 2)
    assert np.array_equal(free, rec) and np.array_equal(free, rep)
    klas = deck.array("klas")
    used = np.nonzero(counts.any(axis=0))[0]
    assert used.size > 0 and set(np.unique(klas[used]).tolist()) <= {1.0, 10.0}
    assert counts.min() >= 0 and counts.max() <= 30
