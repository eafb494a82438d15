"""The complex-step reference of the gradient (oracle/complex_step.py), CPU.

Pinned two ways before the GPU adjoint is checked against it:
  * its real part is the timestep: after 30 steps of the F1 channel deck its
    state is within 1e-12 (normwise) of the C oracle's;
  * its derivative is the loss's: along seeded directions of n and ZBC it
    agrees with fourth-order central differences of its own real run to 1e-6.
"""
import numpy as np
import pytest

import hydrob200 as hb
from hydrob200 import deck as D
from oracle import complex_step as CS
from oracle import oracle as O


@pytest.fixture(scope="module")
def f1_deck(tmp_path_factory):
    root = str(tmp_path_factory.mktemp("f1cs") / "deck")
    D.write_deck(D.config_f1(steps=60), root)
    return root


def _setup(root):
    deck = hb.Deck(root)
    d = CS.ComplexDeck(deck)
    st = deck.state()
    n0 = np.sqrt(deck.array("fnc") / 9.81).copy()
    return deck, d, st, n0, deck.array("zbc").copy()


def fd4(loss, eps):
    """Fourth-order central difference of loss(s) at s = 0."""
    return (8.0 * (loss(eps) - loss(-eps)) - (loss(2 * eps) - loss(-2 * eps))) / (12.0 * eps)


def test_real_part_matches_the_oracle(f1_deck):
    deck, d, st, n0, zbc = _setup(f1_deck)
    (H, U, V, Z), _ = CS.rollout(d, n0, zbc, st["Z"], st["U"], st["V"], 30)
    o = O.OracleDeck(f1_deck)
    o.run(30)
    od = o.dump()
    for k, a in zip("HUVZ", (H, U, V, Z)):
        ref = od[k]
        assert np.max(np.abs(np.real(a) - ref)) / np.max(np.abs(ref)) <= 1e-12, k


def test_complex_step_matches_finite_differences(f1_deck):
    deck, d, st, n0, zbc = _setup(f1_deck)
    rng = np.random.default_rng(7)
    gauges = rng.choice(deck.cells, 10, replace=False)
    n_true = n0 * np.exp(0.2 * rng.standard_normal(deck.cells))
    _, obs = CS.rollout(d, n_true, zbc, st["Z"], st["U"], st["V"], 30, gauges, 10)
    obs = np.real(obs)
    for vn, vz in ((rng.standard_normal(deck.cells), None), (None, rng.standard_normal(deck.cells))):
        L, dd = CS.directional_derivative(d, n0, zbc, st["Z"], st["U"], st["V"], gauges, obs, 10, 30, vn, vz)
        eps = 1e-3 * (np.max(np.abs(n0)) if vn is not None else 1.0)

        def loss(s):
            nn = n0 + s * vn if vn is not None else n0
            zz = zbc + s * vz if vz is not None else zbc
            return np.real(CS.gauge_loss(d, nn, zz, st["Z"], st["U"], st["V"], gauges, obs, 10, 30))

        fd = fd4(loss, eps)
        assert abs(fd - dd) <= 1e-6 * abs(dd), (fd, dd)
