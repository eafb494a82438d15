"""The reverse-mode adjoint (hb_adjoint_*) against the complex-step reference
and finite differences, GPU.

Rollout of the F1 channel deck (KLAS 0, 1, 4, 10), gauge loss every 10 steps
against observations from a run with perturbed Manning coefficients.
  * the rollout's gauge depths equal the complex-step reference's real run to
    1e-11 (relative);
  * directional derivatives g . v of the adjoint gradient, for n and for ZBC,
    equal the complex-step reference's to 1e-8 (relative) and fourth-order
    central differences of the GPU rollout itself to 1e-6;
  * the gradient does not depend on the checkpoint interval (bit for bit);
  * the handle holds the plain rollout's final state after the forward, and a
    second backward gives the same gradient;
  * torch.autograd reaches the same gradient through GaugeLoss.
"""
import numpy as np
import pytest

import hydrob200 as hb
from hydrob200 import deck as D
from hydrob200.adjoint import Adjoint, gauge_loss_function
from oracle import complex_step as CS

pytestmark = pytest.mark.gpu

NSTEPS, OBS_EVERY = 40, 10


@pytest.fixture(scope="module")
def setup(tmp_path_factory):
    root = str(tmp_path_factory.mktemp("adj") / "deck")
    D.write_deck(D.config_f1(steps=60), root)
    deck = hb.Deck(root)
    rng = np.random.default_rng(11)
    gauges = rng.choice(deck.cells, 12, replace=False)
    n0 = np.sqrt(deck.array("fnc") / 9.81).copy()
    n_true = n0 * np.exp(0.2 * rng.standard_normal(deck.cells))
    vn = rng.standard_normal(deck.cells)
    vz = rng.standard_normal(deck.cells)
    return dict(root=root, deck=deck, gauges=gauges, n0=n0, n_true=n_true, zbc=deck.array("zbc").copy(), vn=vn, vz=vz)


def _adjoint(s, k=10):
    a = Adjoint(s["deck"], s["gauges"], OBS_EVERY, NSTEPS, checkpoint_every=k)
    a.set_parameters(s["n_true"], s["zbc"])
    _, obs = a.forward()
    a.set_observations(obs)
    a.set_parameters(s["n0"], s["zbc"])
    return a, obs


def fd4(loss, eps):
    return (8.0 * (loss(eps) - loss(-eps)) - (loss(2 * eps) - loss(-2 * eps))) / (12.0 * eps)


def test_rollout_matches_the_complex_step_reference(setup):
    s = setup
    a, obs = _adjoint(s)
    d = CS.ComplexDeck(s["deck"])
    st = s["deck"].state()
    _, gd = CS.rollout(d, s["n_true"], s["zbc"], st["Z"], st["U"], st["V"], NSTEPS, s["gauges"], OBS_EVERY)
    assert np.max(np.abs(np.real(gd) - obs)) / np.max(np.abs(obs)) <= 1e-11
    a.close()


def test_gradient_against_complex_step_and_finite_differences(setup):
    s = setup
    a, obs = _adjoint(s)
    L, _ = a.forward()
    gn, gz = a.backward()
    d = CS.ComplexDeck(s["deck"])
    st = s["deck"].state()
    for name, g, vn, vz, scale in (("n", gn, s["vn"], None, np.max(s["n0"])), ("zbc", gz, None, s["vz"], 1.0)):
        adj = float(g @ (vn if vn is not None else vz))
        Lc, cs = CS.directional_derivative(d, s["n0"], s["zbc"], st["Z"], st["U"], st["V"], s["gauges"], obs,
                                           OBS_EVERY, NSTEPS, vn, vz)
        assert abs(Lc - L) <= 1e-9 * abs(L)
        assert abs(adj - cs) <= 1e-8 * abs(cs), (name, adj, cs)

        def loss(t):
            return a.loss(s["n0"] + t * vn if vn is not None else s["n0"],
                          s["zbc"] + t * vz if vz is not None else s["zbc"])
        fd = fd4(loss, 1e-3 * scale)
        assert abs(adj - fd) <= 1e-6 * abs(fd), (name, adj, fd)
    a.close()


def test_gradient_independent_of_checkpoint_interval(setup):
    s = setup
    grads = []
    for k in (10, 20, 40, 7):
        a, _ = _adjoint(s, k)
        a.forward()
        grads.append(a.backward())
        a.close()
    for gn, gz in grads[1:]:
        np.testing.assert_array_equal(gn, grads[0][0])
        np.testing.assert_array_equal(gz, grads[0][1])


def test_multi_segment_graphs(tmp_path):
    """120 steps: with k = 10 the forward replays one captured graph of ten
    segments and one of a single segment, with k = 7 one of fourteen segments
    and three single ones, with k = 60 single segments only.  The loss, the
    gradient and the final state agree bit for bit."""
    root = str(tmp_path / "deck")
    D.write_deck(D.config_f1(steps=130), root)
    deck = hb.Deck(root)
    gauges = np.random.default_rng(3).choice(deck.cells, 8, replace=False)
    out = []
    for k in (10, 7, 60):
        a = Adjoint(deck, gauges, OBS_EVERY, 120, checkpoint_every=k)
        _, obs = a.forward()
        a.set_observations(obs + 0.01)
        L, _ = a.forward()
        gn, gz = a.backward()
        out.append((L, gn, gz, a.solver.get_state()))
        a.close()
    L0, gn0, gz0, st0 = out[0]
    for L, gn, gz, st in out[1:]:
        assert L == L0
        np.testing.assert_array_equal(gn, gn0)
        np.testing.assert_array_equal(gz, gz0)
        for f in "HUVZ":
            np.testing.assert_array_equal(st[f], st0[f])


def test_final_state_and_repeated_backward(setup):
    """The forward steps its last segment into the segment buffers (outside
    the k-step graph) and leaves the rollout's final state in the handle: the
    same bits as a plain rollout of the handle from the same initial state,
    whether that segment is the whole run (k = 40), a full segment after graph
    replays (k = 10) or a remainder (k = 7).  A second backward without a new
    forward recomputes that segment and gives the same gradient."""
    s = setup
    st = s["deck"].state()
    hm1 = CS.ComplexDeck(s["deck"]).hm1
    H0, U0, V0, Z0 = (np.real(x) for x in CS.initial_state(st["Z"], st["U"], st["V"], s["zbc"], hm1))
    for k in (40, 10, 7):
        a, _ = _adjoint(s, k)
        a.forward()
        after = a.solver.get_state()
        g1 = a.backward()
        g2 = a.backward()
        np.testing.assert_array_equal(g1[0], g2[0])
        np.testing.assert_array_equal(g1[1], g2[1])
        a.solver.set_state(H0, U0, V0, Z0)
        a.solver.set_position(0)
        a.solver.step(NSTEPS)
        plain = a.solver.get_state()
        for f in "HUVZ":
            np.testing.assert_array_equal(after[f], plain[f], err_msg=f"{f}, k = {k}")
        a.close()


def test_autograd_function(setup):
    import torch
    s = setup
    a, _ = _adjoint(s)
    GaugeLoss = gauge_loss_function()
    n = torch.tensor(s["n0"], dtype=torch.float64, requires_grad=True)
    z = torch.tensor(s["zbc"], dtype=torch.float64, requires_grad=True)
    loss = GaugeLoss.apply(n, z, a)
    (2.0 * loss).backward()
    a.forward()
    gn, gz = a.backward()
    np.testing.assert_array_equal(n.grad.numpy(), 2.0 * gn)
    np.testing.assert_array_equal(z.grad.numpy(), 2.0 * gz)
    a.close()


def test_adjoint_configuration_against_frozen_finite_differences(tmp_path):
    """The adjoint configuration: 24,020-cell channel, 1000 steps, 50 gauges
    every 10 steps, observations from n_true = 0.025 exp(0.2 g), gradient at
    n = 0.025, checkpoint intervals 10, 50 and 100 (bit-identical gradients).

    Directional derivatives g . v for n and ZBC against central differences
    of the same rollout on the CPU oracle with the boundary fixed points'
    iteration counts frozen at the base run (oracle gauge_rollout, modes 1/2):
    the adjoint freezes them too, and without freezing the loss is only
    piecewise smooth (a stopping test that flips between the two runs of a
    difference adds a jump).  Bound 1e-6 relative, at two step sizes."""
    from oracle import oracle as O
    d, n_true, gauges = D.adjoint_case(steps=1000)
    root = str(tmp_path / "c24k")
    D.write_deck(d, root)
    deck = hb.Deck(root)
    T, every = 1000, 10
    st = deck.state()
    zbc = deck.array("zbc").copy()
    n0 = np.full(deck.cells, 0.025)
    grads = []
    for k in (10, 50, 100):
        a = Adjoint(deck, gauges, every, T, checkpoint_every=k)
        a.set_parameters(n_true, zbc)
        _, obs = a.forward()
        a.set_observations(obs)
        a.set_parameters(n0, zbc)
        a.forward()
        grads.append(a.backward())
        a.close()
    for gn, gz in grads[1:]:
        np.testing.assert_array_equal(gn, grads[0][0])
        np.testing.assert_array_equal(gz, grads[0][1])
    gn, gz = grads[0]
    o = O.OracleDeck(root)
    counts = np.zeros((T, 4 * deck.cells), np.int8)
    o.gauge_rollout(n0, zbc, st["Z"], st["U"], st["V"], gauges, every, T, counts, 1)

    def loss(n, z):
        g = o.gauge_rollout(n, z, st["Z"], st["U"], st["V"], gauges, every, T, counts, 2)
        r = g - obs
        return float(np.sum(r * r))

    rng = np.random.default_rng(7)
    vn, vz = rng.standard_normal(deck.cells), rng.standard_normal(deck.cells)
    adj_n, adj_z = float(gn @ vn), float(gz @ vz)
    for rel in (1e-4, 1e-5):
        e = rel * 0.025
        fd_n = (loss(n0 + e * vn, zbc) - loss(n0 - e * vn, zbc)) / (2 * e)
        fd_z = (loss(n0, zbc + rel * vz) - loss(n0, zbc - rel * vz)) / (2 * rel)
        assert abs(adj_n - fd_n) <= 1e-6 * abs(fd_n), ("n", rel, adj_n, fd_n)
        assert abs(adj_z - fd_z) <= 1e-6 * abs(fd_z), ("zbc", rel, adj_z, fd_z)


def test_rejects_codes_without_a_reverse(deck_dir):
    deck = hb.Deck(deck_dir["stress_a"])
    with pytest.raises(hb.HydroError):
        Adjoint(deck, [0, 1], 5, 10)


def test_rejects_a_cell_observed_twice(setup):
    """Each gauge is its own cell: the rollout's cell kernels write one gauge
    depth per cell, and the reverse sweep seeds one loss term per cell."""
    g = list(setup["gauges"][:3]) + [setup["gauges"][0]]
    with pytest.raises(hb.HydroError) as e:
        Adjoint(setup["deck"], g, OBS_EVERY, NSTEPS)
    assert e.value.status == 1
