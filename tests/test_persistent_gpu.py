"""The persistent step sequence (hb_options.persistent), GPU.

A persistent handle runs a whole step sequence as one cooperative launch:
flux records, a grid barrier, cells, a grid barrier, and so on.  Each chunk of
records or cells runs exactly as one CTA of the two-kernel sequence does, so
the bar is the same as for the other forms: bit for bit the reference binary's
own dumps (fp64, variants H and F), and bit for bit the two-kernel sequence in
every precision, for single meshes and batches, through graphs.  The barrier
waits are bounded: a barrier that cannot complete (arrivals that never come)
ends the launch with HB_E_BARRIER_TIMEOUT and leaves the GPU usable.
"""
import time

import numpy as np
import pytest

import hydrob200 as hb
from conftest import golden
from hydrob200.golden import DECKS

pytestmark = pytest.mark.gpu

FLUX = ("FLUX0", "FLUX1", "FLUX2", "FLUX3")


def _bits_equal(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return bool(np.all((a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))))


def _same_run(a, b, what, scenario=None):
    kw = {} if scenario is None else {"scenario": scenario}
    sa, sb = a.get_state(**kw), b.get_state(**kw)
    for k in "HUVZW":
        assert _bits_equal(sa[k], sb[k]), f"{what}: {k}"
    fa, fb = a.flux(**kw), b.flux(**kw)
    for k in FLUX:
        assert _bits_equal(fa[k], fb[k]), f"{what}: {k}"
    np.testing.assert_array_equal(a.klas(**kw), b.klas(**kw))


def _fp64_cases():
    for name, spec in DECKS.items():
        if name == "breach":
            continue
        for b in spec["bins"]:
            if b in ("h64", "f64"):
                yield name, b


@pytest.mark.parametrize("name,binary", list(_fp64_cases()))
def test_persistent_matches_reference_dumps(deck_dir, name, binary):
    deck = hb.Deck(deck_dir[name])
    s = hb.Solver(deck, variant="H" if binary == "h64" else "F", persistent=True)
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
            assert _bits_equal(st[k] if k in st else fl[k], g[k]), f"{name}/{binary}/s{steps}/{k}"


@pytest.mark.parametrize("precision,variant", [("fp64", "H"), ("fp64", "F"), ("split", "H"), ("fp32", "H")])
@pytest.mark.parametrize("name", ["stress_a", "probe", "f1"])
def test_persistent_equals_two_kernel_sequence(deck_dir, name, precision, variant):
    deck = hb.Deck(deck_dir[name])
    two = hb.Solver(deck, precision=precision, variant=variant)
    one = hb.Solver(deck, precision=precision, variant=variant, persistent=True)
    for n in (1, 6, 13, 30):   # sequences of one and of many steps, across table intervals
        two.step(n)
        one.step(n)
        two.sync()
        one.sync()
        _same_run(one, two, f"{name}/{precision}/{variant} after +{n}")
    assert one.position == two.position


def test_persistent_breach_deck(deck_dir):
    """KLAS 7 turns into 0 once breached; the record's code byte changes inside the launch."""
    deck = hb.Deck(deck_dir["breach"])
    two = hb.Solver(deck)
    one = hb.Solver(deck, persistent=True)
    two.step(1)
    one.step(1)
    _same_run(one, two, "breach")


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_persistent_batch_equals_two_kernel_batch(deck_dir, precision):
    names = ["stress_a", "f1", "stress_b", "probe"]
    decks = [hb.Deck(deck_dir[n]) for n in names]
    two = hb.Batch(decks, precision=precision)
    one = hb.Batch(decks, precision=precision, persistent=True)
    for n in (1, 49):
        two.step(n)
        one.step(n)
        two.sync()
        one.sync()
        for i in range(len(decks)):
            _same_run(one, two, f"batch {names[i]} after +{n}", scenario=i)


def test_persistent_graph_replay(deck_dir):
    """A captured graph (barrier reset, cooperative launch, counter tick)
    replayed three times equals 30 plain steps: the boundary time advances."""
    deck = hb.Deck(deck_dir["stress_a"])
    ref = hb.Solver(deck)
    ref.step(30)
    ref.sync()
    s = hb.Solver(deck, persistent=True)
    s.capture_graph(10)
    for _ in range(3):
        s.graph_launch()
    s.sync()
    assert s.position == ref.position
    _same_run(s, ref, "graph x3")


def test_persistent_barrier_timeout_is_a_status(deck_dir):
    """Every barrier also waits for one arrival that never comes: the first
    wait runs out after its 20 ms bound, every CTA leaves the launch, and
    hb_sync returns HB_E_BARRIER_TIMEOUT.  The GPU stays usable: a new
    persistent handle then steps bit for bit like the two-kernel sequence."""
    deck = hb.Deck(deck_dir["stress_a"])
    s = hb.Solver(deck, persistent=True)
    s.set_barrier_limit(20_000_000, phantom_arrivals=1)
    t0 = time.perf_counter()
    s.step(3)
    with pytest.raises(hb.HydroError) as e:
        s.sync()
    assert e.value.status == 5   # HB_E_BARRIER_TIMEOUT
    assert time.perf_counter() - t0 < 10.0
    assert s.device_errors() & (1 << 5)
    s.close()
    two = hb.Solver(deck)
    one = hb.Solver(deck, persistent=True)
    two.step(5)
    one.step(5)
    two.sync()
    one.sync()
    _same_run(one, two, "after a timed-out launch")


def test_persistent_handle_steps_again_after_a_timeout(deck_dir):
    """The give-up flag is per launch: after a launch timed out, the same
    handle (its sticky error bit still set, so hb_sync keeps reporting the
    timeout) runs its next launches to the end once the phantom arrival is
    gone, bit for bit like the two-kernel sequence from the same state."""
    deck = hb.Deck(deck_dir["stress_a"])
    s = hb.Solver(deck, persistent=True)
    s.set_barrier_limit(20_000_000, phantom_arrivals=1)
    s.step(2)
    with pytest.raises(hb.HydroError):
        s.sync()
    s.set_barrier_limit(1_000_000_000, phantom_arrivals=0)
    st = deck.state()
    s.set_position(0)
    s.set_state(st["H"], st["U"], st["V"], st["Z"], st["W"])
    t0 = time.perf_counter()
    s.step(6)
    with pytest.raises(hb.HydroError) as e:
        s.sync()
    assert e.value.status == 5 and time.perf_counter() - t0 < 5.0
    two = hb.Solver(deck)
    two.step(6)
    two.sync()
    a, b = s.get_state(), two.get_state()
    for k in "HUVZW":
        assert _bits_equal(a[k], b[k]), k


def test_persistent_handle_arguments(deck_dir):
    deck = hb.Deck(deck_dir["stress_a"])
    s = hb.Solver(deck, persistent=True)
    with pytest.raises(hb.HydroError) as e:
        s.tile_config = 2
    assert e.value.status == 1
    s.tile_config = 1   # the default edge shape
    with pytest.raises(hb.HydroError) as e:
        s.autotune(2)
    assert e.value.status == 1
    for bad in ((0, 0), (-1, 0), (20_000_000_000, 0), (1_000_000, -1)):
        with pytest.raises(hb.HydroError):
            s.set_barrier_limit(*bad)


@pytest.mark.parametrize("persistent", [False, True])
def test_step_host_block_rows_equal_device_steps(deck_dir, persistent):
    """hb_step_host with H, U, V, Z as the rows of one [4][CELL] host block
    (moved as one copy each way) and W omitted, one step per call, equals
    hb_step + hb_get_state bit for bit (fp64)."""
    deck = hb.Deck(deck_dir["stress_a"])
    a = hb.Solver(deck)
    a.step(6)
    a.sync()
    ref = a.get_state()
    b = hb.Solver(deck, persistent=persistent)
    st = deck.state()
    block = np.stack([st[k] for k in "HUVZ"]).copy()
    for _ in range(6):
        b.step_host(block[0], block[1], block[2], block[3], None, 1)
    b.sync()
    for i, k in enumerate("HUVZ"):
        assert _bits_equal(block[i], ref[k]), k
    assert _bits_equal(b.get_state()["W"], ref["W"])


@pytest.mark.parametrize("persistent", [False, True])
def test_step_host_page_locked_graph_equals_device_steps(deck_dir, persistent):
    """hb_step_host with page-locked buffers (as the end-to-end bench passes
    them), switching buffers, step counts per call, W and the launch shape
    between calls: every call equals hb_step + hb_get_state bit for bit (fp64)."""
    import torch
    deck = hb.Deck(deck_dir["f1"])
    a = hb.Solver(deck)
    b = hb.Solver(deck, persistent=persistent)
    st = deck.state()
    C = deck.cells
    blk1 = torch.empty((4, C), dtype=torch.float64).pin_memory()
    blk2 = torch.empty((4, C), dtype=torch.float64).pin_memory()
    w = torch.empty(C, dtype=torch.float64).pin_memory()
    for i, k in enumerate("HUVZ"):
        blk1[i].copy_(torch.from_numpy(st[k]))
    done = 0
    # (buffer, steps per call, calls), then a new step count, a new buffer with W,
    # and a launch-shape change
    plan = [(blk1, 1, 4), (blk1, 3, 2), (blk2, 1, 2), (blk2, 2, 2), ("shape", 0, 0), (blk2, 2, 2)]
    cur = blk1
    for buf, n, calls in plan:
        if isinstance(buf, str):
            if not persistent:
                b.tile_config = 2
            continue
        if buf is not cur:
            buf.copy_(cur)
            cur = buf
        for c in range(calls):
            b.step_host(buf[0], buf[1], buf[2], buf[3], w if buf is blk2 else None, n)
            done += n
        b.sync()
        a.step(n * calls)
        a.sync()
        ref = a.get_state()
        for i, k in enumerate("HUVZ"):
            assert _bits_equal(buf[i].numpy(), ref[k]), f"{k} after {done} steps"
        if buf is blk2:
            assert _bits_equal(w.numpy(), ref["W"])
    assert b.position == a.position
