"""hb_write_dump writes the reference driver's --dump file (GPU).

The goldens are the reference binary's own dumps (benchmark.cu:141-162), so a
dump written by the library after the same steps must read back to the same
values, bit for bit in fp64, through the same reader.
"""
import numpy as np
import pytest

import hydrob200 as hb
from conftest import golden
from hydrob200.golden import DECKS, read_dump

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,binary,steps", [("stress_a", "h64", 10), ("f1", "h64", 50), ("stress_b", "f64", 50)])
def test_dump_reads_back_as_the_reference_dump(deck_dir, tmp_path, name, binary, steps):
    deck = hb.Deck(deck_dir[name])
    s = hb.Solver(deck, variant="H" if binary == "h64" else "F")
    s.step(steps)
    s.sync()
    path = str(tmp_path / "dump.bin")
    s.write_dump(path)
    d = read_dump(path, np.float64)
    g = golden(name, binary, steps)
    for k in g.files:
        a, b = d[k], g[k]
        same = (a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))
        assert same.all(), f"{name}/{binary}/s{steps}/{k}"


def test_batch_dump_per_scenario(deck_dir, tmp_path):
    decks = [hb.Deck(deck_dir[n]) for n in ("stress_a", "f1")]
    b = hb.Batch(decks)
    b.step(10)
    b.sync()
    for i, n in enumerate(("stress_a", "f1")):
        path = str(tmp_path / f"{n}.bin")
        b.write_dump(path, scenario=i)
        d = read_dump(path, np.float64)
        st = b.get_state(i)
        for k in "HUVZ":
            np.testing.assert_array_equal(d[k], st[k])
