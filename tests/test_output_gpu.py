"""Result files (hb_output_*) against the reference binary's own (GPU).

The reference driver, run with --with-output, writes SIDE.OUT, H2U2V2.OUT,
ZUV.OUT, XY-TEC.DAT and TIMELOG.OUT (mesh.cpp:535-839) at its output cadence
(benchmark.cu:105-124).  The library's writer, fed the library's fp64 states
through the same cadence, must produce the same bytes.  The reference program
is the one oracle/ref.mk builds from the reference sources (oracle/_ref);
the test is skipped where that build is absent.
"""
import os
import shutil
import subprocess

import pytest

import hydrob200 as hb
from hydrob200.output import run_with_output

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "ref_h64")
FILES = ("SIDE.OUT", "H2U2V2.OUT", "ZUV.OUT", "XY-TEC.DAT", "TIMELOG.OUT")


@pytest.mark.skipif(not os.path.exists(REF), reason="reference program not built (oracle/ref.mk)")
@pytest.mark.parametrize("name,steps", [("stress_a", 50), ("f1", 100)])
def test_output_files_equal_the_reference_programs(deck_dir, tmp_path, name, steps):
    ref_deck = tmp_path / "ref"
    shutil.copytree(deck_dir[name], ref_deck)
    (ref_deck / "OUTPUT").mkdir(exist_ok=True)
    (ref_deck / "run").mkdir(exist_ok=True)
    r = subprocess.run([REF, str(steps), "1", "--dump", "state.bin", "--with-output"], cwd=ref_deck / "run",
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-1000:] + r.stderr[-1000:]
    deck = hb.Deck(deck_dir[name])
    s = hb.Solver(deck)
    ours = tmp_path / "ours"
    run_with_output(s, deck, str(ours), steps)
    for f in FILES:
        a = (ref_deck / "OUTPUT" / f).read_bytes()
        b = (ours / f).read_bytes()
        assert a == b, f"{name}/{f}: {len(a)} vs {len(b)} bytes, first difference at {next((i for i in range(min(len(a), len(b))) if a[i] != b[i]), min(len(a), len(b)))}"
