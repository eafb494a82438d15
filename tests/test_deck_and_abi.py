"""Host logic of the library on CPU: the deck reader against the oracle's
reader, error statuses, and the C ABI's exported symbols."""
import os
import re
import shutil

import numpy as np
import pytest

import hydrob200 as hb
from hydrob200 import _lib
from hydrob200 import deck as D
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

ARRAYS = ("nac", "klas", "side", "cosf", "sinf", "slcos", "slsin", "zbc", "zb1", "area", "fnc", "bfeat",
          "qt", "dqt", "zt", "dzt", "zw", "qw", "nhq1")


@pytest.mark.parametrize("name", ["stress_a", "stress_b", "breach", "f1"])
def test_reader_matches_oracle_reader(deck_dir, name):
    """hb_deck_load and the oracle's restatement of mesh.cpp/cell.cpp agree bit for bit."""
    d = hb.Deck(deck_dir[name])
    o = O.OracleDeck(deck_dir[name])
    for k in ARRAYS:
        a, b = d.array(k), o.arr(k)
        assert a.shape == b.shape and np.array_equal(a, b), k
    st = d.state()
    for k in "HUVZW":
        assert np.array_equal(st[k], o.arr(k.lower())), k
    assert d.mesh.steps_per_day == int(o.scalars["mdt"] / o.scalars["dt"])


@pytest.mark.parametrize("name", ["ref_f1", "ref_f2_24k"])
def test_reader_on_the_reference_decks(ref_deck_dir, name):
    """The reference's own shipped decks (data/F1_text with the F1_native_data
    time files, data/F2_24K_text) load through hb_deck_load unchanged and give
    the oracle reader's arrays bit for bit; the fixtures are the packed bytes."""
    import hashlib
    import json
    with open(os.path.join(ROOT, "tests", "golden", "ref_decks.json")) as f:
        pinned = json.load(f)[name]
    h = hashlib.sha256()
    root = ref_deck_dir[name]
    files = sorted(os.path.relpath(os.path.join(dp, fn), root) for dp, _, fns in os.walk(root) for fn in fns)
    for rel in files:
        h.update(rel.encode())
        with open(os.path.join(root, rel), "rb") as f:
            h.update(f.read())
    assert len(files) == pinned["files"] and h.hexdigest() == pinned["sha256"]
    d = hb.Deck(root)
    o = O.OracleDeck(root)
    for k in ARRAYS:
        a, b = d.array(k), o.arr(k)
        assert a.shape == b.shape and np.array_equal(a, b), k
    st = d.state()
    for k in "HUVZW":
        assert np.array_equal(st[k], o.arr(k.lower())), k
    klas = d.array("klas")
    counts = {int(v): int((klas == v).sum()) for v in np.unique(klas)}
    expect = {"ref_f1": {0: 25972, 4: 708, 10: 8, 13: 12}, "ref_f2_24k": {0: 94332, 1: 169, 4: 1579}}[name]
    assert counts == expect
    assert d.cells == {"ref_f1": 6675, "ref_f2_24k": 24020}[name]


def test_reader_missing_file_is_io_error(deck_dir, tmp_path):
    root = tmp_path / "broken"
    shutil.copytree(deck_dir["stress_a"], root)
    os.remove(root / "SOURCES" / "PNAC.DAT")
    with pytest.raises(hb.HydroError) as e:
        hb.Deck(str(root))
    assert e.value.status == 6   # HB_E_IO


def test_reader_bad_node_is_badmesh(deck_dir, tmp_path):
    root = tmp_path / "badnode"
    shutil.copytree(deck_dir["stress_a"], root)
    p = root / "SOURCES" / "PNAP.DAT"
    lines = p.read_text().splitlines()
    parts = lines[1].split()
    parts[1] = "999999"
    lines[1] = " ".join(parts)
    p.write_text("\n".join(lines) + "\n")
    with pytest.raises(hb.HydroError) as e:
        hb.Deck(str(root))
    assert e.value.status == 2   # HB_E_BADMESH


def test_reader_rating_table_too_long_is_badmesh(deck_dir, tmp_path):
    root = tmp_path / "longtable"
    shutil.copytree(deck_dir["stress_a"], root)
    p = root / "BOUNDE" / "NZQ" / "NZQ0001.DAT"
    rows = ["7"] + [f"{1.0 + 0.3 * i} {10.0 * i}" for i in range(7)]
    p.write_text("\n".join(rows) + "\n")
    with pytest.raises(hb.HydroError) as e:
        hb.Deck(str(root))
    assert e.value.status == 2


def _declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        # C declarations only (the C++ overloads after `#ifdef __cplusplus }` are mangled)
        c_part = text.split("}  /* extern \"C\" */")[0]
        names += re.findall(r"\b(hb_[a-z0-9_]+)\s*\(", c_part)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    l = _lib.lib()
    declared = _declared_functions()
    assert len(declared) >= 25
    for name in declared:
        assert hasattr(l, name), name
    assert set(declared) == set(_lib.EXPORTED)


def test_library_exports_reference_signatures():
    """The C++ drop-in overloads of functors.cuh:59-65 are exported with the reference's mangled names."""
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    for sym in ("_Z13CalculateFluxRK8MeshViewiiP11CUstream_st", "_Z10UpdateCellRK8MeshViewP11CUstream_st",
                "_Z13CalculateFluxRK8MeshViewii", "_Z10UpdateCellRK8MeshView"):
        assert sym in out, sym


def test_persistent_option_is_checked_before_any_device_work(deck_dir):
    """A persistent handle takes the edge layout's default launch shape only;
    other combinations are refused by hb_create before it touches a device."""
    import hydrob200 as hb
    deck = hb.Deck(deck_dir["stress_a"])
    for kw in (dict(layout="tile"), dict(tile_config=2), dict(tile_config=9, layout="tile")):
        with pytest.raises(hb.HydroError) as e:
            hb.Solver(deck, persistent=True, **kw)
        assert e.value.status == 1, kw
    assert _lib.lib().hb_set_barrier_limit(None, 1_000_000, 0) == 1


def test_status_strings():
    l = _lib.lib()
    for code in range(10):
        assert l.hb_status_string(code)


def test_cpu_solver_deck_layout(tmp_path):
    """The CPU-solver deck keeps the mesh and turns open boundaries into walls."""
    d = D.stress_deck("s", 6, 4, 3, steps=5)
    root = str(tmp_path / "origin" / "changjiangkou")
    D.write_cpu_solver_deck(d, root, steps=7)
    assert os.path.exists(os.path.join(root, "TIME.DAT")) and os.path.exists(os.path.join(root, "SOURCES", "PNAC.DAT"))
    klas = np.loadtxt(os.path.join(root, "SOURCES", "PKLAS.DAT"), skiprows=1)[:, 1:]
    assert set(np.unique(klas)) <= {0.0, 4.0}
    assert open(os.path.join(root, "TIME.DAT")).readline().split()[0] == "7"
