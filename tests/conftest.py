"""Shared test fixtures: paths, the `gpu` marker and the seeded decks."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "hydro-bench_b200"))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def deck_dir(tmp_path_factory):
    """Writes every golden deck once per session; returns name -> directory."""
    from hydrob200 import deck as D
    from hydrob200.golden import DECKS
    base = tmp_path_factory.mktemp("decks")
    out = {}
    for name, spec in DECKS.items():
        d = spec["make"]()
        path = str(base / name)
        D.write_deck(d, path)
        out[name] = path
    return out


REF_DECKS = ("ref_f1", "ref_f2_24k")


@pytest.fixture(scope="session")
def ref_deck_dir(tmp_path_factory):
    """The reference's own shipped decks (tests/golden/<name>.tar.xz, packed by
    tests/golden/pack_ref_decks.py), unpacked once per session; name -> directory."""
    import tarfile
    base = tmp_path_factory.mktemp("ref_decks")
    out = {}
    for name in REF_DECKS:
        path = str(base / name)
        with tarfile.open(os.path.join(GOLDEN, name + ".tar.xz"), "r:xz") as tar:
            tar.extractall(path, filter="data")
        out[name] = path
    return out


@pytest.fixture(scope="session")
def manifest():
    import json
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def golden(name, binary, steps):
    import numpy as np
    return np.load(os.path.join(GOLDEN, f"{name}__{binary}__s{steps}.npz"))
