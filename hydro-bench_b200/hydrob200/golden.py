"""Registry of the seeded parity decks and the reference dump format."""
from __future__ import annotations

import hashlib
import os
from typing import Dict

import numpy as np

from . import deck as D

# name -> how to build it, which reference builds to dump, after how many steps,
# and whether the fixture keeps every array or only the state.
DECKS = {
    "stress_a": dict(make=lambda: D.stress_deck("stress_a", 20, 10, 7, steps=50, mdt=20),
                     bins=("h64", "f64", "h32", "f32"), steps=(1, 10, 50), full=True),
    "stress_b": dict(make=lambda: D.stress_deck("stress_b", 24, 12, 11, steps=50, mdt=20, jl=0.0),
                     bins=("h64", "f64"), steps=(1, 50), full=True),
    "breach": dict(make=lambda: D.stress_deck("breach", 12, 8, 23, steps=10, with_breach=True),
                   bins=("h64",), steps=(1,), full=True),
    "probe": dict(make=lambda: D.probe_deck("probe"),
                  bins=("h64", "f64"), steps=(7, 13, 45, 58), full=True),
    "f1": dict(make=lambda: D.config_f1(),
               bins=("h64", "f64", "h32"), steps=(1, 50, 100), full=False),
}


def read_dump(path: str, dtype) -> Dict[str, np.ndarray]:
    """Parse a reference ``--dump`` file (``cuda_native_impl/benchmark.cu:141-162``).

    Layout: ``int32 CELL``; H, U, V, Z ``[CELL]``; SLCOS, SLSIN, SIDE ``[4*CELL]``;
    FLUX0..3 ``[4*CELL]``, all of the build's ``Real`` type.
    """
    with open(path, "rb") as f:
        buf = f.read()
    cell = int(np.frombuffer(buf[:4], dtype=np.int32)[0])
    a = np.frombuffer(buf[4:], dtype=dtype)
    out = {}
    off = 0
    for k in ("H", "U", "V", "Z"):
        out[k] = a[off:off + cell].copy(); off += cell
    for k in ("SLCOS", "SLSIN", "SIDE", "FLUX0", "FLUX1", "FLUX2", "FLUX3"):
        out[k] = a[off:off + 4 * cell].copy(); off += 4 * cell
    if off != a.size:
        raise ValueError(f"dump size mismatch: {a.size} values, parsed {off}")
    return out


def deck_digest(root: str) -> str:
    """SHA-256 over every file of a deck (sorted relative paths and bytes)."""
    h = hashlib.sha256()
    for dirpath, dirnames, filenames in os.walk(root):
        dirnames[:] = sorted(d for d in dirnames if d not in ("run", "OUTPUT"))
        for fn in sorted(filenames):
            if not fn.endswith(".DAT"):
                continue
            p = os.path.join(dirpath, fn)
            h.update(os.path.relpath(p, root).encode())
            with open(p, "rb") as f:
                h.update(f.read())
    return h.hexdigest()
