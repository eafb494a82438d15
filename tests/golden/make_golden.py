"""Generate the golden fixtures from the reference's own binaries.

Runs on a machine with a B200 (the reference programs are CUDA). It writes
the seeded decks of :mod:`hydrob200.deck`, runs the reference dump driver
(``cuda_native_impl/benchmark.cu:131-169``, built into ``oracle/_ref`` by
``oracle/ref.mk``) on each, and stores the dumps as compact fixtures:

* ``<deck>__<bin>__s<steps>.npz``: H, U, V, Z, FLUX0..3, SIDE, SLCOS, SLSIN
  for the small decks; H, U, V, Z only for the 6,675-cell deck;
* ``manifest.json``: the SHA-256 of every deck's files (so a test can prove
  the generator still writes the same bytes) and of every dumped array.

Usage::

    python tests/golden/make_golden.py --out /tmp/golden
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "hydro-bench_b200"))

from hydrob200 import deck as D  # noqa: E402
from hydrob200.golden import DECKS, read_dump, deck_digest  # noqa: E402

BINS = {
    "h64": ("ref_h64", np.float64),
    "f64": ("ref_f64", np.float64),
    "h32": ("ref_h32", np.float32),
    "f32": ("ref_f32", np.float32),
}


def run_ref(binary: str, deck_dir: str, steps: int, dump: str) -> None:
    run_dir = os.path.join(deck_dir, "run")
    os.makedirs(run_dir, exist_ok=True)
    cmd = [binary, str(steps), "1", "--dump", dump]
    r = subprocess.run(cmd, cwd=run_dir, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"{cmd} failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--work", default=os.path.join(tempfile.gettempdir(), "hb_golden_decks"),
                    help="where the decks and the reference's dumps are written")
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    refdir = os.path.join(ROOT, "oracle", "_ref")
    manifest = {"decks": {}, "dumps": {}}
    prev = os.path.join(args.out, "manifest.json")
    if args.only and os.path.exists(prev):      # refresh some decks, keep the others' records
        with open(prev) as f:
            manifest = json.load(f)
    for name, spec in DECKS.items():
        if args.only and name not in args.only.split(","):
            continue
        deck = spec["make"]()
        ddir = os.path.join(args.work, name)
        D.write_deck(deck, ddir)
        manifest["decks"][name] = {"sha256": deck_digest(ddir), "cells": deck.cells}
        for bkey in spec["bins"]:
            binary, dtype = BINS[bkey]
            for steps in spec["steps"]:
                dump = os.path.join(ddir, f"dump_{bkey}_{steps}.bin")
                t0 = time.time()
                run_ref(os.path.join(refdir, binary), ddir, steps, dump)
                arrs = read_dump(dump, dtype)
                key = f"{name}__{bkey}__s{steps}"
                manifest["dumps"][key] = {k: hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()
                                          for k, v in arrs.items()}
                keep = arrs if spec["full"] else {k: arrs[k] for k in spec.get("keep", ("H", "U", "V", "Z"))}
                np.savez_compressed(os.path.join(args.out, key + ".npz"), **keep)
                print(f"{key}: {time.time() - t0:.2f}s H=[{arrs['H'].min():.6f},{arrs['H'].max():.6f}]", flush=True)
    with open(os.path.join(args.out, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
