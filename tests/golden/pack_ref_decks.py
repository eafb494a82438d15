"""Pack the reference's own shipped decks as test fixtures.

The reference ships two real hydro-cal decks in its text format:

* ``data/F1_text`` (6,675 quad cells; KLAS 4 walls, KLAS 10 inflow groups
  with a zero hydrograph, KLAS 13 codes that BOUNDA leaves unhandled), run
  with the time files of ``cuda_native_impl/F1_native_data/BINFOR``
  (CALTIME.DAT: DT = 1 s; TIME.DAT: MDT = 3600 s, 50 intervals; JL.DAT);
* ``data/F2_24K_text`` (24,020 cells; 169 KLAS 1 given-level edges in two
  groups; DT = 4 s, HM1 = 0.01, HM2 = 0.1), the deck behind
  ``cuda_native_impl/F2_24K_native_data``.

Their files lie flat in the data directories; the reference's reader
(``cuda_native_impl/hydro-cal-src/src/mesh.cpp:8-30``) wants them split into
``BINFOR/`` and ``SOURCES/`` with ``BOUNDE/`` beside them, which the
``*_native_data`` directories do by symbolic links.  This script assembles
that layout from the files themselves and writes one deterministic
``.tar.xz`` per deck (sorted members, zero times and owners), so the GPU
tests can run the reference program and this library on the same bytes
where the reference checkout is absent.

Usage::

    python tests/golden/pack_ref_decks.py --ref <reference checkout> [--out tests/golden]
"""
from __future__ import annotations

import argparse
import hashlib
import io
import json
import lzma
import os
import sys
import tarfile

BINFOR = ("TIME", "GIRD", "DEPTH", "BOUNDARY", "CALTIME", "JL", "INITIALLEVEL", "INITIALU1", "INITIALV1", "CV")
SOURCES = ("PNAC", "PNAP", "PKLAS", "PZBC", "PXY", "MBZ", "MBQ", "MBW", "MBZQ")

# deck name -> (data directory, directory whose BINFOR overrides the time files, files taken from it)
DECKS = {
    "ref_f1": ("data/F1_text", "cuda_native_impl/F1_native_data/BINFOR", ("CALTIME", "TIME", "JL")),
    "ref_f2_24k": ("data/F2_24K_text", None, ()),
}


def members(ref: str, data: str, override: str, from_override) -> dict:
    """archive path -> bytes, in the layout the reference's reader expects."""
    src = os.path.join(ref, data)
    out = {}
    for name in BINFOR:
        p = os.path.join(ref, override, name + ".DAT") if name in from_override else os.path.join(src, name + ".DAT")
        with open(p, "rb") as f:
            out[f"BINFOR/{name}.DAT"] = f.read()
    for name in SOURCES:
        with open(os.path.join(src, name + ".DAT"), "rb") as f:
            out[f"SOURCES/{name}.DAT"] = f.read()
    bounde = os.path.join(src, "BOUNDE")
    for sub in sorted(os.listdir(bounde)):
        for fn in sorted(os.listdir(os.path.join(bounde, sub))):
            with open(os.path.join(bounde, sub, fn), "rb") as f:
                out[f"BOUNDE/{sub}/{fn}"] = f.read()
    return out


def write_tar_xz(files: dict, path: str) -> None:
    buf = io.BytesIO()
    with tarfile.open(fileobj=buf, mode="w", format=tarfile.USTAR_FORMAT) as tar:
        for name in sorted(files):
            data = files[name]
            ti = tarfile.TarInfo(name)
            ti.size = len(data)
            ti.mtime = 0
            ti.mode = 0o644
            ti.uid = ti.gid = 0
            ti.uname = ti.gname = ""
            tar.addfile(ti, io.BytesIO(data))
    with open(path, "wb") as f:
        f.write(lzma.compress(buf.getvalue(), preset=9))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference checkout (chhnb/hydro-bench)")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    args = ap.parse_args()
    digests = {}
    for name, (data, override, from_override) in DECKS.items():
        files = members(args.ref, data, override, from_override)
        path = os.path.join(args.out, name + ".tar.xz")
        write_tar_xz(files, path)
        h = hashlib.sha256()
        for k in sorted(files):
            h.update(k.encode())
            h.update(files[k])
        digests[name] = {"files": len(files), "sha256": h.hexdigest(), "from": data}
        print(f"{name}: {len(files)} files, {os.path.getsize(path)} bytes", flush=True)
    with open(os.path.join(args.out, "ref_decks.json"), "w") as f:
        json.dump(digests, f, indent=1, sort_keys=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
