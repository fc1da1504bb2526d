"""Generates tests/golden/gio_g2vtk.json from the reference's own GIO reader
in Python (analysis/python/g2vtk, read_header at lines 158-195).

Runs where a reference checkout is available (it loads the g2vtk script
from the reference tree): pass the checkout's root as the first argument or
in GEOFLOW_REFERENCE.  For a few small GIO files written by the oracle's
restatement (oracle/gio_oracle.py) it records the file bytes (hex) and the
header fields that g2vtk parses from them: version, dim, nelems, porder,
gtype, cycle, time and `skip`, the byte where g2vtk starts the field data.
g2vtk predates the multivar flag and the element keys at the end of the
header (io/gio.ipp:489-496), so its `skip` is the offset of the multivar
field; the test records that difference instead of hiding it.
Usage: python tests/golden/make_gio_golden.py <reference checkout>
"""
import importlib.machinery
import importlib.util
import json
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import gio_oracle as GO  # noqa: E402

CASES = [  # (dim, nelems, p, float bytes, gtype, cycle, time)
    (3, 4, 2, 8, 0, 12, 0.375),
    (2, 6, 3, 8, 2, 7, 1.5),
    (3, 2, 3, 4, 1, 3, 0.25),
]


def load_g2vtk():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GEOFLOW_REFERENCE")
    if not ref:
        raise SystemExit("usage: make_gio_golden.py <reference checkout> "
                         "(or set GEOFLOW_REFERENCE)")
    g2vtk = Path(ref) / "analysis" / "python" / "g2vtk"
    if not g2vtk.exists():
        raise SystemExit(f"{g2vtk} not found")
    loader = importlib.machinery.SourceFileLoader("g2vtk", str(g2vtk))
    spec = importlib.util.spec_from_loader("g2vtk", loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def main():
    g2 = load_g2vtk()
    out = []
    with tempfile.TemporaryDirectory() as d:
        for k, (dim, ne, p, fb, gtype, cycle, time) in enumerate(CASES):
            porder = np.full((1, dim), p, np.int32)
            nd = GO.ndata(0, dim, ne, porder)
            rng = np.random.default_rng(20261203 + k)
            data = rng.standard_normal(nd).astype(np.float64 if fb == 8 else np.float32)
            ids = np.arange(ne, dtype=np.uint64) * 11 + 5
            path = f"{d}/u{k}.000000.00000.out"
            GO.write(path, data, 0, dim, ne, porder, gtype=gtype, cycle=cycle, time=time,
                     elemids=ids)
            h = g2.read_header(path, fb)
            out.append(dict(case=[dim, ne, p, fb, gtype, cycle, time],
                            file_hex=open(path, "rb").read().hex(),
                            g2vtk={"vers": h["vers"], "dim": h["dim"], "nelems": h["nelems"],
                                   "porder": list(h["porder"]), "gtype": h["gtype"],
                                   "cycle": h["cycle"], "time": h["time"], "skip": h["skip"]}))
    dst = Path(__file__).resolve().parent / "gio_g2vtk.json"
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {dst}")


if __name__ == "__main__":
    main()
