"""Golden files for the LangmuirPython readers and writers.

Copies the reference's own LangmuirPython test data -- the out.dat, out.chk
and out.parm of LangmuirPython/test/system.0/run.0/sim.0/part.0 and part.1,
which LangmuirPython/test/test.py:13-27 loads -- into one JSON file, so that
the tests need no reference tree.  These are engine outputs: out.dat shows the
FluxWriter column order and field width, out.chk the CheckPointer sections.

Usage:  python tests/golden/make_lp_golden.py
"""
from __future__ import annotations

import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE = os.environ.get("REFERENCE", "/root/reference")


def main():
    base = os.path.join(REFERENCE, "LangmuirPython", "test", "system.0", "run.0", "sim.0")
    out = {}
    for part in ("part.0", "part.1"):
        for name in ("out.dat", "out.chk", "out.parm"):
            with open(os.path.join(base, part, name)) as fh:
                out[f"{part}/{name}"] = fh.read()
    path = os.path.join(HERE, "langmuirpython_system0.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=0)
    print("wrote", path, sum(len(v) for v in out.values()), "characters")


if __name__ == "__main__":
    main()
