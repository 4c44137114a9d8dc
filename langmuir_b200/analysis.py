"""LangmuirPython's analysis entry points in Python 3, over this library.

* ``load_dat`` reads an ``out.dat`` (LangmuirPython/langmuir/datfile.py) into
  a pandas DataFrame.
* ``calculate`` adds the flux statistics of analyze.calculate
  (LangmuirPython/langmuir/analyze.py:98-145): per-agent probability, rate
  and current, the net drain and source rates and currents, carrier totals
  and the simulation speed.
* ``PrecalculatedMesh`` is grid.PrecalculatedMesh (grid.py:474-554): its
  ``coulomb`` sums 1/r over charges with no cutoff and no prefactor. Here
  the sum runs on the GPU, through the same pair kernel as the engine.
"""
from __future__ import annotations

import math

import numpy as np

FLUXES = ["eSourceL", "eSourceR", "hSourceL", "hSourceR", "eDrainL", "eDrainR",
          "hDrainL", "hDrainR", "xSource", "xDrain"]
ELEMENTARY_CHARGE = 1.6021765650e-19  # the value analyze.py falls back to
IFACTOR = ELEMENTARY_CHARGE * 1e21     # analyze.py:32


def load_dat(path: str):
    """An out.dat as a DataFrame (whitespace-separated, header row)."""
    import pandas as pd
    return pd.read_csv(path, sep=r"\s+", engine="python")


def calculate(obj):
    """analyze.calculate: rates are successes per simulation step."""
    for flux in FLUXES:
        a, s = flux + ":attempt", flux + ":success"
        if a not in obj or s not in obj:
            continue
        t = "simulation:time"
        obj[flux + ":prob"] = obj[s] / obj[a].astype(float) * 100.0
        obj[flux + ":rate"] = obj[s] / obj[t].astype(float)
        obj[flux + ":current"] = obj[flux + ":rate"] * IFACTOR
    obj["eDrain:rate"] = obj["eDrainR:rate"] - obj["eDrainL:rate"]
    obj["eDrain:current"] = obj["eDrain:rate"] * IFACTOR
    obj["hDrain:rate"] = obj["hDrainL:rate"] - obj["hDrainR:rate"]
    obj["hDrain:current"] = obj["hDrain:rate"] * IFACTOR
    obj["drain:rate"] = obj["eDrain:rate"] + obj["hDrain:rate"]
    obj["drain:current"] = obj["drain:rate"] * IFACTOR
    obj["eSource:rate"] = obj["eSourceR:rate"] - obj["eSourceL:rate"]
    obj["eSource:current"] = obj["eSource:rate"] * IFACTOR
    obj["hSource:rate"] = obj["hSourceL:rate"] - obj["hSourceR:rate"]
    obj["hSource:current"] = obj["hSource:rate"] * IFACTOR
    obj["source:rate"] = obj["eSource:rate"] + obj["hSource:rate"]
    obj["source:current"] = obj["source:rate"] * IFACTOR
    obj["carrier:count"] = obj["electron:count"] + obj["hole:count"]
    obj["carrier:difference"] = obj["electron:count"] - obj["hole:count"]
    obj["speed"] = obj["real:time"].diff() / obj["simulation:time"].diff().astype(float)
    return obj.fillna(value=0.0)


class PrecalculatedMesh:
    """1/r sums between lattice points of an X x Y x Z grid (unit spacing).

    ``coulomb(xi, yi, zi, xj, yj, zj, q)`` returns q * sum_i 1/r_ij at every j
    (every lattice point when the j's are omitted), r = 0 terms skipped, as
    grid.PrecalculatedMesh.coulomb does.  Computed by the B200 pair kernel
    with a cutoff beyond the lattice diagonal and a prefactor of 1."""

    def __init__(self, nx: int, ny: int, nz: int, device: int = 0):
        from .coulomb import Coulomb
        self.shape = (int(nx), int(ny), int(nz))
        diag2 = (nx - 1) ** 2 + (ny - 1) ** 2 + (nz - 1) ** 2
        self.ctx = Coulomb(nx, ny, nz, cutoff=int(math.isqrt(diag2)) + 1, prefactor=1.0,
                           device=device)

    def close(self):
        self.ctx.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _sites(self, x, y, z):
        nx, ny, _ = self.shape
        x, y, z = (np.asarray(v, np.int64).ravel() for v in (x, y, z))
        return (x + nx * (y + ny * z)).astype(np.int32)

    def coulomb(self, xi, yi, zi, xj=None, yj=None, zj=None, q=1):
        src = self._sites(xi, yi, zi)
        if xj is None and yj is None and zj is None:
            gx, gy, gz = np.indices(self.shape)
            xj, yj, zj = gx, gy, gz
            shape = self.shape
        else:
            shape = np.asarray(xj).shape
        tgt = self._sites(xj, yj, zj)
        v = self.ctx.potentials(src, np.ones(len(src), np.int32), tgt)
        return q * np.asarray(v).reshape(shape)
