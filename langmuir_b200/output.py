"""Langmuir output files written from a GPU replica.

* ``FluxWriter`` -- ``out.dat``: one row per report of the step, every flux
  agent's attempts and successes, the carrier counts and the wall time, as
  FluxWriter writes it (src/langmuirCore/writer.cpp:18-43, 360-379): every
  field right-aligned in output.width columns, the flux agents in the
  reference's order (eSourceL eSourceR hSourceL hSourceR xSource eDrainL
  eDrainR hDrainL hDrainR xDrain).  LangmuirPython's datfile / analyze modules
  read it unchanged.
* ``write_coulomb`` -- ``out.coulomb``: the Coulomb potential at every site,
  "s x y z v" rows with x slowest and z fastest, as Logger::saveCoulombEnergy
  writes it (writer.cpp:545-581); the potentials come from the whole-grid
  kernel 1 (lgm_coulomb_kernel1).
"""
from __future__ import annotations

import time

import numpy as np

from .checkpoint import FLUX_NAMES, reference_flux


class FluxWriter:
    """out.dat of one replica.  ``write()`` appends the current row."""

    def __init__(self, kmc, path: str):
        self.kmc = kmc
        self.path = path
        self.width = max(1, int(kmc.params.output_width))
        self.start = time.monotonic()
        cols = ["simulation:time"]
        for name in FLUX_NAMES:
            cols += [f"{name}:attempt", f"{name}:success"]
        cols += ["electron:count", "hole:count", "real:time"]
        with open(path, "w") as fh:
            fh.write(self._row(cols))

    def _row(self, items) -> str:
        return "".join(str(v).rjust(self.width) for v in items) + "\n"

    def write(self) -> None:
        s = self.kmc.stats()
        row = [s["step"]] + reference_flux(s["counters"]) + [
            s["electrons"], s["holes"], int(1000 * (time.monotonic() - self.start))]
        with open(self.path, "a") as fh:
            fh.write(self._row(row))


def coulomb_grid(kmc, ctx=None) -> np.ndarray:
    """Potential at every site from the replica's carriers and charged
    defects (launchCoulombKernel1 semantics), FP64 per site."""
    from . import _native as N
    from .coulomb import Coulomb
    p = kmc.params
    e, h = kmc.carriers()
    w = kmc.world()
    sites = [e, h]
    charges = [-np.ones(len(e), np.int32), np.ones(len(h), np.int32)]
    if p.defects_charge != 0 and len(w["defects"]):
        sites.append(w["defects"])
        charges.append(np.full(len(w["defects"]), p.defects_charge, np.int32))
    s = np.concatenate(sites).astype(np.int32)
    q = np.concatenate(charges).astype(np.int32)
    own = ctx is None
    if own:
        ctx = Coulomb(p.grid_x, p.grid_y, p.grid_z, cutoff=p.electrostatic_cutoff,
                      sigma=p.coulomb_gaussian_sigma)
    try:
        kind = N.GAUSS if p.coulomb_gaussian_sigma > 0 else N.POINT
        return ctx.kernel1(s, q, kind)
    finally:
        if own:
            ctx.close()


def write_coulomb(kmc, path: str, potentials: np.ndarray | None = None) -> None:
    v = coulomb_grid(kmc) if potentials is None else np.asarray(potentials)
    p = kmc.params
    X, Y, Z = p.grid_x, p.grid_y, p.grid_z
    prec = int(p.output_precision)
    lines = ["s x y z v"]
    for i in range(X):
        for j in range(Y):
            for k in range(Z):
                si = i + X * (j + Y * k)  # Grid::getIndexS (cubicgrid.cpp:102-110)
                lines.append(f"{si} {i} {j} {k} {v[si]:.{prec}e}")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
