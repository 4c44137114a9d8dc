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
* ``IVCurve`` / ``IVCurveSolar`` are ivcurve.IVCurve and IVCurveSolar
  (ivcurve.py:15-160, 314-495): power, current density and irradiance from
  (current nA, voltage V, area nm^2), and for a solar cell the open-circuit
  voltage, short-circuit current, maximum power point and fill factor from a
  fit of i(v) and p(v) (fit.py: FitInterp1D, FitUnivariateSpline, FitPower,
  FitTanh/FitXTanh, FitErf/FitXErf).
* ``iv_sweep`` runs one morphology at several voltages as a batch of GPU
  solar-cell replicas and returns the IVCurveSolar of the measured currents.
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


# ---- current-voltage curves ---------------------------------------------------------------
# units.py conversions the reference's IVCurve uses: i nA, v V, p nW, a nm^2,
# j mA/cm^2, r mW/cm^2.  1 nA/nm^2 = 1e-9 A / 1e-14 cm^2 = 1e8 mA/cm^2, and the
# same factor takes nW/nm^2 to mW/cm^2.
_PER_NM2_TO_PER_CM2_MILLI = 1e8


class _Fit:
    """A fitted curve y(x) with fit.py's solve (fsolve) and minimize (BFGS,
    gtol 1e-2) wrappers."""

    def __init__(self, func):
        self.func = func

    def __call__(self, x):
        return self.func(x)

    def solve(self, y=0.0, x0=0.0):
        from scipy import optimize
        f = self.func if y == 0 else (lambda x: self.func(x) + y)
        return float(optimize.fsolve(f, x0)[0])

    def minimize(self, x0=0.0):
        from scipy import optimize
        return float(optimize.minimize(lambda x: self.func(x[0]), [x0], method="BFGS",
                                       options=dict(gtol=1e-2, disp=False)).x[0])


def _fit(form, x, y, yerr, popt=None, **kw):
    from scipy import interpolate, optimize, special
    yerr = None if yerr is None or not np.count_nonzero(yerr) else yerr
    if form == "interp1d":
        f = interpolate.interp1d(x, y, kind=kw.get("kind", "cubic"), fill_value=np.nan,
                                 bounds_error=False)
        return _Fit(lambda v: f(v)[()])
    if form == "spline":
        f = interpolate.UnivariateSpline(x, y, k=kw.get("k", 3))
        return _Fit(lambda v: f(v)[()])
    if form == "power":
        c = np.polyfit(x, y, kw["order"], w=yerr)
        return _Fit(np.poly1d(c))
    forms = {"tanh": lambda v, a=1, b=1, c=0, d=0: a * np.tanh(b * v + c) + d,
             "xtanh": lambda v, a=1, b=1, c=0, d=0: a * v * np.tanh(b * v + c) + d,
             "erf": lambda v, a=1, b=1, c=0, d=0: a * special.erf(b * v + c) + d,
             "xerf": lambda v, a=1, b=1, c=0, d=0: a * v * special.erf(b * v + c) + d}
    g = forms[form]
    popt, _ = optimize.curve_fit(g, x, y, popt, yerr)
    return _Fit(lambda v: g(v, *popt))


class IVCurve:
    """Current, voltage and area arrays with the derived power p = i v (nW),
    current density j = i / a (mA/cm^2) and irradiance r = p / a (mW/cm^2)."""

    def __init__(self, i, v, a, ierr=None):
        i = np.asarray(i, np.float64)
        v = np.asarray(v, np.float64)
        a = np.full_like(i, float(a)) if np.isscalar(a) else np.asarray(a, np.float64)
        if not (i.shape == v.shape == a.shape):
            raise ValueError("i, v and a must have one shape")
        self.i, self.v, self.a = i, v, a
        self.p = i * v
        self.j = i / a * _PER_NM2_TO_PER_CM2_MILLI
        self.r = self.p / a * _PER_NM2_TO_PER_CM2_MILLI
        self.ierr = np.zeros_like(i) if ierr is None else np.asarray(ierr, np.float64)
        self.perr = self.ierr * v
        self.jerr = self.ierr / a * _PER_NM2_TO_PER_CM2_MILLI
        self.rerr = self.perr / a * _PER_NM2_TO_PER_CM2_MILLI

    def summary(self) -> dict:
        """analyze.Stats of every array: <name>.max/min/rng/avg/std."""
        d = {}
        for name in ("i", "v", "p", "a", "j", "r", "ierr", "jerr", "perr", "rerr"):
            x = getattr(self, name)
            mx, mn = float(np.max(x)), float(np.min(x))
            d.update({f"{name}.max": mx, f"{name}.min": mn, f"{name}.rng": abs(mx - mn),
                      f"{name}.avg": float(np.mean(x)), f"{name}.std": float(np.std(x))})
        return d


class IVCurveSolar(IVCurve):
    """IVCurveSolar: the voltages are shifted by ``v_shift`` (1.5 V in the
    reference) and ``calculate`` finds v_oc (i = 0, from the guess v_shift),
    i_sc = i(0), p_th = v_oc i_sc, the maximum power point (the minimum of p,
    from 0.66 v_oc), p_mp = i_mp v_mp, the densities over the mean area and the
    fill factor 100 p_mp / p_th."""

    def __init__(self, i, v, a, ierr=None, v_shift=1.5, **kwargs):
        self.v_shift = v_shift
        super().__init__(i, np.asarray(v, np.float64) + v_shift, a, ierr)
        self.v_oc = self.i_sc = self.p_th = self.v_mp = self.i_mp = self.p_mp = 0.0
        self.j_sc = self.r_th = self.j_mp = self.r_mp = self.fill = 0.0
        self.ifit = self.pfit = self.jfit = self.rfit = None
        if kwargs:
            self.calculate(**kwargs)

    def calculate(self, mode="interp1d", recycle=False, guess=None, **kwargs):
        v = self.v
        if mode in ("interp1d", "spline"):
            if mode == "interp1d":
                kwargs.setdefault("kind", "cubic")
            else:
                kwargs.setdefault("k", 3)
            self.ifit, self.jfit, self.pfit, self.rfit = (
                _fit(mode, v, y, e, **kwargs) for y, e in ((self.i, self.ierr),
                                                           (self.j, self.jerr),
                                                           (self.p, self.perr),
                                                           (self.r, self.rerr)))
        elif mode == "power":
            order = kwargs.get("order", 8)
            self.ifit = _fit("power", v, self.i, self.ierr, order=order)
            self.jfit = _fit("power", v, self.j, self.jerr, order=order)
            self.pfit = _fit("power", v, self.p, self.perr, order=order + 1)
            self.rfit = _fit("power", v, self.r, self.rerr, order=order + 1)
        elif mode in ("tanh", "erf"):
            i0 = [float(np.min(self.i)), 1.0, -self.v_shift, 0.0]
            j0 = [float(np.min(self.j)), 1.0, -self.v_shift, 0.0]
            self.ifit = _fit(mode, v, self.i, self.ierr, i0)
            self.jfit = _fit(mode, v, self.j, self.jerr, j0)
            self.pfit = _fit("x" + mode, v, self.p, self.perr, i0)
            self.rfit = _fit("x" + mode, v, self.r, self.rerr, j0)
        else:
            raise NotImplementedError(f"unknown fit mode: {mode}")
        guess = self.v_shift if guess is None else guess
        self.v_oc = self.ifit.solve(x0=guess)
        self.i_sc = float(self.ifit(0.0))
        self.p_th = self.v_oc * self.i_sc
        self.v_mp = self.pfit.minimize(0.66 * self.v_oc)
        self.i_mp = float(self.ifit(self.v_mp))
        self.p_mp = self.i_mp * self.v_mp
        area = float(np.mean(self.a))
        self.j_sc = self.i_sc / area * _PER_NM2_TO_PER_CM2_MILLI
        self.j_mp = self.i_mp / area * _PER_NM2_TO_PER_CM2_MILLI
        self.r_th = self.p_th / area * _PER_NM2_TO_PER_CM2_MILLI
        self.r_mp = self.p_mp / area * _PER_NM2_TO_PER_CM2_MILLI
        self.fill = self.p_mp / self.p_th * 100.0
        return self

    def summary(self) -> dict:
        d = super().summary()
        for k in ("v_oc", "i_sc", "p_th", "v_mp", "i_mp", "p_mp", "j_sc", "r_th", "j_mp", "r_mp",
                  "fill"):
            d[k] = float(getattr(self, k))
        return d


def iv_sweep(params, phase, voltages, steps, burn_in=0, device=0, replica0=0, v_shift=1.5,
             mode="interp1d", **fit_kw):
    """One morphology at several voltages: replica k is ``params`` with
    voltage.right = voltages[k], all run as one GPU batch for ``steps`` steps.
    The current of a replica is analyze.calculate's drain:current (net electron
    and hole drain successes per step, times IFACTOR, in nA) over the steps
    after ``burn_in``.  Returns (IVCurveSolar, currents)."""
    from .kmc import KMCBatch, Params
    reps = []
    for v in voltages:
        q = Params.from_text("[Parameters]\n")
        for name, _ in Params._fields_:
            setattr(q, name, getattr(params, name))
        q.set("voltage_right", float(v))
        reps.append(q.check())
    with KMCBatch(reps, device=device, replica0=replica0) as b:
        for k in range(len(reps)):
            b.replica(k).set_morphology(phase)
        if burn_in:
            b.run(burn_in)
        c0 = [np.asarray(b.replica(k).stats()["counters"], np.int64) for k in range(len(reps))]
        b.run(steps - burn_in)
        c1 = [np.asarray(b.replica(k).stats()["counters"], np.int64) for k in range(len(reps))]
    # counters: (attempts, successes) of eSourceL eSourceR hSourceL hSourceR
    # eDrainL eDrainR hDrainL hDrainR ...; analyze.py:120-127 signs
    cur = []
    for a, z in zip(c0, c1):
        d = z - a
        e_rate = (d[11] - d[9]) / float(steps - burn_in)
        h_rate = (d[13] - d[15]) / float(steps - burn_in)
        cur.append((e_rate + h_rate) * IFACTOR)
    cur = np.array(cur)
    area = params.grid_y * params.grid_z
    iv = IVCurveSolar(cur, np.asarray(voltages, np.float64), area, v_shift=v_shift)
    iv.calculate(mode=mode, **fit_kw)
    return iv, cur
