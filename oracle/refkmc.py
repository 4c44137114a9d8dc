"""The reference's own kMC engine, compiled, as a checker (TEST INFRASTRUCTURE).

``oracle/_ref/librefkmc.so`` holds the reference's World, Grid, Potential,
Random and agent classes compiled from its src/langmuirCore sources against
the Qt/Boost stand-ins in ``oracle/refshim`` (recipe: ``make -C oracle ref``),
with the step harness ``oracle/refshim/refkmc.cpp``.  Every random draw comes
from the Philox stream the GPU step and the FP64 oracle use, so the three can
be compared bit for bit:

* world set-up: World::initialize (world.cpp:507-657) with the set-up draws
  in the reference's own order;
* one step: Simulation::performIterations (simulation.cpp:34-111), the loop
  restated in the harness, every agent method the reference's.

Only tests/ use this module; the library never loads it.  ``available()`` is
False where the reference tree was not there to compile it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "librefkmc.so")
_lib = None
_vp = ctypes.c_void_p


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB)
        _lib.ref_kmc_create.restype = _vp
        _lib.ref_kmc_create.argtypes = [_vp, ctypes.c_uint32] + [_vp, ctypes.c_int] * 5 + [
            ctypes.c_char_p, ctypes.c_int]
        sig = {"ref_kmc_sizes": [_vp, _vp],
               "ref_kmc_world": [_vp, _vp, _vp, _vp, _vp, _vp],
               "ref_kmc_carriers": [_vp, _vp, _vp],
               "ref_kmc_step": [_vp, _vp, _vp, ctypes.c_char_p, ctypes.c_int],
               "ref_kmc_counters": [_vp, _vp],
               "ref_kmc_neighbors": [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int],
               "ref_kmc_coupling": [_vp, _vp]}
        for name, args in sig.items():
            fn = getattr(_lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = args
        _lib.ref_kmc_destroy.restype = None
        _lib.ref_kmc_destroy.argtypes = [_vp]
    return _lib


def _arr(a, dtype):
    if a is None or len(a) == 0:
        return None, 0, None
    a = np.ascontiguousarray(a, dtype=dtype)
    return a.ctypes.data, len(a), a


class RefKMC:
    """A reference World built from ``params`` (langmuir_b200.Params) for
    replica ``replica``, optionally from checkpoint lists."""

    def __init__(self, params, replica=0, electrons=None, holes=None, defects=None, traps=None,
                 trap_potentials=None):
        err = ctypes.create_string_buffer(512)
        self._keep = []
        args = []
        for a, dt in ((electrons, np.int32), (holes, np.int32), (defects, np.int32),
                      (traps, np.int32), (trap_potentials, np.float64)):
            ptr, n, keep = _arr(a, dt)
            self._keep.append(keep)
            args += [ptr, n]
        self._h = lib().ref_kmc_create(ctypes.byref(params), ctypes.c_uint32(int(replica)), *args,
                                       err, len(err))
        if not self._h:
            raise RuntimeError("reference World: " + err.value.decode())
        self._h = _vp(self._h)

    def close(self):
        if self._h:
            lib().ref_kmc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def sizes(self):
        s = np.zeros(8, np.int32)
        lib().ref_kmc_sizes(self._h, s.ctypes.data)
        return dict(electrons=int(s[0]), holes=int(s[1]), defects=int(s[2]), traps=int(s[3]),
                    max_electrons=int(s[4]), max_holes=int(s[5]), volume=int(s[6]),
                    step=int(s[7]))

    def world(self):
        z = self.sizes()
        V = z["volume"]
        pe, ph = np.zeros(V), np.zeros(V)
        d = np.zeros(max(z["defects"], 1), np.int32)
        t = np.zeros(max(z["traps"], 1), np.int32)
        tp = np.zeros(max(z["traps"], 1))
        lib().ref_kmc_world(self._h, pe.ctypes.data, ph.ctypes.data, d.ctypes.data, t.ctypes.data,
                            tp.ctypes.data)
        return dict(site_energy=pe, hole_site_energy=ph, defects=d[: z["defects"]],
                    traps=t[: z["traps"]], trap_potentials=tp[: z["traps"]])

    def carriers(self):
        z = self.sizes()
        e = np.zeros(max(z["electrons"], 1), np.int32)
        h = np.zeros(max(z["holes"], 1), np.int32)
        lib().ref_kmc_carriers(self._h, e.ctypes.data, h.ctypes.data)
        return e[: z["electrons"]].copy(), h[: z["holes"]].copy()

    def step(self):
        """One step; returns (outcome, dE) per carrier of the step's start."""
        z = self.sizes()
        n = z["electrons"] + z["holes"]
        out = np.zeros(max(n, 1), np.int32)
        de = np.zeros(max(n, 1))
        err = ctypes.create_string_buffer(512)
        if lib().ref_kmc_step(self._h, out.ctypes.data, de.ctypes.data, err, len(err)) != 0:
            raise RuntimeError("reference step: " + err.value.decode())
        return out[:n].copy(), de[:n].copy()

    @property
    def counters(self):
        c = np.zeros(20, np.uint64)
        lib().ref_kmc_counters(self._h, c.ctypes.data)
        return c

    def neighbors(self, site, hopping_range):
        out = np.zeros(64, np.int32)
        n = lib().ref_kmc_neighbors(self._h, int(site), int(hopping_range), out.ctypes.data, 64)
        if n < 0:
            raise RuntimeError("Grid::neighborsSite failed")
        return out[:n].copy()

    def coupling(self, hopping_range):
        h = hopping_range + 1
        out = np.zeros(h ** 3)
        lib().ref_kmc_coupling(self._h, out.ctypes.data)
        return out
