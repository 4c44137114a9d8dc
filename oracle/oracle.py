"""ctypes wrapper for the CPU checker.

TEST INFRASTRUCTURE ONLY.  Loads the FP64 restatement (``_build/liblgm_oracle.so``)
and, when it was built, the compiled reference kernels (``_ref/libkernelcl_ref.so``).
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (the CPU baseline and
the reference arm) import this module, and only as the checker or the timed CPU
baseline; the product package never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liblgm_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libkernelcl_ref.so")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")

# Agent::Type (include/agent.h:33-55)
EMPTY, ELECTRON, HOLE, DEFECT, SOURCE, DRAIN = range(6)


def reference_tree():
    """The reference source tree the compiled-reference recipes read: the
    REFERENCE environment variable, else the tree's usual mount point; None
    where neither holds it (a GPU box has no copy)."""
    path = os.environ.get("REFERENCE", "/root/reference")
    return path if os.path.isdir(path) else None


def build(ref: bool = False) -> None:
    """Compile the oracle (and the compiled-reference checker when ``ref``)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    tree = reference_tree()
    if ref and tree:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE={tree}"], check=True)


_lib = None
_ref = None


class KmcConfig(ctypes.Structure):
    """orc_kmc_config (lgm_oracle.h)."""
    _fields_ = [("inverse_kt", ctypes.c_double), ("exciton_binding", ctypes.c_double),
                ("coulomb_carriers", ctypes.c_int32), ("defects_charge", ctypes.c_int32),
                ("image_terms", ctypes.c_uint32),
                ("rate_e_source_l", ctypes.c_double), ("rate_e_source_r", ctypes.c_double),
                ("rate_h_source_l", ctypes.c_double), ("rate_h_source_r", ctypes.c_double),
                ("rate_e_drain_l", ctypes.c_double), ("rate_e_drain_r", ctypes.c_double),
                ("rate_h_drain_l", ctypes.c_double), ("rate_h_drain_r", ctypes.c_double),
                ("max_electrons", ctypes.c_int32), ("max_holes", ctypes.c_int32),
                ("seed", ctypes.c_uint32), ("replica", ctypes.c_uint32),
                ("solar", ctypes.c_int32), ("generation_rate", ctypes.c_double),
                ("recombination_rate", ctypes.c_double), ("recombination_range", ctypes.c_int32),
                ("hopping_range_neighbors", ctypes.c_int32),
                ("phase", ctypes.c_void_p), ("confine", ctypes.c_int32),
                ("bonds", ctypes.c_void_p), ("nbonds", ctypes.c_int32),
                ("source_metropolis", ctypes.c_int32), ("source_coulomb", ctypes.c_int32),
                ("balance_charges", ctypes.c_int32), ("voltage_left", ctypes.c_double),
                ("voltage_right", ctypes.c_double)]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int] * 5 + [ctypes.c_double] * 2
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_table.argtypes = [ctypes.c_void_p, ctypes.c_int, _f64p]
        L.orc_self_table.argtypes = [ctypes.c_void_p, _f64p]
        L.orc_coupling_table.argtypes = [ctypes.c_void_p, _f64p]
        for f in ("orc_index_x", "orc_index_y", "orc_index_z"):
            getattr(L, f).argtypes = [ctypes.c_void_p, ctypes.c_int]
            getattr(L, f).restype = ctypes.c_int
        L.orc_index_s.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 3
        L.orc_index_s.restype = ctypes.c_int
        L.orc_neighbors.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _i32p]
        L.orc_neighbors.restype = ctypes.c_int
        L.orc_species_potential.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p, _i32p,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_species_potential.restype = ctypes.c_double
        L.orc_species_potential_right_image.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p,
                                                        _i32p, ctypes.c_int, ctypes.c_int]
        L.orc_species_potential_right_image.restype = ctypes.c_double
        L.orc_kernel2.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p, _i32p, ctypes.c_int,
                                  ctypes.c_int, _f64p, ctypes.c_int]
        L.orc_kernel1.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p, _i32p, ctypes.c_int,
                                  _f64p, ctypes.c_int]
        L.orc_coulomb_cpu.argtypes = [ctypes.c_void_p, _i32p, _i32p, ctypes.c_int, _i32p, _i32p,
                                      ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int, _u8p, _u8p,
                                      ctypes.c_double, _f64p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_int]
        L.orc_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
        L.orc_kmc_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(KmcConfig), _f64p, _i32p,
                                   ctypes.c_int, ctypes.c_uint32, _i32p,
                                   ctypes.POINTER(ctypes.c_int32), _i32p,
                                   ctypes.POINTER(ctypes.c_int32),
                                   np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS"),
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.orc_potentials.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint, _i32p, _i32p,
                                     ctypes.c_int, _i32p, ctypes.c_int, _f64p, ctypes.c_int]
        _lib = L
    return _lib


def ref_lib():
    """The reference's own kernel.cl compiled as C, or None if it was not built."""
    global _ref
    if _ref is None and os.path.exists(REF_PATH):
        R = ctypes.CDLL(REF_PATH)
        R.ref_kernel2.argtypes = [ctypes.c_int, _i32p, _i32p, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_int, _f64p]
        R.ref_kernel2.restype = ctypes.c_int
        R.ref_kernel1.argtypes = [ctypes.c_int, _i32p, _i32p, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f64p]
        R.ref_kernel1.restype = ctypes.c_int
        _ref = R
    return _ref


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


class Oracle:
    """One lattice + electrostatics set-up (World::initialize order)."""

    def __init__(self, grid_x, grid_y, grid_z, cutoff=50, hopping_range=1, sigma=0.0,
                 prefactor=None):
        if prefactor is None:
            prefactor = electrostatic_prefactor()
        self.dims = (int(grid_x), int(grid_y), int(grid_z))
        self.cutoff = int(cutoff)
        self.hopping_range = int(hopping_range)
        self.sigma = float(sigma)
        self.prefactor = float(prefactor)
        self.volume = self.dims[0] * self.dims[1] * self.dims[2]
        self._c = lib().orc_create(*self.dims, self.cutoff, self.hopping_range, self.sigma,
                                   self.prefactor)
        if not self._c:
            raise ValueError("invalid oracle set-up")

    def __del__(self):
        c = getattr(self, "_c", None)
        if c and _lib is not None:
            _lib.orc_destroy(c)
            self._c = None

    # -- tables --------------------------------------------------------------
    def table(self, which: str) -> np.ndarray:
        n = self.cutoff + 1
        out = np.empty(n * n * n, dtype=np.float64)
        lib().orc_table(self._c, {"R1": 0, "R2": 1, "iR": 2, "eR": 3}[which], out)
        return out.reshape(n, n, n)

    def self_table(self) -> np.ndarray:
        n = self.hopping_range + 1
        out = np.empty(n ** 3, dtype=np.float64)
        lib().orc_self_table(self._c, out)
        return out.reshape(n, n, n)

    def coupling_table(self) -> np.ndarray:
        n = self.hopping_range + 1
        out = np.empty(n ** 3, dtype=np.float64)
        lib().orc_coupling_table(self._c, out)
        return out.reshape(n, n, n)

    # -- lattice ---------------------------------------------------------------
    def xyz(self, site):
        L = lib()
        return (L.orc_index_x(self._c, site), L.orc_index_y(self._c, site),
                L.orc_index_z(self._c, site))

    def site(self, x, y, z):
        return lib().orc_index_s(self._c, x, y, z)

    def neighbors(self, site, hopping_range=None):
        hr = self.hopping_range if hopping_range is None else hopping_range
        out = np.empty(40, dtype=np.int32)
        n = lib().orc_neighbors(self._c, int(site), int(hr), out)
        return out[:n].copy()

    # -- sums ------------------------------------------------------------------
    def species_potential(self, site, sites, charges, gauss=False, image=False):
        s, q = _i32(sites), _i32(charges)
        return lib().orc_species_potential(self._c, int(site), s, q, len(s), int(gauss),
                                           int(image))

    def species_potential_right_image(self, site, sites, charges, gauss=False):
        s, q = _i32(sites), _i32(charges)
        return lib().orc_species_potential_right_image(self._c, int(site), s, q, len(s),
                                                       int(gauss))

    def potentials(self, src, q, tgt, gauss=False, terms=1, threads=0):
        src, q, tgt = _i32(src), _i32(q), _i32(tgt)
        out = np.empty(len(tgt), dtype=np.float64)
        lib().orc_potentials(self._c, int(gauss), int(terms), src, q, len(src), tgt, len(tgt),
                             out, int(threads))
        return out

    def kernel2(self, s, q, n, gauss=False, threads=0):
        s, q = _i32(s), _i32(q)
        o = np.empty(len(s), dtype=np.float64)
        lib().orc_kernel2(self._c, int(gauss), s, q, int(n), len(s), o, int(threads))
        return o

    def kernel1(self, s, q, gauss=False, threads=0):
        s, q = _i32(s), _i32(q)
        o = np.empty(self.volume, dtype=np.float64)
        lib().orc_kernel1(self._c, int(gauss), s, q, len(s), o, int(threads))
        return o

    def coulomb_cpu(self, e_site, e_fsite, h_site, h_fsite, d_site=(), defects_charge=0,
                    e_type=None, h_type=None, exciton_binding=0.0, threads=0,
                    want_potentials=False):
        e_site, e_fsite = _i32(e_site), _i32(e_fsite)
        h_site, h_fsite = _i32(h_site), _i32(h_fsite)
        d_site = _i32(d_site)
        nv = self.volume + 35
        if e_type is None:
            e_type = np.zeros(nv, dtype=np.uint8)
            e_type[e_site] = ELECTRON
        if h_type is None:
            h_type = np.zeros(nv, dtype=np.uint8)
            h_type[h_site] = HOLE
        n = len(e_site) + len(h_site)
        de = np.empty(n, dtype=np.float64)
        p1 = np.empty(n, dtype=np.float64) if want_potentials else None
        p2 = np.empty(n, dtype=np.float64) if want_potentials else None
        lib().orc_coulomb_cpu(
            self._c, e_site, e_fsite, len(e_site), h_site, h_fsite, len(h_site), d_site,
            len(d_site), int(defects_charge), np.ascontiguousarray(e_type, dtype=np.uint8),
            np.ascontiguousarray(h_type, dtype=np.uint8), float(exciton_binding), de,
            p1.ctypes.data if p1 is not None else None,
            p2.ctypes.data if p2 is not None else None, int(threads))
        if want_potentials:
            return de, p1, p2
        return de


class KmcOracle:
    """The oracle's kMC step on a world (site energies, defects, carriers)."""

    def __init__(self, orc: "Oracle", site_energy, defects, electrons, holes, cfg: KmcConfig,
                 step=0, phase=None, bonds=None):
        self.orc = orc
        self.cfg = cfg
        # keep the morphology arrays alive while the config points at them
        self._phase = None if phase is None else np.ascontiguousarray(phase, dtype=np.uint8)
        self._bonds = None if bonds is None else np.ascontiguousarray(bonds, dtype=np.int32)
        if self._phase is not None:
            cfg.phase = self._phase.ctypes.data
        if self._bonds is not None and len(self._bonds):
            cfg.bonds = self._bonds.ctypes.data
            cfg.nbonds = len(self._bonds) // 2
        self.pot = np.ascontiguousarray(site_energy, dtype=np.float64)
        self.defects = np.ascontiguousarray(defects, dtype=np.int32)
        self.e = np.zeros(max(cfg.max_electrons, 1), np.int32)
        self.h = np.zeros(max(cfg.max_holes, 1), np.int32)
        self.ne = ctypes.c_int32(len(electrons))
        self.nh = ctypes.c_int32(len(holes))
        self.e[: len(electrons)] = electrons
        self.h[: len(holes)] = holes
        self.counters = np.zeros(20, np.uint64)
        self.step_no = int(step)

    def step(self, threads=0):
        n = self.ne.value + self.nh.value
        outcome = np.zeros(max(n, 1), np.int32)
        de = np.zeros(max(n, 1), np.float64)
        lib().orc_kmc_step(self.orc._c, ctypes.byref(self.cfg), self.pot, self.defects,
                           len(self.defects), self.step_no, self.e, ctypes.byref(self.ne), self.h,
                           ctypes.byref(self.nh), self.counters, outcome.ctypes.data,
                           de.ctypes.data, int(threads))
        self.step_no += 1
        return outcome[:n].copy(), de[:n].copy()

    def carriers(self):
        return self.e[: self.ne.value].copy(), self.h[: self.nh.value].copy()


def philox4x32_10(ctr, key):
    out = np.empty(4, dtype=np.uint32)
    lib().orc_philox4x32_10(np.asarray(ctr, dtype=np.uint32), np.asarray(key, dtype=np.uint32),
                            out)
    return out


def electrostatic_prefactor(dielectric=3.5):
    """setCalculatedValues (include/parameters.h:384-390) with the reference defaults
    (parameters.h:358-362)."""
    e, eps0, a = 1.60217646e-19, 8.854187817e-12, 1e-9
    return e / (4.0 * np.pi * dielectric * eps0 * a)


def inverse_kt(temperature=300.0):
    """parameters.h:387 with boltzmann.constant 1.3806504e-23."""
    return 1.60217646e-19 / (1.3806504e-23 * temperature)


def ref_kernel2(s, q, n, cutoff, xsize, ysize, prefactor, sigma=0.0, gauss=False,
                work_size=256):
    R = ref_lib()
    if R is None:
        raise RuntimeError("compiled reference kernels not built (oracle/_ref)")
    s, q = _i32(s), _i32(q)
    o = np.empty(len(s), dtype=np.float64)
    rc = R.ref_kernel2(int(gauss), s, q, int(n), len(s), int(cutoff), int(xsize), int(ysize),
                       float(prefactor), float(sigma), int(work_size), o)
    if rc != 0:
        raise RuntimeError(f"ref_kernel2 failed ({rc})")
    return o


def ref_kernel1(s, q, cutoff, dims, prefactor, sigma=0.0, gauss=False, work=(4, 4, 4)):
    R = ref_lib()
    if R is None:
        raise RuntimeError("compiled reference kernels not built (oracle/_ref)")
    s, q = _i32(s), _i32(q)
    o = np.empty(dims[0] * dims[1] * dims[2], dtype=np.float64)
    rc = R.ref_kernel1(int(gauss), s, q, len(s), int(cutoff), dims[0], dims[1], dims[2],
                       float(prefactor), float(sigma), work[0], work[1], work[2], o)
    if rc != 0:
        raise RuntimeError(f"ref_kernel1 failed ({rc})")
    return o
