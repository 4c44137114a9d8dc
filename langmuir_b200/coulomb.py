"""Python face of the Coulomb hot path.

``Coulomb`` wraps one ``lgm_ctx`` (host arrays in, host arrays out, or device
pointers for stream-ordered use).  ``OpenClHelper`` mirrors the reference's
helper class (src/langmuirCore/include/openclhelper.h:22-241): the same method
names, the same packing of electrons, holes and charged defects
(openclhelper.cpp:372-544) and the same ``m_offset`` semantics of
``getOutputHost`` / ``getOutputHostFuture`` (openclhelper.cpp:567-583), with
errors raised instead of qFatal.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())


def _out(out, n: int) -> np.ndarray:
    """A caller's output array (float64, C-contiguous, n long), or a new one."""
    if out is None:
        return np.empty(n, dtype=np.float64)
    if (not isinstance(out, np.ndarray) or out.dtype != np.float64 or out.shape != (n,)
            or not out.flags.c_contiguous):
        raise ValueError(f"out must be a C-contiguous float64 array of length {n}")
    return out


class Coulomb:
    """One B200 context: lattice, cutoff, prefactor, sigma, precision, path."""

    def __init__(self, grid_x=128, grid_y=128, grid_z=1, cutoff=50, prefactor=None, sigma=0.0,
                 device=0, precision=N.PREC_FP32C, path=N.PATH_RSQRT, max_charges=0,
                 max_targets=0):
        cfg = N.default_config()
        cfg.grid_x, cfg.grid_y, cfg.grid_z = int(grid_x), int(grid_y), int(grid_z)
        cfg.electrostatic_cutoff = int(cutoff)
        if prefactor is not None:
            cfg.electrostatic_prefactor = float(prefactor)
        cfg.coulomb_gaussian_sigma = float(sigma)
        cfg.precision = int(precision)
        cfg.path = int(path)
        cfg.max_charges = int(max_charges)
        cfg.max_targets = int(max_targets)
        self.config = cfg
        self.volume = cfg.grid_x * cfg.grid_y * cfg.grid_z
        h = ctypes.c_void_p()
        N.check(N.lib().lgm_create(ctypes.byref(cfg), int(device), ctypes.byref(h)), None)
        self._h = h

    @property
    def prefactor(self) -> float:
        return self.config.electrostatic_prefactor

    def close(self):
        h = getattr(self, "_h", None)
        if h and h.value and N._lib is not None:
            N._lib.lgm_destroy(h)
        self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st):
        N.check(st, self._h)

    # -- host-buffer entry points ----------------------------------------------
    def potentials(self, src_site, src_q, tgt_site, kind=N.POINT, terms=N.TERM_DIRECT, out=None):
        """Potentials at the targets (lgm_potentials).  out: a float64 array
        of len(tgt_site) to fill and return (a caller stepping a simulation
        reuses one), else a new one."""
        s, q, t = _i32(src_site), _i32(src_q), _i32(tgt_site)
        if len(s) != len(q):
            raise ValueError("src_site and src_q differ in length")
        out = _out(out, len(t))
        self._check(N.lib().lgm_potentials(self._h, int(kind), int(terms), s, q, len(s), t,
                                           len(t), out))
        return out

    def kernel2(self, s, q, n, kind=N.POINT, out=None):
        s, q = _i32(s), _i32(q)
        out = _out(out, len(s))
        self._check(N.lib().lgm_coulomb_kernel2(self._h, int(kind), s, q, int(n), len(s), out))
        return out

    def kernel1(self, s, q, kind=N.POINT):
        s, q = _i32(s), _i32(q)
        out = np.empty(self.volume, dtype=np.float64)
        self._check(N.lib().lgm_coulomb_kernel1(self._h, int(kind), s, q, len(s), out))
        return out

    # -- device-pointer entry points (integers are CUDA device addresses) ------
    def potentials_async(self, d_src_site, d_src_q, n, d_tgt_site, t, d_out, kind=N.POINT,
                         terms=N.TERM_DIRECT, stream=0):
        self._check(N.lib().lgm_potentials_async(self._h, int(kind), int(terms), d_src_site,
                                                 d_src_q, int(n), d_tgt_site, int(t), d_out,
                                                 stream or None))

    def kernel1_async(self, d_s, d_q, n, d_out, kind=N.POINT, stream=0):
        self._check(N.lib().lgm_coulomb_kernel1_async(self._h, int(kind), d_s, d_q, int(n),
                                                      d_out, stream or None))

    def sync(self, stream=0):
        self._check(N.lib().lgm_sync(self._h, stream or None))

    def autotune(self, n, t, kind=N.POINT, terms=N.TERM_DIRECT) -> int:
        v = ctypes.c_int32(-1)
        self._check(N.lib().lgm_autotune(self._h, int(kind), int(terms), int(n), int(t),
                                         ctypes.byref(v)))
        return v.value

    def set_variant(self, v: int):
        self._check(N.lib().lgm_set_variant(self._h, int(v)))

    @staticmethod
    def variants():
        out = []
        for v in range(N.lib().lgm_variant_count()):
            a, b, c = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
            N.lib().lgm_variant_info(v, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
            f = ctypes.c_int32()
            N.lib().lgm_variant_flags(v, ctypes.byref(f))
            k, st = ctypes.c_int32(), ctypes.c_int32()
            N.lib().lgm_variant_items(v, ctypes.byref(k), ctypes.byref(st))
            out.append({"threads": a.value, "target_pairs": b.value, "run": c.value,
                        "warp_skip": bool(f.value & 1), "culled": bool(f.value & 2),
                        "warp_specialised": bool(f.value & 4), "chunks_per_item": k.value,
                        "stages": st.value})
        return out

    def set_timing(self, on: bool = True):
        self._check(N.lib().lgm_set_timing(self._h, int(bool(on))))

    def set_launch_overlap(self, on: bool = True):
        """Programmatic stream serialization between the call's kernels
        (lgm_set_launch_overlap); on by default, the same results either way."""
        self._check(N.lib().lgm_set_launch_overlap(self._h, int(bool(on))))

    def set_counting(self, on: bool = True):
        """Culled pair sums count the pairs they examine (lgm_set_counting)."""
        self._check(N.lib().lgm_set_counting(self._h, int(bool(on))))

    def last_launch(self) -> dict:
        info = N.LaunchInfo()
        self._check(N.lib().lgm_last_launch(self._h, ctypes.byref(info)))
        return {k: getattr(info, k) for k, _ in N.LaunchInfo._fields_}


class Carrier:
    """The parts of a ChargeAgent the helper reads and writes
    (chargeagent.h: getCurrentSite, getFutureSite, charge, setOpenCLID)."""

    __slots__ = ("site", "future_site", "charge", "opencl_id")

    def __init__(self, site, charge, future_site=None):
        self.site = int(site)
        self.future_site = int(site if future_site is None else future_site)
        self.charge = int(charge)
        self.opencl_id = 0


class OpenClHelper:
    """Mirror of LangmuirCore::OpenClHelper over the B200 library.

    ``world`` provides ``electrons`` and ``holes`` (lists of Carrier),
    ``defect_site_ids`` (list of int) and ``parameters`` (a mapping of the
    reference's input keys: grid.x, grid.y, grid.z, electrostatic.cutoff,
    electrostatic.prefactor, coulomb.gaussian.sigma, defects.charge,
    use.opencl, coulomb.carriers)."""

    def __init__(self, world):
        self.world = world
        self.ok_cl = False
        self.use_opencl = False
        self._ctx = None
        self._ctx64 = None
        self._o = np.zeros(0, dtype=np.float64)
        self._s = np.zeros(0, dtype=np.int32)
        self._q = np.zeros(0, dtype=np.int32)
        self._kind = N.POINT
        self._offset = 0

    # openclhelper.cpp:17-187
    def initializeOpenCL(self, gpuID=-1):
        p = self.world.parameters
        self.ok_cl = False
        for ctx in (self._ctx, self._ctx64):
            if ctx is not None:
                ctx.close()
        self._ctx = self._ctx64 = None
        self._device = max(int(gpuID), 0)
        try:
            self._ctx = Coulomb(**self._context_args(), device=self._device)
        except (N.LgmError, ImportError):
            if p.get("use.opencl", False):
                raise
            return
        self.ok_cl = True

    def _context_args(self):
        p = self.world.parameters
        return dict(grid_x=p["grid.x"], grid_y=p["grid.y"], grid_z=p["grid.z"],
                    cutoff=p.get("electrostatic.cutoff", 50),
                    prefactor=p.get("electrostatic.prefactor"),
                    sigma=p.get("coulomb.gaussian.sigma", 0.0))

    # openclhelper.cpp:190-218
    def toggleOpenCL(self, on: bool) -> bool:
        p = self.world.parameters
        if on and self.ok_cl and p.get("coulomb.carriers", False):
            self.use_opencl = True
        else:
            self.use_opencl = False
        return self.use_opencl

    def _pack(self, future: bool):
        """Host packing of openclhelper.cpp:380-424 (or 228-255 for kernel 1)."""
        w = self.world
        s, q = [], []
        for i, c in enumerate(w.electrons):
            s.append(c.site); q.append(c.charge); c.opencl_id = i
        ne = len(w.electrons)
        for i, c in enumerate(w.holes):
            s.append(c.site); q.append(c.charge); c.opencl_id = i + ne
        dq = int(w.parameters.get("defects.charge", 0))
        if dq != 0:
            for site in w.defect_site_ids:
                s.append(site); q.append(dq)
        self._offset = len(s)
        if future:
            for c in w.electrons:
                s.append(c.future_site); q.append(c.charge)
            for c in w.holes:
                s.append(c.future_site); q.append(c.charge)
        self._s, self._q = _i32(s), _i32(q)
        return self._s, self._q

    def _require(self):
        if self._ctx is None:
            raise N.LgmError(N.ERR_STATE, "initializeOpenCL() has not succeeded")

    def launchCoulombKernel2(self):
        self._require()
        s, q = self._pack(True)
        self._kind = N.POINT
        self._o = self._ctx.kernel2(s, q, self._offset, N.POINT)

    def launchGaussKernel2(self):
        self._require()
        s, q = self._pack(True)
        self._kind = N.GAUSS
        self._o = self._ctx.kernel2(s, q, self._offset, N.GAUSS)

    def launchCoulombKernel1(self):
        self._require()
        s, q = self._pack(False)
        self._o = self._ctx.kernel1(s, q, N.POINT)

    def launchGaussKernel1(self):
        self._require()
        s, q = self._pack(False)
        self._o = self._ctx.kernel1(s, q, N.GAUSS)

    def getOutputHost(self, index: int) -> float:
        return float(self._o[index])

    def getOutputHostFuture(self, index: int) -> float:
        return float(self._o[index + self._offset])

    # openclhelper.cpp:560-565: one entry of the host site and charge mirrors
    # (the next launch packs them from the world again, as the reference does)
    def copySiteAndChargeToHostVector(self, index: int, site: int, charge: int = -1):
        if index >= len(self._s):
            self._s = np.resize(self._s, index + 1)
            self._q = np.resize(self._q, index + 1)
        self._s[index] = site
        self._q[index] = charge

    # openclhelper.cpp:546-558 and ChargeAgent::compareCoulomb
    # (chargeagent.cpp:298-370)
    def compareHostAndDeviceForAllCarriers(self):
        """Every carrier's potentials from the last kernel-2 launch against
        FP64 sums over the same sources (a second context in FP64, made on the
        first call).  A carrier fails when its energy change differs by more
        than 1e-4 (signed, as the reference tests it) or either potential by
        more than 1e-4 percent.  Returns (number failed, per-carrier rows
        (gpu1, gpu2, cpu1, cpu2, gpu, cpu, failed) in opencl_id order), where
        the reference prints each comparison."""
        self._require()
        nc = len(self.world.electrons) + len(self.world.holes)
        if nc == 0 or len(self._o) < self._offset + nc:
            return 0, []
        if self._ctx64 is None:
            self._ctx64 = Coulomb(**self._context_args(), device=self._device,
                                  precision=N.PREC_FP64)
        src, q = self._s[: self._offset], self._q[: self._offset]
        tgt = np.concatenate([self._s[:nc], self._s[self._offset: self._offset + nc]])
        cpu = self._ctx64.potentials(src, q, tgt, self._kind)
        selfterm = self._ctx.prefactor * self._q[:nc].astype(np.float64)  # iR[1][0][0] = 1
        gpu1 = self._o[:nc]
        gpu2 = self._o[self._offset: self._offset + nc] - selfterm
        cpu1, cpu2 = cpu[:nc], cpu[nc:] - selfterm
        qd = self._q[:nc].astype(np.float64)
        gpu, cpuv = qd * (gpu2 - gpu1), qd * (cpu2 - cpu1)

        def pdiff(a, b):
            with np.errstate(invalid="ignore", divide="ignore"):
                return np.abs(a - b) / (0.5 * (np.abs(b) + np.abs(a))) * 100.0
        failed = ((gpu - cpuv) > 1e-4) | (pdiff(gpu1, cpu1) > 1e-4) | (pdiff(gpu2, cpu2) > 1e-4)
        rows = list(zip(gpu1, gpu2, cpu1, cpu2, gpu, cpuv, failed))
        return int(failed.sum()), rows
