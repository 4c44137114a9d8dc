"""Input keys and the GPU kMC step (include/langmuir_b200_kmc.h) from Python.

``Params`` mirrors ``lgm_params``: every key of the reference's KeyValueParser
(keyvalueparser.cpp:15-105) as an attribute named with underscores
(``grid.x`` -> ``grid_x``), defaults from SimulationParameters
(parameters.h:285-378).  ``Params.parse(text)`` reads a Langmuir input file;
``check()`` derives the prefactor and 1/kT and validates.

``KMC`` is one replica stepped on the GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N

_i32 = ctypes.c_int32
_f64 = ctypes.c_double

# LGM_GUARD_BAND_MIN (langmuir_b200_kmc.h): the narrowest FP64 guard band, the
# FP32C error bound of a decision's potentials relative to their scale N.
GUARD_BAND_MIN = 8e-6


class Params(ctypes.Structure):
    _fields_ = [
        ("simulation_type", ctypes.c_char * 16), ("current_step", ctypes.c_uint32),
        ("iterations_real", _i32), ("random_seed", ctypes.c_uint64),
        ("grid_z", _i32), ("grid_y", _i32), ("grid_x", _i32), ("hopping_range", _i32),
        ("output_is_on", _i32), ("iterations_print", _i32), ("output_precision", _i32),
        ("output_width", _i32), ("output_stub", ctypes.c_char * 64),
        ("output_ids_on_delete", _i32), ("output_ids_on_encounter", _i32),
        ("output_coulomb", _i32), ("output_step_chk", _i32),
        ("output_chk_trap_potential", _i32), ("output_potential", _i32),
        ("output_xyz", _i32), ("output_xyz_e", _i32), ("output_xyz_h", _i32),
        ("output_xyz_d", _i32), ("output_xyz_t", _i32), ("output_xyz_mode", _i32),
        ("image_traps", _i32), ("image_defects", _i32), ("image_carriers", _i32),
        ("electron_percentage", _f64), ("hole_percentage", _f64), ("seed_charges", _f64),
        ("defect_percentage", _f64), ("trap_percentage", _f64), ("trap_potential", _f64),
        ("gaussian_stdev", _f64), ("seed_percentage", _f64),
        ("voltage_right", _f64), ("voltage_left", _f64), ("slope_z", _f64),
        ("coulomb_carriers", _i32), ("coulomb_gaussian_sigma", _f64), ("defects_charge", _i32),
        ("exciton_binding", _f64), ("temperature_kelvin", _f64),
        ("source_rate", _f64), ("e_source_l_rate", _f64), ("e_source_r_rate", _f64),
        ("h_source_l_rate", _f64), ("h_source_r_rate", _f64), ("generation_rate", _f64),
        ("source_metropolis", _i32), ("source_coulomb", _i32), ("source_scale_area", _f64),
        ("balance_charges", _i32),
        ("drain_rate", _f64), ("e_drain_l_rate", _f64), ("e_drain_r_rate", _f64),
        ("h_drain_l_rate", _f64), ("h_drain_r_rate", _f64),
        ("recombination_rate", _f64), ("recombination_range", _i32),
        ("use_opencl", _i32), ("work_x", _i32), ("work_y", _i32), ("work_z", _i32),
        ("work_size", _i32), ("opencl_threshold", _i32), ("opencl_device_id", _i32),
        ("max_threads", _i32),
        ("boltzmann_constant", _f64), ("dielectric_constant", _f64),
        ("elementary_charge", _f64), ("permittivity_space", _f64), ("grid_factor", _f64),
        ("electrostatic_cutoff", _i32), ("electrostatic_prefactor", _f64), ("inverse_kt", _f64),
        ("image_charges", _i32), ("site_disorder", _f64),
        ("morphology_confine", _i32), ("generation_interface", _i32),
        ("guard_band", _f64),
    ]

    @classmethod
    def default(cls, **keys) -> "Params":
        p = cls()
        N.lib().lgm_params_default(ctypes.byref(p))
        for k, v in keys.items():
            p.set(k, v)
        return p

    def set(self, key: str, value):
        name = key.replace(".", "_")
        if not hasattr(self, name):
            raise KeyError(key)
        if isinstance(getattr(self, name), bytes):
            value = value.encode() if isinstance(value, str) else value
        setattr(self, name, value)

    def parse(self, text: str) -> "Params":
        err = ctypes.create_string_buffer(512)
        st = N.lib().lgm_params_parse(text.encode(), ctypes.byref(self), err, len(err))
        if st != N.OK:
            raise N.LgmError(st, err.value.decode())
        return self

    @classmethod
    def from_text(cls, text: str) -> "Params":
        return cls.default().parse(text)

    def format(self) -> str:
        """The [Parameters] section of a checkpoint (lgm_params_format)."""
        need = N.lib().lgm_params_format(ctypes.byref(self), None, 0)
        buf = ctypes.create_string_buffer(need)
        N.lib().lgm_params_format(ctypes.byref(self), buf, need)
        return buf.value.decode()

    def check(self) -> "Params":
        err = ctypes.create_string_buffer(512)
        st = N.lib().lgm_params_check(ctypes.byref(self), err, len(err))
        if st != N.OK:
            raise N.LgmError(st, err.value.decode())
        return self


class Stats(ctypes.Structure):
    _fields_ = [("step", ctypes.c_uint32), ("electrons", _i32), ("holes", _i32),
                ("max_electrons", _i32), ("max_holes", _i32), ("defects", _i32),
                ("traps", _i32), ("proposals", ctypes.c_uint64), ("accepted", ctypes.c_uint64),
                ("guard_evaluations", ctypes.c_uint64), ("counters", ctypes.c_uint64 * 20)]


_vp = ctypes.c_void_p
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")

class WorldConfig(ctypes.Structure):
    """lgm_world_config: a world restored from a checkpoint."""
    _fields_ = [("electrons", ctypes.c_void_p), ("n_electrons", _i32),
                ("holes", ctypes.c_void_p), ("n_holes", _i32),
                ("defects", ctypes.c_void_p), ("n_defects", _i32),
                ("traps", ctypes.c_void_p), ("n_traps", _i32),
                ("trap_potentials", ctypes.c_void_p), ("n_trap_potentials", _i32),
                ("flux", ctypes.c_void_p), ("n_flux", _i32)]


N.SIGNATURES.update({
    "lgm_params_default": (None, [ctypes.POINTER(Params)]),
    "lgm_params_format": (_i32, [ctypes.POINTER(Params), ctypes.c_char_p, _i32]),
    "lgm_kmc_create_from": (_i32, [ctypes.POINTER(Params), ctypes.POINTER(WorldConfig), _i32,
                                   ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p)]),
    "lgm_params_size": (_i32, []),
    "lgm_params_parse": (_i32, [ctypes.c_char_p, ctypes.POINTER(Params), ctypes.c_char_p, _i32]),
    "lgm_params_check": (_i32, [ctypes.POINTER(Params), ctypes.c_char_p, _i32]),
    "lgm_kmc_create": (_i32, [ctypes.POINTER(Params), _i32, ctypes.c_uint32,
                              ctypes.POINTER(_vp)]),
    "lgm_kmc_destroy": (_i32, [_vp]),
    "lgm_kmc_last_error": (ctypes.c_char_p, [_vp]),
    "lgm_kmc_run": (_i32, [_vp, _i32]),
    "lgm_kmc_stats_get": (_i32, [_vp, ctypes.POINTER(Stats)]),
    "lgm_kmc_get_carriers": (_i32, [_vp, _i32p, _i32, _i32p, _i32]),
    "lgm_kmc_set_carriers": (_i32, [_vp, _i32p, _i32, _i32p, _i32]),
    "lgm_kmc_get_world": (_i32, [_vp, _vp, _vp, _i32, _vp, _vp, _i32]),
    "lgm_kmc_last_outcomes": (_i32, [_vp, _vp, _vp, _i32]),
    "lgm_kmc_set_morphology": (_i32, [_vp, np.ctypeslib.ndpointer(dtype=np.uint8,
                                                                  flags="C_CONTIGUOUS")]),
    "lgm_kmc_world_host": (_i32, [ctypes.POINTER(Params), ctypes.c_uint32, _vp, _vp, _i32, _vp,
                                  _vp, _i32, _vp, _i32, _vp, _i32, _vp]),
})
if N._lib is not None:  # bind the new symbols if the library was already loaded
    for _name in ("lgm_params_default", "lgm_params_format", "lgm_kmc_create_from",
                  "lgm_params_size", "lgm_params_parse",
                  "lgm_params_check", "lgm_kmc_create", "lgm_kmc_destroy", "lgm_kmc_last_error",
                  "lgm_kmc_run", "lgm_kmc_stats_get", "lgm_kmc_get_carriers",
                  "lgm_kmc_set_carriers", "lgm_kmc_get_world", "lgm_kmc_last_outcomes",
                  "lgm_kmc_set_morphology", "lgm_kmc_world_host"):
        _fn = getattr(N._lib, _name)
        _fn.restype, _fn.argtypes = N.SIGNATURES[_name]


def world_host(params: Params, replica: int = 0) -> dict:
    """The world a replica starts from, built on the host alone
    (lgm_kmc_world_host): site energies, defects, traps with their
    potentials, and the seeded electron and hole lists."""
    V = params.grid_x * params.grid_y * params.grid_z
    cap = V
    pot = np.zeros(V, np.float64)
    d = np.zeros(cap, np.int32)
    t = np.zeros(cap, np.int32)
    tp = np.zeros(cap, np.float64)
    e = np.zeros(cap, np.int32)
    h = np.zeros(cap, np.int32)
    cnt = np.zeros(4, np.int32)
    st = N.lib().lgm_kmc_world_host(ctypes.byref(params), int(replica), pot.ctypes.data,
                                    d.ctypes.data, cap, t.ctypes.data, tp.ctypes.data, cap,
                                    e.ctypes.data, cap, h.ctypes.data, cap, cnt.ctypes.data)
    if st != N.OK:
        raise N.LgmError(st, (N.lib().lgm_kmc_last_error(None) or b"").decode())
    nd, nt, ne, nh = (int(x) for x in cnt)
    return dict(site_energy=pot, defects=d[:nd].copy(), traps=t[:nt].copy(),
                trap_potentials=tp[:nt].copy(), electrons=e[:ne].copy(), holes=h[:nh].copy())


class KMC:
    """One replica on the GPU: the world is built from ``params`` and the
    (random.seed, replica) Philox stream."""

    def __init__(self, params: Params, device: int = 0, replica: int = 0, world=None):
        """world: optional dict of site lists restored from a checkpoint --
        electrons, holes, defects, traps, trap_potentials, flux (see
        lgm_world_config) -- placed before the rest is drawn."""
        h = ctypes.c_void_p()
        if world is None:
            st = N.lib().lgm_kmc_create(ctypes.byref(params), int(device), int(replica),
                                        ctypes.byref(h))
        else:
            keep = []

            def arr(key, dtype):
                a = np.ascontiguousarray(world.get(key, []), dtype=dtype)
                keep.append(a)
                return (a.ctypes.data if a.size else None), int(a.size)
            w = WorldConfig()
            for key, dt in (("electrons", np.int32), ("holes", np.int32), ("defects", np.int32),
                            ("traps", np.int32), ("trap_potentials", np.float64),
                            ("flux", np.uint64)):
                ptr, n = arr(key, dt)
                setattr(w, key, ptr)
                setattr(w, "n_" + key, n)
            st = N.lib().lgm_kmc_create_from(ctypes.byref(params), ctypes.byref(w), int(device),
                                             int(replica), ctypes.byref(h))
        if st != N.OK:
            raise N.LgmError(st, N.lib().lgm_kmc_last_error(None).decode())
        self._h = h
        self.params = params
        self.replica = int(replica)
        self.volume = params.grid_x * params.grid_y * params.grid_z

    def _check(self, st):
        if st != N.OK:
            raise N.LgmError(st, N.lib().lgm_kmc_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None) and self._h.value and N._lib is not None:
            N._lib.lgm_kmc_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self, steps: int):
        self._check(N.lib().lgm_kmc_run(self._h, int(steps)))

    def stats(self) -> dict:
        s = Stats()
        self._check(N.lib().lgm_kmc_stats_get(self._h, ctypes.byref(s)))
        d = {k: getattr(s, k) for k, _ in Stats._fields_ if k != "counters"}
        d["counters"] = list(s.counters)
        return d

    def carriers(self):
        s = self.stats()
        e = np.zeros(max(s["max_electrons"], 1), np.int32)
        h = np.zeros(max(s["max_holes"], 1), np.int32)
        self._check(N.lib().lgm_kmc_get_carriers(self._h, e, len(e), h, len(h)))
        return e[: s["electrons"]].copy(), h[: s["holes"]].copy()

    def set_carriers(self, e, h):
        e = np.ascontiguousarray(e, dtype=np.int32)
        h = np.ascontiguousarray(h, dtype=np.int32)
        self._check(N.lib().lgm_kmc_set_carriers(self._h, e, len(e), h, len(h)))

    def world(self):
        s = self.stats()
        pot = np.zeros(self.volume, np.float64)
        d = np.zeros(max(s["defects"], 1), np.int32)
        t = np.zeros(max(s["traps"], 1), np.int32)
        tp = np.zeros(max(s["traps"], 1), np.float64)
        self._check(N.lib().lgm_kmc_get_world(self._h, pot.ctypes.data, d.ctypes.data, len(d),
                                              t.ctypes.data, tp.ctypes.data, len(t)))
        return dict(site_energy=pot, defects=d[: s["defects"]].copy(),
                    traps=t[: s["traps"]].copy(), trap_potentials=tp[: s["traps"]].copy())

    def set_morphology(self, phase):
        """phase[site]: 0 donor, 1 acceptor (x fastest, then y, then z)."""
        ph = np.ascontiguousarray(np.asarray(phase).reshape(-1), dtype=np.uint8)
        if ph.size != self.volume:
            raise ValueError("phase must have one entry per lattice site")
        self._check(N.lib().lgm_kmc_set_morphology(self._h, ph))

    def last_outcomes(self, n):
        o = np.zeros(max(n, 1), np.int32)
        de = np.zeros(max(n, 1), np.float64)
        self._check(N.lib().lgm_kmc_last_outcomes(self._h, o.ctypes.data, de.ctypes.data, len(o)))
        return o[:n].copy(), de[:n].copy()


N.SIGNATURES.update({
    "lgm_kmc_batch_create": (_i32, [ctypes.POINTER(Params), _i32, _i32, ctypes.c_uint32,
                                    ctypes.POINTER(_vp)]),
    "lgm_kmc_batch_destroy": (_i32, [_vp]),
    "lgm_kmc_batch_last_error": (ctypes.c_char_p, [_vp]),
    "lgm_kmc_batch_run": (_i32, [_vp, _i32]),
    "lgm_kmc_batch_size": (_i32, [_vp]),
    "lgm_kmc_batch_replica": (_vp, [_vp, _i32]),
    "lgm_kmc_batch_tuning": (_i32, [_vp, ctypes.POINTER(_i32), ctypes.POINTER(_i32),
                                    ctypes.POINTER(_i32), ctypes.POINTER(_i32)]),
    "lgm_kmc_batch_set_fused": (_i32, [_vp, _i32]),
    "lgm_kmc_batch_fused_count": (_i32, [_vp]),
    "lgm_kmc_batch_time_pair": (_i32, [_vp, _i32, ctypes.POINTER(ctypes.c_float)]),
    "lgm_kmc_batch_count_pairs": (_i32, [_vp, ctypes.POINTER(ctypes.c_uint64)]),
    "lgm_kmc_batch_culled_count": (_i32, [_vp]),
})
if N._lib is not None:
    for _name in ("lgm_kmc_batch_create", "lgm_kmc_batch_destroy", "lgm_kmc_batch_last_error",
                  "lgm_kmc_batch_run", "lgm_kmc_batch_size", "lgm_kmc_batch_replica",
                  "lgm_kmc_batch_tuning", "lgm_kmc_batch_set_fused", "lgm_kmc_batch_fused_count",
                  "lgm_kmc_batch_time_pair", "lgm_kmc_batch_count_pairs",
                  "lgm_kmc_batch_culled_count"):
        _fn = getattr(N._lib, _name)
        _fn.restype, _fn.argtypes = N.SIGNATURES[_name]


class _Borrowed(KMC):
    """A replica owned by a batch (accessors only)."""

    def __init__(self, handle, params):
        self._h = ctypes.c_void_p(handle)
        self.params = params
        self.volume = params.grid_x * params.grid_y * params.grid_z

    def close(self):
        self._h = None

    def run(self, steps):
        raise RuntimeError("run the batch, not one of its replicas")


class KMCBatch:
    """Replicas of uneven size advanced together on one GPU; replica i has the
    random stream of a single replica with id replica0 + i."""

    def __init__(self, params_list, device=0, replica0=0, fused_max_charges=None):
        """``fused_max_charges``: replicas with room for at most this many
        charges advance by the fused one-block step (None: the library's
        default bound, 0: none)."""
        arr = (Params * len(params_list))(*params_list)
        h = ctypes.c_void_p()
        st = N.lib().lgm_kmc_batch_create(arr, len(params_list), int(device), int(replica0),
                                          ctypes.byref(h))
        if st != N.OK:
            raise N.LgmError(st, N.lib().lgm_kmc_batch_last_error(None).decode())
        self._h = h
        self._params = list(params_list)
        if fused_max_charges is not None:
            st = N.lib().lgm_kmc_batch_set_fused(self._h, int(fused_max_charges))
            if st != N.OK:
                raise N.LgmError(st, N.lib().lgm_kmc_batch_last_error(self._h).decode())

    @property
    def fused_count(self) -> int:
        """Replicas on the fused step."""
        return N.lib().lgm_kmc_batch_fused_count(self._h)

    @property
    def culled_count(self) -> int:
        """Replicas whose pair sum culls source chunks beyond the cutoff."""
        return N.lib().lgm_kmc_batch_culled_count(self._h)

    def close(self):
        if getattr(self, "_h", None) and self._h.value and N._lib is not None:
            N._lib.lgm_kmc_batch_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return N.lib().lgm_kmc_batch_size(self._h)

    def run(self, steps):
        st = N.lib().lgm_kmc_batch_run(self._h, int(steps))
        if st != N.OK:
            raise N.LgmError(st, N.lib().lgm_kmc_batch_last_error(self._h).decode())

    def replica(self, i) -> KMC:
        ptr = N.lib().lgm_kmc_batch_replica(self._h, int(i))
        if not ptr:
            raise IndexError(i)
        return _Borrowed(ptr, self._params[i])

    def tuning(self) -> dict:
        a, b, c, d = (ctypes.c_int32() for _ in range(4))
        N.lib().lgm_kmc_batch_tuning(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                     ctypes.byref(d))
        return {"threads": a.value, "target_pairs": b.value, "chunks_per_item": c.value,
                "items": d.value}

    def time_pair(self, reps: int = 5) -> float:
        """Median CUDA-event time (ms) of the batched pair sum alone, over
        the charges the last step packed."""
        ms = ctypes.c_float()
        st = N.lib().lgm_kmc_batch_time_pair(self._h, int(reps), ctypes.byref(ms))
        if st != N.OK:
            raise N.LgmError(st, N.lib().lgm_kmc_batch_last_error(self._h).decode())
        return ms.value

    def count_pairs(self) -> int:
        """Source-target pairs the batched pair sum examines over the charges
        the last step packed (culled replicas: the pairs of source groups
        within the cutoff of a warp's targets; the others: all pairs)."""
        n = ctypes.c_uint64()
        st = N.lib().lgm_kmc_batch_count_pairs(self._h, ctypes.byref(n))
        if st != N.OK:
            raise N.LgmError(st, N.lib().lgm_kmc_batch_last_error(self._h).decode())
        return n.value
