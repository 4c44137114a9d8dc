"""ctypes binding of the C ABI (include/langmuir_b200.h).

This is the path LangmuirPython reaches the B200 kernels through.  There is
no fallback: if ``_lib/liblangmuir_b200.so`` is missing, importing the native
layer raises, and every compute call goes to the CUDA library.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "_lib", "liblangmuir_b200.so")

# status codes (langmuir_b200.h)
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_OUT_OF_RANGE = 2
ERR_CUDA = 3
ERR_NO_DEVICE = 4
ERR_CAPACITY = 5
ERR_TIMEOUT = 6
ERR_PARSE = 7
ERR_UNSUPPORTED = 8
ERR_STATE = 9

POINT, GAUSS = 0, 1
PREC_FP32C, PREC_FP64 = 0, 1
PATH_RSQRT, PATH_TABLE, PATH_TABLE64 = 0, 1, 2
TERM_DIRECT, TERM_IMAGE_LEFT, TERM_IMAGE_RIGHT = 1, 2, 4


class LgmError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class Config(ctypes.Structure):
    _fields_ = [
        ("grid_x", ctypes.c_int32), ("grid_y", ctypes.c_int32), ("grid_z", ctypes.c_int32),
        ("electrostatic_cutoff", ctypes.c_int32),
        ("electrostatic_prefactor", ctypes.c_double),
        ("coulomb_gaussian_sigma", ctypes.c_double),
        ("work_x", ctypes.c_int32), ("work_y", ctypes.c_int32), ("work_z", ctypes.c_int32),
        ("work_size", ctypes.c_int32),
        ("opencl_threshold", ctypes.c_int32),
        ("max_charges", ctypes.c_int32),
        ("max_targets", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("path", ctypes.c_int32),
    ]


class LaunchInfo(ctypes.Structure):
    _fields_ = [
        ("pairs_tested", ctypes.c_int64),
        ("ctas", ctypes.c_int32),
        ("splits", ctypes.c_int32),
        ("threads", ctypes.c_int32),
        ("targets_per_thread", ctypes.c_int32),
        ("kernel_launches", ctypes.c_int32),
        ("pair_kernel_ms", ctypes.c_float),
        ("variant", ctypes.c_int32),
        ("pairs_examined", ctypes.c_int64),
    ]


class Peaks(ctypes.Structure):
    """lgm_peaks: measured FP32 FMA and MUFU rsqrt throughput."""
    _fields_ = [("ffma_tflops", ctypes.c_double), ("ffma2_tflops", ctypes.c_double),
                ("rsqrt_per_s", ctypes.c_double), ("sm_count", ctypes.c_int32),
                ("clock_mhz_attribute", ctypes.c_double)]


def probe_peaks(device=0) -> dict:
    """lgm_probe_peaks: FFMA, FFMA2 and MUFU rsqrt rates measured on `device`."""
    p = Peaks()
    st = lib().lgm_probe_peaks(int(device), ctypes.byref(p))
    if st != OK:
        raise LgmError(st, "lgm_probe_peaks")
    return {k: getattr(p, k) for k, _ in Peaks._fields_}


_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_vp = ctypes.c_void_p

# Every symbol include/langmuir_b200.h declares, with its ctypes signature.
SIGNATURES = {
    "lgm_abi_version": (ctypes.c_int32, []),
    "lgm_status_string": (ctypes.c_char_p, [ctypes.c_int32]),
    "lgm_config_default": (None, [ctypes.POINTER(Config)]),
    "lgm_create": (ctypes.c_int32, [ctypes.POINTER(Config), ctypes.c_int32, ctypes.POINTER(_vp)]),
    "lgm_destroy": (ctypes.c_int32, [_vp]),
    "lgm_last_error": (ctypes.c_char_p, [_vp]),
    "lgm_potentials": (ctypes.c_int32, [_vp, ctypes.c_int32, ctypes.c_uint32, _i32p, _i32p,
                                        ctypes.c_int32, _i32p, ctypes.c_int32, _f64p]),
    "lgm_potentials_async": (ctypes.c_int32, [_vp, ctypes.c_int32, ctypes.c_uint32, _vp, _vp,
                                              ctypes.c_int32, _vp, ctypes.c_int32, _vp, _vp]),
    "lgm_sync": (ctypes.c_int32, [_vp, _vp]),
    "lgm_coulomb_kernel2": (ctypes.c_int32, [_vp, ctypes.c_int32, _i32p, _i32p, ctypes.c_int32,
                                             ctypes.c_int32, _f64p]),
    "lgm_coulomb_kernel1": (ctypes.c_int32, [_vp, ctypes.c_int32, _i32p, _i32p, ctypes.c_int32,
                                             _f64p]),
    "lgm_coulomb_kernel1_async": (ctypes.c_int32, [_vp, ctypes.c_int32, _vp, _vp,
                                                   ctypes.c_int32, _vp, _vp]),
    "lgm_last_launch": (ctypes.c_int32, [_vp, ctypes.POINTER(LaunchInfo)]),
    "lgm_set_timing": (ctypes.c_int32, [_vp, ctypes.c_int32]),
    "lgm_set_launch_overlap": (ctypes.c_int32, [_vp, ctypes.c_int32]),
    "lgm_set_counting": (ctypes.c_int32, [_vp, ctypes.c_int32]),
    "lgm_probe_peaks": (ctypes.c_int32, [ctypes.c_int32, _vp]),
    "lgm_selftest_timeout": (ctypes.c_int32, [ctypes.c_int32, ctypes.c_int32]),
    "lgm_autotune": (ctypes.c_int32, [_vp, ctypes.c_int32, ctypes.c_uint32, ctypes.c_int32,
                                      ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    "lgm_set_variant": (ctypes.c_int32, [_vp, ctypes.c_int32]),
    "lgm_coulomb_kernel2_noalloc": (ctypes.c_int32, [ctypes.c_int32, ctypes.c_int32,
                                                     ctypes.c_int32, ctypes.c_int32,
                                                     ctypes.c_double, _vp, _vp, ctypes.c_int32,
                                                     ctypes.c_int32, _vp, _vp]),
    "lgm_variant_count": (ctypes.c_int32, []),
    "lgm_variant_flags": (ctypes.c_int32, [ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    "lgm_variant_items": (ctypes.c_int32, [ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                           ctypes.POINTER(ctypes.c_int32)]),
    "lgm_variant_info": (ctypes.c_int32, [ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                          ctypes.POINTER(ctypes.c_int32),
                                          ctypes.POINTER(ctypes.c_int32)]),
}

_lib = None


def lib():
    """Load the native library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"langmuir_b200 native library missing: {LIB_PATH} "
                "(build it with `python -m langmuir_b200.build`); there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, ctx=None):
    if status != OK:
        msg = lib().lgm_last_error(ctx)
        msg = msg.decode() if msg else lib().lgm_status_string(status).decode()
        raise LgmError(status, msg)


def default_config(**overrides) -> Config:
    cfg = Config()
    lib().lgm_config_default(ctypes.byref(cfg))
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    return cfg
