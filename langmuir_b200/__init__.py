"""langmuir_b200 -- the Coulomb hot path of the Langmuir kMC engine on B200.

Native CUDA (sm_100a) kernels behind a C ABI (include/langmuir_b200.h); this
package is the ctypes face of that ABI.  Importing ``Coulomb`` or
``OpenClHelper`` loads ``_lib/liblangmuir_b200.so`` and fails loudly if it is
missing: there is no CPU fallback.
"""
from ._native import (GAUSS, PATH_RSQRT, PATH_TABLE, PATH_TABLE64, POINT, PREC_FP32C, PREC_FP64,
                      TERM_DIRECT, TERM_IMAGE_LEFT, TERM_IMAGE_RIGHT, LgmError)
from .coulomb import Carrier, Coulomb, OpenClHelper
from .kmc import GUARD_BAND_MIN, KMC, KMCBatch, Params

__all__ = ["GUARD_BAND_MIN", "Coulomb", "OpenClHelper", "Carrier", "KMC", "KMCBatch", "Params", "LgmError", "POINT", "GAUSS", "PREC_FP32C",
           "PREC_FP64", "PATH_RSQRT", "PATH_TABLE", "PATH_TABLE64", "TERM_DIRECT", "TERM_IMAGE_LEFT",
           "TERM_IMAGE_RIGHT"]
