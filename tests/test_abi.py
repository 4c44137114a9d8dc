"""The C ABI library: loads without a GPU and exports every declared symbol."""
import ctypes
import os
import re

import pytest

from langmuir_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h)
           for h in ("langmuir_b200.h", "langmuir_b200_kmc.h", "langmuir_b200_cnn.h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(lgm_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_builds_and_loads():
    from langmuir_b200 import build
    build.build()
    assert os.path.exists(N.LIB_PATH)
    N.lib()


def test_every_declared_symbol_is_exported():
    import langmuir_b200  # noqa: F401  (binds the kMC entry points too)
    import langmuir_b200.surrogate  # noqa: F401  (and the CNN kernels)
    L = ctypes.CDLL(N.LIB_PATH)
    names = declared_functions()
    assert "lgm_coulomb_kernel2" in names and "lgm_create" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # the Python binding covers the whole header
    assert set(names) <= set(N.SIGNATURES), set(names) - set(N.SIGNATURES)


def test_abi_version_and_status_strings():
    assert N.lib().lgm_abi_version() == 1
    assert N.lib().lgm_status_string(0) == b"ok"
    assert N.lib().lgm_status_string(N.ERR_OUT_OF_RANGE) == b"site out of range"


def test_config_defaults_match_reference():
    cfg = N.default_config()
    # parameters.h:285-378 defaults
    assert (cfg.grid_x, cfg.grid_y, cfg.grid_z) == (128, 128, 1)
    assert cfg.electrostatic_cutoff == 50
    assert cfg.work_size == 256 and cfg.opencl_threshold == 256
    assert (cfg.work_x, cfg.work_y, cfg.work_z) == (4, 4, 4)
    assert cfg.electrostatic_prefactor == pytest.approx(0.4114184, rel=1e-6)


def test_create_validates_before_touching_a_device():
    cfg = N.default_config(grid_x=0)
    h = ctypes.c_void_p()
    st = N.lib().lgm_create(ctypes.byref(cfg), 0, ctypes.byref(h))
    assert st == N.ERR_INVALID_ARGUMENT
    assert b"grid" in N.lib().lgm_last_error(None)
    cfg = N.default_config(grid_x=4000)
    assert N.lib().lgm_create(ctypes.byref(cfg), 0, ctypes.byref(h)) == N.ERR_UNSUPPORTED


@pytest.mark.parametrize("dims,ok", [((418, 8, 1), True), ((419, 8, 1), False),
                                     ((8, 836, 1), True), ((8, 837, 1), False),
                                     ((8, 8, 835), True), ((8, 8, 836), False)])
def test_lattice_bound_for_exact_fp32_r2(dims, ok):
    """6 max(2X, Y, Z+1)^2 < 2^22 keeps every intermediate of the expanded r^2
    exact in FP32 (right-image targets reach x' = 2X - 1): the largest lattices
    pass validation (and then report the missing device here), one more site
    along any axis is refused as unsupported."""
    X, Y, Z = dims
    cfg = N.default_config(grid_x=X, grid_y=Y, grid_z=Z)
    h = ctypes.c_void_p()
    st = N.lib().lgm_create(ctypes.byref(cfg), 0, ctypes.byref(h))
    if ok:
        assert st != N.ERR_UNSUPPORTED
        if st == N.OK:
            N.lib().lgm_destroy(h)
    else:
        assert st == N.ERR_UNSUPPORTED


@pytest.mark.parametrize("dims", [(418, 8, 1), (8, 836, 1), (8, 8, 835), (418, 836, 835)])
def test_both_r2_orders_are_exact_at_the_lattice_bound(dims):
    """The plain tile forms r^2 - 1/2 as ((d + tt) + x a) + y b) + z c; the
    skip tile's vote forms it as (tt + x a) + y b + (d + z c).  Emulating the
    FP32 FMAs and adds step by step (each rounded once to FP32) at extreme
    coordinates of the largest accepted lattices -- targets at x' in [-X, 2X)
    for the image terms -- both orders give the exact r^2 - 1/2, so the vote
    sees the plain tile's bits."""
    import itertools
    import numpy as np
    X, Y, Z = dims
    f32 = np.float32

    def fma(a, b, c):  # one rounding, as FFMA: a*b + c is exact in float64 here
        return f32(np.float64(a) * np.float64(b) + np.float64(c))

    def add(a, b):
        return f32(np.float64(a) + np.float64(b))

    sx, sy, sz = {0, X - 1, X // 2}, {0, Y - 1, Y // 2}, {0, Z - 1, Z // 2}
    tx = {-X, -1, 0, X // 2, X - 1, 2 * X - 1}
    for xs, ys, zs, xt, yt, zt in itertools.product(sx, sy, sz, tx, sy, sz):
        a, b, c = f32(-2 * xs), f32(-2 * ys), f32(-2 * zs)
        d = f32(xs * xs + ys * ys + zs * zs - 0.5)
        tt = f32(xt * xt + yt * yt + zt * zt)
        want = (xt - xs) ** 2 + (yt - ys) ** 2 + (zt - zs) ** 2 - 0.5
        plain = fma(zt, c, fma(yt, b, fma(xt, a, add(d, tt))))
        vote = add(fma(yt, b, fma(xt, a, tt)), fma(zt, c, d))
        assert float(plain) == want and float(vote) == want, (xs, ys, zs, xt, yt, zt)


def test_create_without_gpu_reports_no_device():
    from tests.conftest import HAS_GPU
    if HAS_GPU:
        pytest.skip("a GPU is present")
    cfg = N.default_config()
    h = ctypes.c_void_p()
    st = N.lib().lgm_create(ctypes.byref(cfg), 0, ctypes.byref(h))
    assert st == N.ERR_NO_DEVICE
    assert not h.value


def test_null_context_is_rejected():
    assert N.lib().lgm_destroy(None) == N.OK
    assert N.lib().lgm_sync(None, None) == N.ERR_INVALID_ARGUMENT


def test_variant_table():
    n = N.lib().lgm_variant_count()
    assert n >= 4
    import ctypes as C
    a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
    for v in range(n):
        assert N.lib().lgm_variant_info(v, C.byref(a), C.byref(b), C.byref(c)) == N.OK
        assert a.value % 32 == 0 and b.value >= 1 and 128 % c.value == 0
    assert N.lib().lgm_variant_info(n, None, None, None) == N.ERR_INVALID_ARGUMENT
    f = C.c_int32()
    flags = []
    for v in range(n):
        assert N.lib().lgm_variant_flags(v, C.byref(f)) == N.OK
        flags.append(f.value)
    assert 0 in flags and 1 in flags  # plain and warp-skip tiles both present
    assert N.lib().lgm_variant_flags(n, C.byref(f)) == N.ERR_INVALID_ARGUMENT


def test_out_array_checks():
    """The Python wrapper's result arrays: a caller's float64 array of the
    right length is used as it is; anything else is refused before any call."""
    import numpy as np
    from langmuir_b200.coulomb import _out
    a = np.zeros(5)
    assert _out(a, 5) is a
    assert _out(None, 3).shape == (3,)
    for bad in (np.zeros(4), np.zeros(5, np.float32), np.zeros(10)[::2], [0.0] * 5):
        with pytest.raises(ValueError):
            _out(bad, 5)
