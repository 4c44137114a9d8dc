"""The allocation-free kernel-2 entry (lgm_coulomb_kernel2_noalloc).

Callers that cannot allocate device memory -- engines that fix their device
memory at start-up, plugins whose memory belongs to the host application --
use this entry with their own buffers; its working memory is a fixed array
inside the library.  This test calls it through the C ABI, twice in a row (the
second call smaller than the first, so stale contents of the shared array
would show), and checks each result against the existing kernel-2 entry within
the parity tolerance of the suite: |V_new - V_existing| <= 1e-6 * N, with N
the same sum taken over |q|.  It must pass alone in a fresh process and after
the rest of the suite.

The other cases cover what a caller can meet: targets that are electrode
(drain) ids beyond the lattice, a call of the full capacity, a call on a
non-default stream, a call with no sources, and the range checks of sources
and targets, which return LGM_ERR_OUT_OF_RANGE as the existing entry does.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL32 = 1e-6


def packed_kernel2_case(X, Y, Z, ne, nh, seed):
    """Carriers at distinct random sites, then one nearest-neighbour proposal
    each, packed as the reference's launchCoulombKernel2 packs them."""
    rng = np.random.default_rng(seed)
    vol = X * Y * Z
    sites = rng.choice(vol, ne + nh, replace=False).astype(np.int64)
    q = np.concatenate([-np.ones(ne), np.ones(nh)]).astype(np.int32)
    xyz = np.stack([sites % X, (sites // X) % Y, sites // (X * Y)], 1)
    axis = rng.integers(0, 3, len(sites))
    step = rng.choice([-1, 1], len(sites))
    fut = xyz.copy()
    fut[np.arange(len(sites)), axis] += step
    dims = np.array([X, Y, Z])
    off = (fut < 0) | (fut >= dims)
    fut[off] = xyz[off] - (fut[off] - xyz[off])
    fsites = fut[:, 0] + X * (fut[:, 1] + Y * fut[:, 2])
    s = np.concatenate([sites, fsites]).astype(np.int32)
    return s, np.concatenate([q, q]).astype(np.int32), ne + nh


def test_noalloc_entry_matches_existing_entry_on_two_calls():
    import torch
    import langmuir_b200 as L
    from langmuir_b200 import _native as N

    X, Y, Z, cutoff = 128, 96, 16, 50
    lib = N.lib()
    dev = torch.device("cuda", 0)
    with L.Coulomb(X, Y, Z, cutoff=cutoff) as ctx:
        prefactor = ctx.prefactor
        for ne, nh, seed in [(4000, 3800, 1), (1500, 900, 2)]:
            s, q, n = packed_kernel2_case(X, Y, Z, ne, nh, seed)
            want = ctx.kernel2(s, q, n)                  # the existing entry
            norm = ctx.kernel2(s, np.abs(q), n)
            d_s = torch.from_numpy(s).to(dev)
            d_q = torch.from_numpy(q).to(dev)
            d_o = torch.full((len(s),), float("nan"), dtype=torch.float64, device=dev)
            torch.cuda.synchronize(dev)
            st = lib.lgm_coulomb_kernel2_noalloc(X, Y, Z, cutoff, prefactor, d_s.data_ptr(),
                                                 d_q.data_ptr(), n, len(s), d_o.data_ptr(), None)
            assert st == N.OK, lib.lgm_status_string(st)
            got = d_o.cpu().numpy()
            err = np.abs(got - want)
            assert np.all(err <= TOL32 * norm + 1e-13), float((err / norm).max())


def _call(lib, N, X, Y, Z, cutoff, prefactor, s, q, n, stream=None):
    """One call of the allocation-free entry on device copies of s and q."""
    import torch
    dev = torch.device("cuda", 0)
    d_s = torch.from_numpy(np.ascontiguousarray(s, np.int32)).to(dev)
    d_q = torch.from_numpy(np.ascontiguousarray(q, np.int32)).to(dev)
    d_o = torch.full((max(len(s), 1),), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    st = lib.lgm_coulomb_kernel2_noalloc(X, Y, Z, cutoff, prefactor, d_s.data_ptr(),
                                         d_q.data_ptr(), n, len(s), d_o.data_ptr(),
                                         None if stream is None else stream.cuda_stream)
    return st, d_o[:len(s)].cpu().numpy()


def test_noalloc_entry_with_drain_targets_full_capacity_and_a_side_stream():
    import torch
    import langmuir_b200 as L
    from langmuir_b200 import _native as N
    from oracle import oracle as O

    lib = N.lib()
    X, Y, Z, cutoff = 256, 256, 16, 50
    vol = X * Y * Z
    rng = np.random.default_rng(7)
    with L.Coulomb(X, Y, Z, cutoff=cutoff) as ctx:
        pref = ctx.prefactor
        # drain ids as targets (carriers proposing to leave through an electrode)
        s, q, n = packed_kernel2_case(64, 48, 8, 700, 650, 3)
        s[n + np.arange(0, n, 17)] = 64 * 48 * 8 + rng.integers(0, 35, len(range(0, n, 17)))
        with L.Coulomb(64, 48, 8, cutoff=cutoff) as small:
            want = small.kernel2(s, q, n)
            st, got = _call(lib, N, 64, 48, 8, cutoff, small.prefactor, s, q, n)
        assert st == N.OK, lib.lgm_status_string(st)
        orc = O.Oracle(64, 48, 8, cutoff=cutoff)
        ref = orc.kernel2(s, q, n)
        norm = orc.kernel2(s, np.abs(q), n)
        assert np.all(np.abs(got - want) <= TOL32 * norm + 1e-13)
        assert np.all(np.abs(got - ref) <= TOL32 * norm + 1e-13)

        # the full capacity: 32,768 sources and 65,536 targets
        s, q, n = packed_kernel2_case(X, Y, Z, 16384, 16384, 4)
        assert n == 32768 and len(s) == 65536
        want = ctx.kernel2(s, q, n)
        norm = ctx.kernel2(s, np.abs(q), n)
        st, got = _call(lib, N, X, Y, Z, cutoff, pref, s, q, n)
        assert st == N.OK, lib.lgm_status_string(st)
        assert np.all(np.abs(got - want) <= TOL32 * norm + 1e-13)

        # on a non-default stream, after the larger call
        s, q, n = packed_kernel2_case(X, Y, Z, 900, 1100, 5)
        want = ctx.kernel2(s, q, n)
        norm = ctx.kernel2(s, np.abs(q), n)
        side = torch.cuda.Stream()
        st, got = _call(lib, N, X, Y, Z, cutoff, pref, s, q, n, stream=side)
        assert st == N.OK, lib.lgm_status_string(st)
        assert np.all(np.abs(got - want) <= TOL32 * norm + 1e-13)
        assert vol > 0


def test_noalloc_entry_with_no_sources_and_range_errors():
    from langmuir_b200 import _native as N

    lib = N.lib()
    X, Y, Z, cutoff = 40, 30, 6, 20
    vol = X * Y * Z
    t = np.array([0, 5, vol - 1, vol + 34], np.int32)
    # no sources: every potential is zero, drain ids are valid targets
    st, got = _call(lib, N, X, Y, Z, cutoff, 0.41, t, np.zeros(4, np.int32), 0)
    assert st == N.OK and np.all(got == 0.0)
    # no sources and a target beyond the drain ids: the range error, as kernel 2 gives
    bad = t.copy()
    bad[2] = vol + 35
    st, _ = _call(lib, N, X, Y, Z, cutoff, 0.41, bad, np.zeros(4, np.int32), 0)
    assert st == N.ERR_OUT_OF_RANGE
    # a source outside the lattice (a drain id is no source)
    s = np.array([3, vol, 7, 9], np.int32)
    st, _ = _call(lib, N, X, Y, Z, cutoff, 0.41, s, np.array([1, -1, 1, -1], np.int32), 2)
    assert st == N.ERR_OUT_OF_RANGE
    # a negative target
    s = np.array([3, 4, -2, 9], np.int32)
    st, _ = _call(lib, N, X, Y, Z, cutoff, 0.41, s, np.array([1, -1, 1, -1], np.int32), 2)
    assert st == N.ERR_OUT_OF_RANGE
    # the error does not stick: the next good call succeeds
    s = np.array([3, 4, 8, 9], np.int32)
    st, got = _call(lib, N, X, Y, Z, cutoff, 1.0, s, np.array([1, -1, 1, -1], np.int32), 2)
    assert st == N.OK and np.all(np.isfinite(got))


def test_noalloc_entry_rejects_sizes_beyond_its_limits():
    import torch
    from langmuir_b200 import _native as N

    lib = N.lib()
    d = torch.zeros(8, dtype=torch.int32, device="cuda")
    o = torch.zeros(8, dtype=torch.float64, device="cuda")
    # more sources or targets than the fixed array holds: a clear status, no launch
    assert lib.lgm_coulomb_kernel2_noalloc(64, 64, 16, 50, 0.41, d.data_ptr(), d.data_ptr(),
                                           32769, 40000, o.data_ptr(), None) == N.ERR_CAPACITY
    assert lib.lgm_coulomb_kernel2_noalloc(64, 64, 16, 50, 0.41, d.data_ptr(), d.data_ptr(),
                                           10, 65537, o.data_ptr(), None) == N.ERR_CAPACITY
    assert lib.lgm_coulomb_kernel2_noalloc(64, 64, 16, 50, 0.41, d.data_ptr(), d.data_ptr(),
                                           9, 8, o.data_ptr(), None) == N.ERR_INVALID_ARGUMENT
    assert lib.lgm_status_string(N.ERR_CAPACITY) == b"capacity exceeded"
    assert ctypes.sizeof(ctypes.c_int32) == 4
