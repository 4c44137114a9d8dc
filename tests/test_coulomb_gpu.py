"""GPU parity of the Coulomb pair sums against the FP64 oracle, through the C ABI.

Tolerance (FP32C path), per target g:
    |V_gpu - V_oracle| <= 1e-6 * N_g,   N_g = prefactor * sum_j |q_j| w(r_gj)
(the condition-aware bound: FP32 terms with FP32 runs of 8 folded into FP64);
FP64 path: 1e-12 relative to N_g.  The reference's own acceptance test
(ChargeAgent::compareCoulomb, chargeagent.cpp:364-370) asks 1e-4 % = 1e-6
relative per site potential.
"""
import os
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL32 = 1e-6
TOL64 = 1e-12


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


@pytest.fixture(scope="module")
def lgm():
    import langmuir_b200
    return langmuir_b200


def norm_of(orc, s, q, n, gauss=False):
    return orc.kernel2(s, np.abs(np.asarray(q)), n, gauss=gauss)


def assert_close(got, want, norm, tol):
    err = np.abs(got - want)
    bound = tol * norm + 1e-13
    bad = np.nonzero(err > bound)[0]
    assert bad.size == 0, (f"{bad.size} targets off; worst idx {bad[np.argmax(err[bad] / bound[bad])]} "
                           f"err {err[bad].max():.3e} norm {norm[bad].min():.3e}")


def packed_case(orc, rng, ne, nh, nd=0, dq=0, drains=0):
    """Reference kernel-2 packing (openclhelper.cpp:380-424)."""
    vol = orc.volume
    sites = rng.choice(vol, ne + nh + nd, replace=False).astype(np.int32)
    q = np.concatenate([-np.ones(ne), np.ones(nh), np.full(nd, dq)]).astype(np.int32)
    fut = []
    for s in sites[: ne + nh]:
        nb = orc.neighbors(int(s), 1)
        fut.append(nb[rng.integers(len(nb))])
    fut = np.asarray(fut, dtype=np.int32)
    if drains:
        fut[rng.choice(len(fut), drains, replace=False)] = vol + rng.integers(0, 35, drains)
    s_all = np.concatenate([sites, fut]).astype(np.int32)
    q_all = np.concatenate([q, q[: ne + nh]]).astype(np.int32)
    return s_all, q_all, ne + nh + nd


# ---- golden fixtures (the reference's kernel.cl compiled as C) ----------------------
@pytest.mark.parametrize("name", ["k2_point_2d", "k2_point_3d_cut", "k2_gauss_3d",
                                  "k2_gauss_3d_defects"])
@pytest.mark.parametrize("precision", [0, 1])
def test_kernel2_golden(lgm, oracle_mod, name, precision):
    g = golden(name)
    X, Y, Z = (int(v) for v in g["dims"])
    sigma = float(g["sigma"])
    kind = lgm.GAUSS if sigma > 0 else lgm.POINT
    with lgm.Coulomb(X, Y, Z, cutoff=int(g["cutoff"]), prefactor=float(g["prefactor"]),
                     sigma=sigma, precision=precision) as c:
        o = c.kernel2(g["s"], g["q"], int(g["n"]), kind)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=int(g["cutoff"]), sigma=sigma,
                            prefactor=float(g["prefactor"]))
    nrm = norm_of(orc, g["s"], g["q"], int(g["n"]), gauss=sigma > 0)
    assert_close(o, g["o"], nrm, TOL32 if precision == 0 else TOL64)


@pytest.mark.parametrize("name", ["k1_point", "k1_gauss"])
def test_kernel1_golden(lgm, oracle_mod, name):
    g = golden(name)
    X, Y, Z = (int(v) for v in g["dims"])
    sigma = float(g["sigma"])
    kind = lgm.GAUSS if sigma > 0 else lgm.POINT
    with lgm.Coulomb(X, Y, Z, cutoff=int(g["cutoff"]), prefactor=float(g["prefactor"]),
                     sigma=sigma) as c:
        o = c.kernel1(g["s"], g["q"], kind)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=int(g["cutoff"]), sigma=sigma,
                            prefactor=float(g["prefactor"]))
    nrm = orc.kernel1(g["s"], np.abs(g["q"]), gauss=sigma > 0)
    assert_close(o, g["o"], nrm, TOL32)


# ---- seeded random cases against the oracle ------------------------------------------
CASES = {
    # name: X, Y, Z, cutoff, ne, nh, nd, dq, sigma, drains
    "2d_small": (64, 48, 1, 50, 150, 0, 0, 0, 0.0, 3),
    "2d_mixed": (128, 128, 1, 50, 82, 81, 0, 0, 0.0, 2),
    "3d_cut": (40, 36, 20, 12, 300, 280, 40, 1, 0.0, 5),
    "3d_gauss": (48, 40, 24, 30, 500, 500, 0, 0, 1.0, 4),
    "3d_gauss_wide": (32, 32, 16, 10, 200, 150, 30, -2, 2.5, 0),
    "ragged": (17, 13, 7, 5, 37, 29, 3, 1, 0.0, 1),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("path", [0, 1])
def test_kernel2_random(lgm, oracle_mod, name, path):
    X, Y, Z, c, ne, nh, nd, dq, sigma, drains = CASES[name]
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c, sigma=sigma)
    s, q, n = packed_case(orc, rng, ne, nh, nd, dq, drains)
    kind = lgm.GAUSS if sigma > 0 else lgm.POINT
    with lgm.Coulomb(X, Y, Z, cutoff=c, sigma=sigma, path=path) as ctx:
        o = ctx.kernel2(s, q, n, kind)
    want = orc.kernel2(s, q, n, gauss=sigma > 0)
    assert_close(o, want, norm_of(orc, s, q, n, sigma > 0), TOL32)


@pytest.mark.parametrize("terms", [3, 5, 7])
def test_image_terms(lgm, oracle_mod, terms):
    X, Y, Z, c = 50, 30, 6, 20
    rng = np.random.default_rng(terms)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    src = rng.choice(X * Y * Z, 120, replace=False).astype(np.int32)
    q = rng.choice([-1, 1], 120).astype(np.int32)
    tgt = rng.choice(X * Y * Z, 90).astype(np.int32)
    with lgm.Coulomb(X, Y, Z, cutoff=c) as ctx:
        o = ctx.potentials(src, q, tgt, lgm.POINT, terms)
    for g, t in enumerate(tgt):
        want = orc.species_potential(int(t), src, q)
        nrm = orc.species_potential(int(t), src, np.abs(q))
        if terms & 2:
            want += orc.species_potential(int(t), src, q, image=True)
            nrm -= orc.species_potential(int(t), src, np.abs(q), image=True)
        if terms & 4:
            want += orc.species_potential_right_image(int(t), src, q)
            nrm -= orc.species_potential_right_image(int(t), src, np.abs(q))
        assert abs(o[g] - want) <= TOL32 * nrm + 1e-13


def test_kernel1_random_3d(lgm, oracle_mod):
    X, Y, Z, c = 30, 28, 10, 15
    rng = np.random.default_rng(7)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    s = rng.choice(X * Y * Z, 400, replace=False).astype(np.int32)
    q = rng.choice([-1, 1], 400).astype(np.int32)
    with lgm.Coulomb(X, Y, Z, cutoff=c) as ctx:
        o = ctx.kernel1(s, q)
    assert_close(o, orc.kernel1(s, q), orc.kernel1(s, np.abs(q)), TOL32)


# ---- edge cases ----------------------------------------------------------------------
def test_empty_inputs(lgm):
    with lgm.Coulomb(16, 16, 4, cutoff=8) as ctx:
        assert ctx.kernel2(np.zeros(0, np.int32), np.zeros(0, np.int32), 0).size == 0
        o = ctx.potentials(np.zeros(0, np.int32), np.zeros(0, np.int32), [5, 6, 7])
        np.testing.assert_array_equal(o, 0.0)
        assert ctx.potentials([3], [1], np.zeros(0, np.int32)).size == 0


def test_colocated_and_shell(lgm, oracle_mod):
    """r = 0 pairs (a charge at its own site, an electron and a hole sharing a
    site) contribute nothing; a charge exactly at r = cutoff is excluded."""
    X, Y, Z, c = 40, 8, 4, 10
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    a = orc.site(5, 3, 1)
    src = np.array([a, a, orc.site(15, 3, 1), orc.site(14, 3, 1), orc.site(6, 3, 1)], np.int32)
    q = np.array([-1, 1, 1, 2, -1], np.int32)
    tgt = np.array([a, orc.site(5, 3, 2), X * Y * Z + 3], np.int32)
    with lgm.Coulomb(X, Y, Z, cutoff=c) as ctx:
        o = ctx.potentials(src, q, tgt)
    for g, t in enumerate(tgt):
        want = orc.species_potential(int(t), src, q)
        assert abs(o[g] - want) <= TOL32 * max(orc.species_potential(int(t), src, np.abs(q)),
                                               1e-12) + 1e-13
    # at site a: r=0 pairs skipped, (15,3,1) at r = 10 = cutoff excluded,
    # (14,3,1) at r = 9 (q=2), (6,3,1) at r = 1 (q=-1)
    assert o[0] == pytest.approx(orc.prefactor * (2 / 9 - 1.0), rel=1e-6)


def test_largest_lattice_with_both_images(lgm, oracle_mod):
    """At the largest accepted lattice (2X = Y = 836) the expanded r^2 of a pair
    at opposite corners, and of right-image targets at x' = 2X - 1 - x, stays
    exact: potentials at the corners match the FP64 oracle to the FP32 bound."""
    X, Y, Z, c = 418, 836, 1, 40
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    rng = np.random.default_rng(17)
    corner = []
    for x0 in (0, X - 12):
        for y0 in (0, Y - 12):
            for _ in range(40):
                corner.append(orc.site(x0 + int(rng.integers(12)), y0 + int(rng.integers(12)), 0))
    src = np.unique(np.array(corner, np.int32))
    q = np.where(rng.random(len(src)) < 0.5, -1, 1).astype(np.int32)
    tgt = src.copy()
    with lgm.Coulomb(X, Y, Z, cutoff=c) as ctx:
        got = ctx.potentials(src, q, tgt, lgm.POINT, 7)
    want = orc.potentials(src, q, tgt, False, 7)
    aq = np.abs(q).astype(np.int32)
    nrm = (orc.potentials(src, aq, tgt, False, 1) - orc.potentials(src, aq, tgt, False, 2)
           - orc.potentials(src, aq, tgt, False, 4))
    assert np.all(np.abs(got - want) <= TOL32 * np.maximum(nrm, 1e-12) + 1e-13)
    assert np.abs(want).max() > 0


def test_full_lattice_of_charges(lgm, oracle_mod):
    X, Y, Z, c = 12, 10, 6, 7
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    s = np.arange(X * Y * Z, dtype=np.int32)
    q = np.where(s % 3 == 0, 1, -1).astype(np.int32)
    with lgm.Coulomb(X, Y, Z, cutoff=c) as ctx:
        o = ctx.kernel2(s, q, len(s))
    assert_close(o, orc.kernel2(s, q, len(s)), norm_of(orc, s, q, len(s)), TOL32)


def test_range_errors(lgm):
    import langmuir_b200._native as N
    with lgm.Coulomb(8, 8, 2, cutoff=5) as ctx:
        with pytest.raises(lgm.LgmError) as e:
            ctx.potentials([8 * 8 * 2], [1], [0])
        assert e.value.status == N.ERR_OUT_OF_RANGE
        with pytest.raises(lgm.LgmError) as e:
            ctx.potentials([0], [1], [8 * 8 * 2 + 35])
        assert e.value.status == N.ERR_OUT_OF_RANGE
        # drain ids volume .. volume+34 are valid targets
        ctx.potentials([0], [1], [8 * 8 * 2 + 34])
        with pytest.raises(lgm.LgmError):
            ctx.kernel2([1, 2], [1, 1], 3)
        # the messages name the role and the index in the caller's array, for
        # separate source and target arrays and for kernel 2's shared one
        with pytest.raises(lgm.LgmError) as e:
            ctx.potentials([0, 5], [1, 1], [0, 8 * 8 * 2 + 35])
        assert "target 1:" in str(e.value)
        with pytest.raises(lgm.LgmError) as e:
            ctx.kernel2(np.array([1, 2, 3, 8 * 8 * 2 + 35], np.int32), np.ones(4, np.int32), 2)
        assert "target 3:" in str(e.value)
        with pytest.raises(lgm.LgmError) as e:  # a drain id is a target, never a source
            ctx.kernel2(np.array([1, 8 * 8 * 2, 3], np.int32), np.ones(3, np.int32), 2)
        assert "source 1:" in str(e.value)
        # the context stays usable, and kernel 2 still sums correctly after the errors
        o = ctx.kernel2(np.array([0, 1, 8 * 8 * 2], np.int32), np.array([1, 1, 1], np.int32), 2)
        assert o[0] == o[1] and o[0] > 0


def test_async_range_error_reported_by_sync(lgm):
    import torch
    import langmuir_b200._native as N
    with lgm.Coulomb(8, 8, 2, cutoff=5) as ctx:
        s = torch.tensor([1, 2, 500], dtype=torch.int32, device="cuda")
        q = torch.tensor([1, -1, 1], dtype=torch.int32, device="cuda")
        o = torch.empty(3, dtype=torch.float64, device="cuda")
        ctx.potentials_async(s.data_ptr(), q.data_ptr(), 3, s.data_ptr(), 3, o.data_ptr(),
                             stream=torch.cuda.current_stream().cuda_stream)
        with pytest.raises(lgm.LgmError) as e:
            ctx.sync(torch.cuda.current_stream().cuda_stream)
        assert e.value.status == N.ERR_OUT_OF_RANGE
        # the context stays usable
        ctx.potentials_async(s.data_ptr(), q.data_ptr(), 2, s.data_ptr(), 2, o.data_ptr(),
                             stream=torch.cuda.current_stream().cuda_stream)
        ctx.sync(torch.cuda.current_stream().cuda_stream)


# ---- OpenClHelper mirror: the coulombGPU assembly equals coulombCPU ---------------------
def test_openclhelper_mirror_matches_coulomb_cpu(lgm, oracle_mod):
    X, Y, Z, c = 64, 64, 4, 50
    rng = np.random.default_rng(21)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    vol = X * Y * Z
    sites = rng.choice(vol, 700, replace=False).astype(np.int32)
    e_site, h_site, d_site = sites[:300], sites[300:680], sites[680:]
    e_f = np.array([rng.choice(orc.neighbors(int(s))) for s in e_site], np.int32)
    h_f = np.array([rng.choice(orc.neighbors(int(s))) for s in h_site], np.int32)

    class World:
        parameters = {"grid.x": X, "grid.y": Y, "grid.z": Z, "electrostatic.cutoff": c,
                      "defects.charge": 1, "use.opencl": True, "coulomb.carriers": True}
        electrons = [lgm.Carrier(s, -1, f) for s, f in zip(e_site, e_f)]
        holes = [lgm.Carrier(s, 1, f) for s, f in zip(h_site, h_f)]
        defect_site_ids = list(d_site)

    w = World()
    helper = lgm.OpenClHelper(w)
    helper.initializeOpenCL(0)
    assert helper.toggleOpenCL(True)
    helper.launchCoulombKernel2()
    de_cpu, p1, p2 = orc.coulomb_cpu(e_site, e_f, h_site, h_f, d_site, defects_charge=1,
                                     want_potentials=True)
    # condition numbers: the same sums with |q| (the per-target error scale)
    s_src = np.concatenate([e_site, h_site, d_site]).astype(np.int32)
    n1 = orc.potentials(s_src, np.ones(len(s_src), np.int32),
                        np.concatenate([e_site, h_site]))
    n2 = orc.potentials(s_src, np.ones(len(s_src), np.int32), np.concatenate([e_f, h_f]))
    sI = orc.self_table()[1, 0, 0]
    e_occ, h_occ = set(e_site.tolist()), set(h_site.tolist())

    def bind(ch, site):  # bindingPotential, chargeagent.cpp:463-481 (exciton.binding 0)
        other = h_occ if ch.charge < 0 else e_occ
        return sI if site in other else 0.0

    for i, ch in enumerate(w.electrons + w.holes):
        # ChargeAgent::coulombGPU (chargeagent.cpp:273-296)
        g1 = helper.getOutputHost(ch.opencl_id) + bind(ch, ch.site)
        g2 = (helper.getOutputHostFuture(ch.opencl_id) - sI * ch.charge
              + bind(ch, ch.future_site))
        de_gpu = ch.charge * (g2 - g1)
        # compareCoulomb thresholds (chargeagent.cpp:364-370): 1e-4 absolute on
        # dE, 1e-4 % on each site potential
        assert abs(de_gpu - de_cpu[i]) <= 1e-4
        assert abs(g1 - p1[i]) <= TOL32 * n1[i] + 1e-13
        assert abs(g2 - p2[i]) <= TOL32 * n2[i] + 1e-13
    # compareHostAndDeviceForAllCarriers: its FP64 side is the oracle's sum, its
    # GPU side the launch's output, its flags the reference's rule
    nfail, rows = helper.compareHostAndDeviceForAllCarriers()
    gpu1, gpu2, cpu1, cpu2, gpu, cpu, flag = (np.array(c) for c in zip(*rows))
    q_src = np.concatenate([-np.ones(300), np.ones(380), np.ones(20)]).astype(np.int32)
    qc = q_src[:680].astype(np.float64)
    pref = helper._ctx.prefactor
    want1 = orc.potentials(s_src, q_src, np.concatenate([e_site, h_site]))
    want2 = orc.potentials(s_src, q_src, np.concatenate([e_f, h_f])) - pref * qc
    np.testing.assert_allclose(cpu1, want1, rtol=0, atol=1e-12 * n1.max())
    np.testing.assert_allclose(cpu2, want2, rtol=0, atol=1e-12 * n2.max())
    ids = [ch.opencl_id for ch in w.electrons + w.holes]
    assert np.array_equal(gpu1, [helper.getOutputHost(i) for i in ids])
    assert np.array_equal(gpu2, [helper.getOutputHostFuture(i) - pref * qc[i] for i in ids])
    with np.errstate(invalid="ignore", divide="ignore"):
        rule = (((gpu - cpu) > 1e-4) | (np.abs(gpu1 - cpu1) / (0.5 * (np.abs(cpu1) + np.abs(gpu1)))
                                        * 100.0 > 1e-4)
                | (np.abs(gpu2 - cpu2) / (0.5 * (np.abs(cpu2) + np.abs(gpu2))) * 100.0 > 1e-4))
    assert np.array_equal(flag.astype(bool), rule) and nfail == int(rule.sum())


# ---- full-size configuration: parity and size-independent properties --------------------
def test_full_size_3d_config_parity_and_symmetry(lgm, oracle_mod):
    """256x256x16, 2% occupancy split e/h (~21k charges): FP32C against the
    FP64 oracle on every target, the sign-flip identity V(-q) = -V(q) bit for
    bit, and FP64 GPU path against the oracle."""
    X, Y, Z, c = 256, 256, 16, 50
    rng = np.random.default_rng(2)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    ne = nh = int(0.01 * X * Y * Z)
    s, q, n = packed_case(orc, rng, ne, nh, drains=10)
    with lgm.Coulomb(X, Y, Z, cutoff=c) as ctx:
        o = ctx.kernel2(s, q, n)
        o_neg = ctx.kernel2(s, -q, n)
    want = orc.kernel2(s, q, n)
    nrm = norm_of(orc, s, q, n)
    assert_close(o, want, nrm, TOL32)
    np.testing.assert_array_equal(o_neg, -o)
    rel = np.abs(o - want) / nrm
    assert rel.max() < 1e-6
    with lgm.Coulomb(X, Y, Z, cutoff=c, precision=1) as ctx:
        o64 = ctx.kernel2(s, q, n)
    assert_close(o64, want, nrm, TOL64)


def test_skip_tile_equals_plain_tile(lgm, oracle_mod):
    """The warp-skip tile (spatially sorted targets, a warp vote per source)
    gives bit for bit the plain tile's potentials: skipped pairs lie outside
    the cutoff and each target keeps its order over the sources."""
    X, Y, Z, c = 128, 96, 8, 20
    rng = np.random.default_rng(12)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    s, q, n = packed_case(orc, rng, 2500, 2300, 0, 0, drains=2)
    with lgm.Coulomb(X, Y, Z, cutoff=c) as ctx:
        vs = ctx.variants()
        plain = next(i for i, v in enumerate(vs) if not v["warp_skip"] and v["threads"] == 128
                     and v["target_pairs"] == 4 and v["run"] == 32)
        skip = next(i for i, v in enumerate(vs) if v["warp_skip"] and not v["culled"]
                    and v["threads"] == 128 and v["target_pairs"] == 4 and v["run"] == 32)
        out = {}
        for v in (plain, skip):
            ctx.set_variant(v)
            out[v] = (ctx.potentials(s[:n], q[:n], s, lgm.POINT, 7), ctx.last_launch()["splits"])
    assert out[plain][1] == out[skip][1]
    np.testing.assert_array_equal(out[plain][0], out[skip][0])


def culled_variants(ctx):
    return [i for i, v in enumerate(ctx.variants()) if v["culled"]]


def terms_norm(orc, src, q, tgt, gauss, terms):
    """N = sum over the direct and image terms of |q| w: the scale of the
    FP32 error of a sum with images."""
    aq = np.abs(np.asarray(q))
    d = orc.potentials(src, aq, tgt, gauss=gauss, terms=1)
    nrm = d.copy()
    for bit in (2, 4):
        if terms & bit:
            nrm += d - orc.potentials(src, aq, tgt, gauss=gauss, terms=1 | bit)
    return nrm


def test_culled_sums_are_deterministic_and_independent_of_source_order(lgm, oracle_mod):
    """The culled variants sort the sources by lattice cell and then by
    (site, index): the source order, and so every sum, is a function of the
    set of sources.  Two calls agree bit for bit, and so do the same sources
    given in another order; images at both electrodes, Gaussian charges and
    the 1/sqrt(k) table path included.  Every variant is within the parity
    bound of the oracle."""
    X, Y, Z, c = 96, 80, 12, 30
    rng = np.random.default_rng(31)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c, sigma=1.0)
    src = rng.choice(X * Y * Z, 3000, replace=False).astype(np.int32)
    q = np.where(rng.random(3000) < 0.5, -1, 1).astype(np.int32)
    tgt = rng.integers(0, X * Y * Z, 5000).astype(np.int32)
    perm = rng.permutation(3000)
    terms = lgm.TERM_DIRECT | lgm.TERM_IMAGE_LEFT | lgm.TERM_IMAGE_RIGHT
    for kind, path in [(lgm.POINT, 0), (lgm.GAUSS, 0), (lgm.POINT, 1), (lgm.POINT, 2),
                       (lgm.GAUSS, 2)]:
        gauss = kind == lgm.GAUSS
        want = orc.potentials(src, q, tgt, gauss=gauss, terms=terms)
        nrm = terms_norm(orc, src, q, tgt, gauss, terms)
        # the FP64-table path adds FP64 terms: held to the FP64 path's bound
        tol = TOL64 if path == lgm.PATH_TABLE64 else TOL32
        with lgm.Coulomb(X, Y, Z, cutoff=c, sigma=1.0, path=path) as ctx:
            for v in culled_variants(ctx):
                ctx.set_variant(v)
                a = ctx.potentials(src, q, tgt, kind, terms)
                b = ctx.potentials(src, q, tgt, kind, terms)
                p = ctx.potentials(src[perm], q[perm], tgt, kind, terms)
                np.testing.assert_array_equal(a, b)
                np.testing.assert_array_equal(a, p)
                assert_close(a, want, nrm, tol)


def test_culled_sums_examine_fewer_pairs(lgm, oracle_mod):
    """On the 256x256x16 electron-hole world with images at both electrodes
    the culled sum examines far fewer pairs than the reference tests, and at
    least every pair inside the cutoff."""
    X, Y, Z, c = 256, 256, 16, 50
    rng = np.random.default_rng(2)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    ne = nh = int(0.01 * X * Y * Z)
    s, q, n = packed_case(orc, rng, ne, nh, drains=10)
    terms = lgm.TERM_DIRECT | lgm.TERM_IMAGE_LEFT | lgm.TERM_IMAGE_RIGHT
    with lgm.Coulomb(X, Y, Z, cutoff=c) as ctx:
        ctx.set_variant(culled_variants(ctx)[0])
        ctx.set_counting(True)
        o = ctx.potentials(s[:n], q[:n], s, lgm.POINT, terms)
        info = ctx.last_launch()
    want = orc.potentials(s[:n], q[:n], s, terms=terms)
    nrm = terms_norm(orc, s[:n], q[:n], s, False, terms)
    assert_close(o, want, nrm, TOL32)
    assert info["pairs_tested"] == 3 * len(s) * n
    assert 0 < info["pairs_examined"] < 0.5 * info["pairs_tested"]


def test_warp_specialised_culled_sums_equal_the_culled_sums(lgm, oracle_mod):
    """A warp-specialised culled variant (producer warp, ring of stages, items
    taken from a counter) adds every target's terms in the order of a culled
    variant with the same tile, FP32 run and chunks per item: the sums are
    equal bit for bit, for every path and kind, with images at both
    electrodes (a group one warp shape skips adds +0 in the other), and with
    the same warp shape so are the pairs examined."""
    X, Y, Z, c = 128, 128, 16, 40
    rng = np.random.default_rng(12)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c, sigma=1.0)
    ne = nh = int(0.008 * X * Y * Z)
    s, q, n = packed_case(orc, rng, ne, nh, drains=6)
    terms = lgm.TERM_DIRECT | lgm.TERM_IMAGE_LEFT | lgm.TERM_IMAGE_RIGHT
    pairs = 0
    for kind, path in [(lgm.POINT, 0), (lgm.GAUSS, 0), (lgm.POINT, 1), (lgm.POINT, 2),
                       (lgm.GAUSS, 2)]:
        with lgm.Coulomb(X, Y, Z, cutoff=c, sigma=1.0, path=path) as ctx:
            vs = ctx.variants()
            shape = lambda v: (vs[v]["threads"] * vs[v]["target_pairs"], vs[v]["run"],
                               vs[v]["chunks_per_item"])
            for w in [i for i, v in enumerate(vs) if v["warp_specialised"]]:
                twins = [i for i, v in enumerate(vs) if v["culled"] and
                         not v["warp_specialised"] and shape(i) == shape(w)]
                for t in twins:
                    got = []
                    for v in (t, w):
                        ctx.set_variant(v)
                        ctx.set_counting(True)
                        got.append((ctx.potentials(s[:n], q[:n], s, kind, terms),
                                    ctx.last_launch()["pairs_examined"]))
                        ctx.set_counting(False)
                    np.testing.assert_array_equal(got[0][0], got[1][0])
                    assert got[0][1] > 0 and got[1][1] > 0
                    if vs[t]["target_pairs"] == vs[w]["target_pairs"]:
                        assert got[0][1] == got[1][1]
                    pairs += 1
    assert pairs >= 10


# ---- every compiled tile variant is exact to the same bound --------------------------
def test_every_variant_and_autotune(lgm, oracle_mod):
    X, Y, Z, c = 96, 80, 12, 30
    rng = np.random.default_rng(99)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    s, q, n = packed_case(orc, rng, 1500, 1400, 100, 1, drains=3)
    want = orc.kernel2(s, q, n)
    nrm = norm_of(orc, s, q, n)
    with lgm.Coulomb(X, Y, Z, cutoff=c) as ctx:
        for v in range(len(ctx.variants())):
            ctx.set_variant(v)
            assert_close(ctx.kernel2(s, q, n), want, nrm, TOL32)
            assert ctx.last_launch()["variant"] == v
        ctx.set_variant(-1)
        best = ctx.autotune(n, len(s))
        assert 0 <= best < len(ctx.variants())
        assert_close(ctx.kernel2(s, q, n), want, nrm, TOL32)
        assert ctx.last_launch()["variant"] == best


def test_probe_peaks_measure_plausible_rates():
    """lgm_probe_peaks: the FP32 FMA rate lies under the derived peak (SMs x
    128 lanes x 2 x the clock attribute) and above a third of it; MUFU rsqrt
    runs at most at 16 per SM per clock."""
    from langmuir_b200 import _native as N
    p = N.probe_peaks(0)
    derived = p["sm_count"] * 128 * 2 * p["clock_mhz_attribute"] * 1e6 / 1e12
    for key in ("ffma_tflops", "ffma2_tflops"):
        assert derived / 3 < p[key] <= derived * 1.02, (key, p[key], derived)
    assert 0 < p["rsqrt_per_s"] <= 16.5 * p["sm_count"] * p["clock_mhz_attribute"] * 1e6


def test_bounded_wait_runs_out_and_the_context_stays_usable(lgm, oracle_mod):
    """Failure detection without a fault: a pipeline stage that no copy fills
    makes the pair kernels' bounded wait run out (a small limit), the device
    error word reports LGM_ERR_TIMEOUT, and a kernel-2 call afterwards on the
    same device is still correct."""
    from langmuir_b200 import _native as N
    assert N.lib().lgm_selftest_timeout(0, 1 << 10) == N.ERR_TIMEOUT
    assert N.lib().lgm_selftest_timeout(0, 0) == N.ERR_INVALID_ARGUMENT
    X, Y, Z, c = 40, 30, 6, 20
    rng = np.random.default_rng(4)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    s, q, n = packed_case(orc, rng, 300, 280, 0, 0)
    with lgm.Coulomb(X, Y, Z, cutoff=c) as ctx:
        assert_close(ctx.kernel2(s, q, n), orc.kernel2(s, q, n), norm_of(orc, s, q, n), TOL32)


def test_out_array_reused(lgm):
    """A caller's result array is filled in place, call after call, with the
    same values as a fresh one; a wrong one is refused before any work."""
    rng = np.random.default_rng(5)
    s = rng.choice(16 * 16 * 4, 60, replace=False).astype(np.int32)
    q = np.where(np.arange(60) % 2 == 0, 1, -1).astype(np.int32)
    out = np.full(60, np.nan)
    with lgm.Coulomb(16, 16, 4, cutoff=10) as ctx:
        want = ctx.potentials(s[:30], q[:30], s)
        for _ in range(2):
            got = ctx.potentials(s[:30], q[:30], s, out=out)
            assert got is out
            np.testing.assert_array_equal(out, want)
        np.testing.assert_array_equal(ctx.kernel2(s, q, 30, out=out), ctx.kernel2(s, q, 30))
        with pytest.raises(ValueError):
            ctx.potentials(s[:30], q[:30], s, out=np.empty(59))


def test_launch_overlap_gives_the_same_bits(lgm, oracle_mod):
    """The call's kernels launched with programmatic dependent launch (the
    default) and in plain stream order give the same bits, call after call:
    every kernel waits for the one ahead before touching memory, and the last
    one clears the bins the next call counts into."""
    X, Y, Z, c = 64, 48, 10, 20
    rng = np.random.default_rng(8)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    s = rng.choice(X * Y * Z, 1800, replace=False).astype(np.int32)
    q = np.where(rng.random(1800) < 0.5, -1, 1).astype(np.int32)
    terms = lgm.TERM_DIRECT | lgm.TERM_IMAGE_LEFT | lgm.TERM_IMAGE_RIGHT
    with lgm.Coulomb(X, Y, Z, cutoff=c) as ctx:
        got = []
        for on in (True, False, True):
            ctx.set_launch_overlap(on)
            got.append(ctx.potentials(s[:900], q[:900], s, lgm.POINT, terms))
            got.append(ctx.potentials(s[:900], q[:900], s, lgm.POINT, terms))
    for g in got[1:]:
        np.testing.assert_array_equal(g, got[0])
    want = orc.potentials(s[:900], q[:900], s, terms=terms)
    assert_close(got[0], want, terms_norm(orc, s[:900], q[:900], s, False, terms), TOL32)
