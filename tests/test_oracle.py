"""The CPU oracle, pinned against the reference's own code and known answers.

Pins: golden fixtures produced by the reference's LangmuirPython grid.py and by
its kernel.cl compiled as C (tests/golden/make_golden.py); the table check of
LangmuirPython/test/test.py:177-201; Philox4x32-10 known-answer vectors;
analytic cases (one charge, cutoff shell, r = 0 skip, the prefactor).
"""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


# ---- Philox (Salmon et al., SC'11) known-answer vectors ------------------------
def test_philox_known_answers(oracle_mod):
    O = oracle_mod
    assert list(O.philox4x32_10([0, 0, 0, 0], [0, 0])) == [
        0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(O.philox4x32_10([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)) == [
        0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert list(O.philox4x32_10([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                                [0xA4093822, 0x299F31D0])) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


# ---- constants -----------------------------------------------------------------
def test_prefactor_and_beta(oracle_mod):
    # parameters.h:386-387 with the defaults of parameters.h:358-362
    assert oracle_mod.electrostatic_prefactor() == pytest.approx(0.411418, rel=1e-5)
    assert oracle_mod.inverse_kt(300.0) == pytest.approx(38.6817, rel=1e-5)


# ---- tables (potential.cpp:246-349; test.py:177-201) ----------------------------
def test_tables_brute_force_3x4x5(oracle_mod):
    orc = oracle_mod.Oracle(3, 4, 5, cutoff=5, hopping_range=1)
    R1, R2, iR = orc.table("R1"), orc.table("R2"), orc.table("iR")
    for dx in range(6):
        for dy in range(6):
            for dz in range(6):
                r2 = dx * dx + dy * dy + dz * dz
                assert R2[dx, dy, dz] == r2
                assert R1[dx, dy, dz] == pytest.approx(np.sqrt(r2), abs=1e-15)
                assert iR[dx, dy, dz] == (0.0 if r2 == 0 else 1.0 / np.sqrt(r2))


@pytest.mark.parametrize("name", ["mesh_3x4x5", "mesh_9x7x4"])
def test_tables_match_reference_mesh(oracle_mod, name):
    g = golden(name)
    nx, ny, nz = (int(v) for v in g["dims"])
    orc = oracle_mod.Oracle(nx, ny, nz, cutoff=max(nx, ny, nz) + 1)
    R2, R1, iR = orc.table("R2"), orc.table("R1"), orc.table("iR")
    np.testing.assert_array_equal(R2[:nx, :ny, :nz], g["r2"])
    np.testing.assert_array_equal(R1[:nx, :ny, :nz], g["r1"])
    np.testing.assert_array_equal(iR[:nx, :ny, :nz], g["ri"])


@pytest.mark.parametrize("name", ["mesh_3x4x5", "mesh_9x7x4"])
def test_sums_match_reference_mesh(oracle_mod, name):
    # PrecalculatedMesh.coulomb: no cutoff, no prefactor, r = 0 contributes 0
    g = golden(name)
    nx, ny, nz = (int(v) for v in g["dims"])
    big = nx + ny + nz + 2
    orc = oracle_mod.Oracle(nx, ny, nz, cutoff=big, prefactor=1.0)
    src = [orc.site(*p) for p in g["src"]]
    q = np.ones(len(src), dtype=np.int32)
    for t, want in zip(g["tgt"], g["v"]):
        got = orc.species_potential(orc.site(*t), src, q)
        assert got == pytest.approx(want, rel=1e-14, abs=1e-14)


def test_self_and_coupling_tables(oracle_mod):
    orc = oracle_mod.Oracle(8, 8, 8, cutoff=10, hopping_range=2, sigma=0.0)
    sI = orc.self_table()
    assert sI[1, 0, 0] == pytest.approx(orc.prefactor)
    assert sI[0, 0, 0] == 0.0
    cpl = orc.coupling_table()
    assert cpl[0, 0, 0] == 0.0
    assert cpl[1, 0, 0] == pytest.approx(1.0 / 3.0)
    assert cpl[2, 0, 0] == pytest.approx((1.0 / 3.0) * 3.0 * (1.0 / 27.0))


# ---- the compiled reference kernels (golden) ------------------------------------
@pytest.mark.parametrize("name", ["k2_point_2d", "k2_point_3d_cut", "k2_gauss_3d",
                                  "k2_gauss_3d_defects"])
def test_kernel2_matches_reference_kernel(oracle_mod, name):
    g = golden(name)
    X, Y, Z = (int(v) for v in g["dims"])
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=int(g["cutoff"]), sigma=float(g["sigma"]),
                            prefactor=float(g["prefactor"]))
    o = orc.kernel2(g["s"], g["q"], int(g["n"]), gauss=float(g["sigma"]) > 0)
    np.testing.assert_allclose(o, g["o"], rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("name", ["k1_point", "k1_gauss"])
def test_kernel1_matches_reference_kernel(oracle_mod, name):
    g = golden(name)
    X, Y, Z = (int(v) for v in g["dims"])
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=int(g["cutoff"]), sigma=float(g["sigma"]),
                            prefactor=float(g["prefactor"]))
    o = orc.kernel1(g["s"], g["q"], gauss=float(g["sigma"]) > 0)
    np.testing.assert_allclose(o, g["o"], rtol=1e-13, atol=1e-13)


def test_kernel2_live_reference_if_built(oracle_mod):
    if oracle_mod.ref_lib() is None:
        pytest.skip("compiled reference kernels not built here")
    rng = np.random.default_rng(5)
    X, Y, Z, c = 14, 11, 7, 6
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    s = rng.choice(X * Y * Z, 70, replace=False).astype(np.int32)
    q = rng.choice([-1, 1, 2], 70).astype(np.int32)
    ref = oracle_mod.ref_kernel2(s, q, 50, c, X, Y, orc.prefactor, work_size=32)
    np.testing.assert_allclose(orc.kernel2(s, q, 50), ref, rtol=1e-13, atol=1e-13)


# ---- species sums and analytic cases ----------------------------------------------
def test_species_sum_equals_kernel2_semantics(oracle_mod):
    rng = np.random.default_rng(3)
    X, Y, Z, c = 20, 16, 6, 8
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    s = rng.choice(X * Y * Z, 60, replace=False).astype(np.int32)
    q = rng.choice([-1, 1], 60).astype(np.int32)
    k2 = orc.kernel2(s, q, 60)
    for g in range(60):
        assert orc.species_potential(int(s[g]), s, q) == pytest.approx(k2[g], rel=1e-13, abs=1e-15)


def test_single_charge_and_cutoff_shell(oracle_mod):
    orc = oracle_mod.Oracle(64, 1, 1, cutoff=10)
    src = [orc.site(20, 0, 0)]
    for d in range(1, 15):
        v = orc.species_potential(orc.site(20 + d, 0, 0), src, [1])
        want = orc.prefactor / d if d < 10 else 0.0  # r = c is excluded
        assert v == pytest.approx(want, rel=1e-15)
    assert orc.species_potential(src[0], src, [1]) == 0.0  # r = 0 skipped


def test_image_distance(oracle_mod):
    orc = oracle_mod.Oracle(30, 5, 5, cutoff=20)
    s_src = [orc.site(3, 2, 2)]
    # left image: dx = x_i + x_j + 1, opposite sign (cubicgrid.cpp:117-120)
    v = orc.species_potential(orc.site(4, 2, 2), s_src, [1], image=True)
    assert v == pytest.approx(-orc.prefactor / 8.0)
    # right image (extension): dx = 2X - 1 - x_i - x_j
    v = orc.species_potential_right_image(orc.site(25, 2, 2), [orc.site(26, 2, 2)], [1])
    assert v == pytest.approx(-orc.prefactor / 8.0)


def test_neighbors_match_reference_order(oracle_mod):
    orc = oracle_mod.Oracle(6, 5, 4, cutoff=5, hopping_range=1)
    s = orc.site(2, 2, 2)
    want = [orc.site(1, 2, 2), orc.site(3, 2, 2), orc.site(2, 1, 2), orc.site(2, 3, 2),
            orc.site(2, 2, 1), orc.site(2, 2, 3)]
    assert list(orc.neighbors(s, 1)) == want
    assert len(orc.neighbors(orc.site(0, 0, 0), 1)) == 3
    # range 2 in 3-D (cubicgrid.cpp:308-437) includes the body diagonals
    orc7 = oracle_mod.Oracle(7, 7, 7, cutoff=5, hopping_range=2)
    nb = orc7.neighbors(orc7.site(3, 3, 3), 2)
    assert len(nb) == 32 and len(set(nb.tolist())) == 32
    assert orc7.site(2, 2, 2) in nb and orc7.site(3, 3, 5) in nb
    orc2d = oracle_mod.Oracle(6, 6, 1, cutoff=5, hopping_range=2)
    assert len(orc2d.neighbors(orc2d.site(2, 2, 0), 2)) == 12


def test_coulomb_cpu_equals_gpu_assembly(oracle_mod):
    """coulombCPU (chargeagent.cpp:215-271) equals coulombGPU's assembly
    (chargeagent.cpp:273-296) from kernel-2 potentials."""
    rng = np.random.default_rng(11)
    X, Y, Z, c = 18, 14, 5, 9
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    vol = X * Y * Z
    sites = rng.choice(vol, 50, replace=False).astype(np.int32)
    e, h = sites[:20], sites[20:45]
    d = sites[45:]
    # an electron and a hole sharing a site exercises bindingPotential
    h = h.copy(); h[0] = e[0]
    ef = np.array([orc.neighbors(int(s))[rng.integers(3)] for s in e], dtype=np.int32)
    hf = np.array([orc.neighbors(int(s))[rng.integers(3)] for s in h], dtype=np.int32)
    de, p1, p2 = orc.coulomb_cpu(e, ef, h, hf, d, defects_charge=1, exciton_binding=0.1,
                                 want_potentials=True)
    s_all = np.concatenate([e, h, d, ef, hf]).astype(np.int32)
    q_all = np.concatenate([-np.ones(20), np.ones(25), np.ones(5), -np.ones(20),
                            np.ones(25)]).astype(np.int32)
    o = orc.kernel2(s_all, q_all, 50)
    sI = orc.self_table()[1, 0, 0]
    etype = np.zeros(vol + 35, np.uint8); etype[e] = oracle_mod.ELECTRON
    htype = np.zeros(vol + 35, np.uint8); htype[h] = oracle_mod.HOLE
    for i in range(45):
        q = -1 if i < 20 else 1
        site = (e if i < 20 else h)[i if i < 20 else i - 20]
        fs = (ef if i < 20 else hf)[i if i < 20 else i - 20]

        def bind(st):
            if q < 0:
                return sI + 0.1 if htype[st] == oracle_mod.HOLE else 0.0
            return sI - 0.1 if etype[st] == oracle_mod.ELECTRON else 0.0
        a = o[i] + bind(site)
        b = o[i + 50] - sI * q + bind(fs)
        assert de[i] == pytest.approx(q * (b - a), rel=1e-12, abs=1e-13)
