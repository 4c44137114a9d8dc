"""The kMC step: the oracle's invariants (CPU) and the GPU step against the
oracle, step by step (GPU).

Parity bar: carrier lists (occupancies, list order), per-carrier outcomes and
the sixteen flux counters are bit-exact after every step under the shared
Philox stream; Coulomb energy changes agree to the reference's own
compareCoulomb threshold (|dE_gpu - dE_cpu| <= 1e-4, chargeagent.cpp:368).
Decisions whose FP32 energy lies inside the guard band of the threshold are
redone in FP64 on the GPU; the tests report how many.
"""
import numpy as np
import pytest

import langmuir_b200 as L
from langmuir_b200 import _native as N
from oracle import refkmc
from oracle.kmc_setup import (assert_same_world, independent_world, interface_bonds,  # noqa: F401
                              oracle_for, rates)


def make_params(**keys):
    base = dict(simulation_type="transistor", random_seed=7, seed_charges=1.0,
                coulomb_carriers=1, iterations_real=1000, iterations_print=10)
    base.update(keys)
    p = L.Params.default()
    for k, v in base.items():
        p.set(k, v)
    return p


def blob_phase(X, Y, Z, seed):
    """A seeded two-phase morphology: smoothed noise thresholded at its median."""
    rng = np.random.default_rng(seed)
    f = rng.normal(size=(Z, Y, X))
    for _ in range(3):
        for ax in range(3):
            if f.shape[ax] > 1:
                f = (f + np.roll(f, 1, ax) + np.roll(f, -1, ax)) / 3
    return (f > np.median(f)).astype(np.uint8).reshape(-1)


# ---- CPU: the oracle step's invariants ------------------------------------------------
def test_oracle_step_invariants(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(3)
    X, Y, Z = 20, 16, 3
    V = X * Y * Z
    orc = O.Oracle(X, Y, Z, cutoff=50)
    pot = np.linspace(0, 1, X)[np.arange(V) % X] + rng.normal(0, 0.02, V)
    defects = rng.choice(V, 10, replace=False)
    free = np.setdiff1d(np.arange(V), defects)
    e = rng.choice(free, 30, replace=False)
    h = rng.choice(free, 25, replace=False)
    cfg = O.KmcConfig(inverse_kt=O.inverse_kt(300.0), coulomb_carriers=1, max_electrons=60,
                      max_holes=60, rate_e_source_l=0.9, rate_e_drain_r=0.9, rate_h_source_r=0.5,
                      rate_h_drain_l=0.9, seed=5)
    k = O.KmcOracle(orc, pot, defects, e, h, cfg)
    for _ in range(40):
        outcome, de = k.step(threads=2)
        e_now, h_now = k.carriers()
        assert len(set(e_now)) == len(e_now) and len(set(h_now)) == len(h_now)
        assert not set(e_now) & set(defects) and not set(h_now) & set(defects)
        assert np.all((outcome >= 0) & (outcome <= 4))
    c = k.counters.astype(np.int64)
    # carriers = start + injected - drained
    assert len(k.carriers()[0]) == 30 + c[1] + c[3] - c[9] - c[11]
    assert len(k.carriers()[1]) == 25 + c[5] + c[7] - c[13] - c[15]
    assert c[0] == c[2] == c[4] == c[6] == 40  # one attempt per source per step


def test_oracle_step_is_deterministic(oracle_mod):
    O = oracle_mod
    orc = O.Oracle(16, 16, 2, cutoff=50)
    V = 16 * 16 * 2
    pot = np.zeros(V)
    e = np.arange(0, V, 23)[:15]
    cfg = O.KmcConfig(inverse_kt=38.68, coulomb_carriers=1, max_electrons=40, max_holes=0,
                      rate_e_source_l=0.9, rate_e_drain_r=0.9, seed=11)
    runs = []
    for _ in range(2):
        k = O.KmcOracle(orc, pot, [], e, [], cfg)
        for _ in range(25):
            k.step()
        runs.append(k.carriers()[0])
    np.testing.assert_array_equal(runs[0], runs[1])


# ---- GPU: bit-exact parity of the fused step ------------------------------------------
CASES = {
    "2d_holes_traps": dict(grid_x=48, grid_y=40, grid_z=1, hole_percentage=0.02,
                           electron_percentage=0.0, trap_percentage=0.05, trap_potential=0.1,
                           voltage_left=1.0, e_source_l_rate=0.0, h_source_l_rate=0.5,
                           h_drain_r_rate=0.9, steps=150),
    "3d_eh_images_disorder": dict(grid_x=32, grid_y=28, grid_z=8, electron_percentage=0.02,
                                  hole_percentage=0.02, trap_percentage=0.02,
                                  trap_potential=0.2, site_disorder=0.05, image_charges=3,
                                  voltage_right=1.0, h_source_r_rate=0.5, h_drain_l_rate=0.9,
                                  steps=80),
    "range2_charged_defects": dict(grid_x=24, grid_y=24, grid_z=6, electron_percentage=0.03,
                                   hole_percentage=0.01, defect_percentage=0.02,
                                   defects_charge=1, hopping_range=2, voltage_right=0.5,
                                   h_source_l_rate=0.3, h_drain_r_rate=0.9, steps=80),
    "gauss_cutoff30": dict(grid_x=20, grid_y=20, grid_z=20, electron_percentage=0.01,
                           hole_percentage=0.01, coulomb_gaussian_sigma=1.0,
                           electrostatic_cutoff=30, h_source_l_rate=0.3, h_drain_r_rate=0.9,
                           steps=50),
    "no_coulomb": dict(grid_x=40, grid_y=30, grid_z=2, electron_percentage=0.05,
                       coulomb_carriers=0, voltage_right=2.0, steps=100),
    "solar_2d_recombination": dict(simulation_type="solarcell", grid_x=40, grid_y=40,
                                   grid_z=1, electron_percentage=0.03, hole_percentage=0.03,
                                   seed_charges=0.5, voltage_right=1.0, generation_rate=0.3,
                                   source_scale_area=0, recombination_rate=0.2,
                                   recombination_range=1, steps=120),
    "solar_3d_same_site": dict(simulation_type="solarcell", grid_x=20, grid_y=20, grid_z=6,
                               electron_percentage=0.04, hole_percentage=0.04, seed_charges=0.5,
                               voltage_right=0.5, generation_rate=0.5, source_scale_area=0,
                               recombination_rate=0.5, recombination_range=0, image_charges=1,
                               steps=80),
    "solar_confined_interface": dict(simulation_type="solarcell", grid_x=32, grid_y=24,
                                     grid_z=4, electron_percentage=0.03, hole_percentage=0.03,
                                     seed_charges=0.0, voltage_right=0.5, generation_rate=0.6,
                                     source_scale_area=0, recombination_rate=0.1,
                                     recombination_range=1, morphology_confine=1,
                                     generation_interface=1, steps=120, morphology=3),
    "solar_3d_gauss_confined": dict(simulation_type="solarcell", grid_x=24, grid_y=24,
                                    grid_z=12, electron_percentage=0.02, hole_percentage=0.02,
                                    seed_charges=0.0, coulomb_gaussian_sigma=1.0,
                                    electrostatic_cutoff=30, voltage_right=0.5,
                                    generation_rate=0.8, source_scale_area=0,
                                    recombination_rate=0.05, recombination_range=1,
                                    morphology_confine=1, generation_interface=1, steps=150,
                                    morphology=5),
    "source_metropolis_coulomb": dict(grid_x=32, grid_y=24, grid_z=4, electron_percentage=0.03,
                                      hole_percentage=0.03, defect_percentage=0.02,
                                      defects_charge=1, voltage_right=1.0, e_source_l_rate=0.6,
                                      e_source_r_rate=0.3, h_source_l_rate=0.4,
                                      h_source_r_rate=0.7, e_drain_r_rate=0.9,
                                      h_drain_l_rate=0.9, source_metropolis=1, source_coulomb=1,
                                      steps=80),
    "source_metropolis": dict(grid_x=32, grid_y=24, grid_z=1, electron_percentage=0.03,
                              hole_percentage=0.02, voltage_right=0.5, e_source_l_rate=0.6,
                              h_source_r_rate=0.7, e_drain_r_rate=0.9, h_drain_l_rate=0.9,
                              source_metropolis=1, steps=80),
    "solar_balance_charges": dict(simulation_type="solarcell", grid_x=24, grid_y=24, grid_z=4,
                                  electron_percentage=0.05, hole_percentage=0.05,
                                  seed_charges=0.3, voltage_right=0.5, generation_rate=0.4,
                                  source_scale_area=0, recombination_rate=0.3,
                                  recombination_range=1, balance_charges=1,
                                  e_source_l_rate=0.5, e_source_r_rate=0.5,
                                  h_source_l_rate=0.5, h_source_r_rate=0.5, steps=100),
    "solar_balance_equal_voltages_coulomb": dict(
        simulation_type="solarcell", grid_x=24, grid_y=24, grid_z=4, electron_percentage=0.05,
        hole_percentage=0.05, seed_charges=0.3, voltage_right=0.0, generation_rate=0.4,
        source_scale_area=0, recombination_rate=0.3, recombination_range=1, balance_charges=1,
        e_source_l_rate=0.5, e_source_r_rate=0.5, h_source_l_rate=0.5, h_source_r_rate=0.5,
        source_metropolis=1, source_coulomb=1, steps=100),
    "2d_128_holes_1pct": dict(grid_x=128, grid_y=128, grid_z=1, hole_percentage=0.01,
                              electron_percentage=0.0, trap_percentage=0.05,
                              trap_potential=0.1, voltage_left=1.0, e_source_l_rate=0.0,
                              h_source_l_rate=0.9, h_drain_r_rate=0.9, steps=200),
}


def run_parity(O, name, keys, replica=0):
    keys = dict(keys)
    steps = keys.pop("steps")
    morph = keys.pop("morphology", None)
    p = make_params(**keys)
    with L.KMC(p, device=0, replica=replica) as g:
        phase = None
        if morph is not None:
            phase = blob_phase(p.grid_x, p.grid_y, p.grid_z, morph)
            g.set_morphology(phase)
        st = g.stats()
        e0, h0 = g.carriers()
        world = independent_world(p, replica)
        assert_same_world(g.world(), world)
        np.testing.assert_array_equal(e0, world["electrons"])
        np.testing.assert_array_equal(h0, world["holes"])
        k = oracle_for(O, p, world, e0, h0, st["max_electrons"], st["max_holes"], replica,
                       phase=phase)
        worst = 0.0
        for s in range(steps):
            n0 = len(k.carriers()[0]) + len(k.carriers()[1])
            out_o, de_o = k.step()
            g.run(1)
            out_g, de_g = g.last_outcomes(n0)
            np.testing.assert_array_equal(out_g, out_o, err_msg=f"{name}: outcomes, step {s}")
            e_g, h_g = g.carriers()
            e_o, h_o = k.carriers()
            np.testing.assert_array_equal(e_g, e_o, err_msg=f"{name}: electrons, step {s}")
            np.testing.assert_array_equal(h_g, h_o, err_msg=f"{name}: holes, step {s}")
            met = (out_o == 1) | (out_o == 2)  # dE enters only Metropolis decisions
            if met.any():
                worst = max(worst, float(np.abs(de_g[met] - de_o[met]).max()))
        stg = g.stats()
        np.testing.assert_array_equal(np.array(stg["counters"], np.uint64), k.counters)
        assert stg["step"] == steps
        assert worst <= 1e-4, f"{name}: max |dE_gpu - dE_oracle| = {worst:.3e}"
        return stg, worst


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_gpu_step_matches_oracle(oracle_mod, name):
    stg, worst = run_parity(oracle_mod, name, CASES[name])
    assert stg["proposals"] > 0


@pytest.mark.gpu
def test_gpu_step_replicas_differ_and_repeat(oracle_mod):
    keys = dict(CASES["no_coulomb"])
    keys.pop("steps")
    p = make_params(**keys)
    out = []
    for rep in (0, 1, 0):
        with L.KMC(p, replica=rep) as g:
            g.run(30)
            out.append(g.carriers()[0])
    np.testing.assert_array_equal(out[0], out[2])
    assert not np.array_equal(out[0], out[1])


@pytest.mark.gpu
def test_gpu_set_carriers_and_errors():
    p = make_params(**{k: v for k, v in CASES["no_coulomb"].items() if k != "steps"})
    with L.KMC(p) as g:
        e, h = g.carriers()
        g.set_carriers(e[:5], h)
        assert len(g.carriers()[0]) == 5
        with pytest.raises(L.LgmError):
            g.set_carriers([1, 1], [])  # two electrons on one site
    bad = make_params(grid_x=8, grid_y=8, grid_z=1, electron_percentage=0.0,
                      hole_percentage=0.0)
    with pytest.raises(L.LgmError) as e:
        L.KMC(bad)
    assert "zero rate" in str(e.value) or "maxElectronAgents" in str(e.value)


# ---- GPU: batched replicas reproduce single-replica runs ---------------------------------
def uneven_params(n, seed=1):
    """Replicas of uneven size, occupancy, voltage and traps (as the batched
    configuration draws them)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        xy = int(rng.choice([16, 24, 32, 48]))
        z = int(rng.choice([1, 2, 4]))
        occ = float(rng.uniform(0.005, 0.03))
        out.append(make_params(grid_x=xy, grid_y=xy, grid_z=z, electron_percentage=occ,
                               hole_percentage=occ / 2, voltage_right=float(rng.uniform(0.1, 2.0)),
                               trap_percentage=float(rng.uniform(0.0, 0.1)),
                               trap_potential=float(rng.uniform(0.05, 0.3)),
                               h_source_r_rate=0.5, h_drain_l_rate=0.9))
    return out


def _capacities(params):
    out = []
    for p in params:
        with L.KMC(p) as k:
            st = k.stats()
            out.append(st["max_electrons"] + st["max_holes"])
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fused", "per_phase", "mixed"])
def test_batch_matches_single_replicas(form):
    """Both step forms of the batch, alone and together in one graph, give
    every replica the trajectory of a single replica with its id."""
    params = uneven_params(9)
    steps = 40
    caps = _capacities(params)
    bound = {"fused": max(caps), "per_phase": 0, "mixed": int(np.median(caps))}[form]
    with L.KMCBatch(params, replica0=100, fused_max_charges=bound) as b:
        n_fused = b.fused_count
        assert n_fused == sum(c <= bound for c in caps)
        b.run(steps)
        got = [b.replica(i).carriers() for i in range(len(params))]
        stats = [b.replica(i).stats() for i in range(len(params))]
        assert (b.tuning()["items"] > 0) == (n_fused < len(params))
    if form == "mixed":
        assert 0 < n_fused < len(params)
    for i, p in enumerate(params):
        with L.KMC(p, replica=100 + i) as g:
            g.run(steps)
            e, h = g.carriers()
            s = g.stats()
        np.testing.assert_array_equal(got[i][0], e, err_msg=f"replica {i} electrons")
        np.testing.assert_array_equal(got[i][1], h, err_msg=f"replica {i} holes")
        assert stats[i]["counters"] == s["counters"] and stats[i]["step"] == steps


@pytest.mark.gpu
def test_batch_time_pair_leaves_the_run_unchanged():
    """lgm_kmc_batch_time_pair times the per-phase batch's pair sum on its
    own: it refuses before a step has run, returns a positive time after, and
    the replicas then follow the same trajectories as a batch never timed."""
    params = uneven_params(4, seed=3)
    got = []
    for timed in (False, True):
        with L.KMCBatch(params, replica0=30, fused_max_charges=0) as b:
            if timed:
                with pytest.raises(N.LgmError) as e:
                    b.time_pair(3)
                assert e.value.status == N.ERR_STATE
            b.run(10)
            if timed:
                assert b.time_pair(3) > 0.0
            b.run(10)
            got.append([b.replica(i).carriers() for i in range(len(params))])
    for (e0, h0), (e1, h1) in zip(*got):
        np.testing.assert_array_equal(e0, e1)
        np.testing.assert_array_equal(h0, h1)


@pytest.mark.gpu
def test_batch_culled_replicas_match_single_replicas():
    """Per-phase replicas with room for 8 or more source chunks take the
    culled pair sum (one persistent launch over every such replica's work
    items), the smaller ones the work-item kernel, in one batch: each replica
    follows the trajectory of the standalone replica with its id, also after
    the pair sum was timed and counted in between."""
    rng = np.random.default_rng(8)
    params = []
    for i in range(6):
        xy = [48, 64, 96, 128, 128, 112][i]
        z = [1, 1, 2, 2, 1, 2][i]
        occ = float(rng.uniform(0.02, 0.04))
        params.append(make_params(grid_x=xy, grid_y=xy, grid_z=z, electron_percentage=occ,
                                  hole_percentage=occ / 2,
                                  electrostatic_cutoff=[20, 50, 30, 50, 40, 50][i],
                                  voltage_right=float(rng.uniform(0.1, 2.0)),
                                  trap_percentage=0.05, trap_potential=0.1,
                                  h_source_r_rate=0.5, h_drain_l_rate=0.9))
    steps = 24
    with L.KMCBatch(params, replica0=60, fused_max_charges=0) as b:
        assert 0 < b.culled_count < len(params)
        b.run(steps // 2)
        assert b.time_pair(3) > 0.0
        examined = b.count_pairs()
        full = sum(2 * (r.stats()["electrons"] + r.stats()["holes"]) ** 2
                   for r in (b.replica(i) for i in range(len(params))))
        assert 0 < examined < full
        b.run(steps - steps // 2)
        got = [(b.replica(i).carriers(), b.replica(i).stats()) for i in range(len(params))]
    for i, p in enumerate(params):
        with L.KMC(p, replica=60 + i) as g:
            g.run(steps)
            (e, h), s = g.carriers(), g.stats()
        np.testing.assert_array_equal(got[i][0][0], e, err_msg=f"replica {i} electrons")
        np.testing.assert_array_equal(got[i][0][1], h, err_msg=f"replica {i} holes")
        assert got[i][1]["counters"] == s["counters"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["solar_confined_interface", "solar_3d_gauss_confined"])
def test_fused_batch_solar_matches_single_replicas(case):
    """Solar-cell replicas (exciton source, recombination, confinement) with a
    morphology each: the fused step against single replicas."""
    keys = dict(CASES[case])
    steps = keys.pop("steps")
    morph = keys.pop("morphology")
    params = []
    for i in range(4):
        kk = dict(keys, random_seed=20 + i)
        params.append(make_params(**kk))
    phases = [blob_phase(p.grid_x, p.grid_y, p.grid_z, morph + i) for i, p in enumerate(params)]
    with L.KMCBatch(params, replica0=50) as b:
        assert b.fused_count == len(params)
        for i in range(len(params)):
            b.replica(i).set_morphology(phases[i])
        b.run(steps)
        got = [(b.replica(i).carriers(), b.replica(i).stats()) for i in range(len(params))]
    for i, p in enumerate(params):
        with L.KMC(p, replica=50 + i) as g:
            g.set_morphology(phases[i])
            g.run(steps)
            (e, h), s = g.carriers(), g.stats()
        np.testing.assert_array_equal(got[i][0][0], e, err_msg=f"{case} replica {i} electrons")
        np.testing.assert_array_equal(got[i][0][1], h, err_msg=f"{case} replica {i} holes")
        assert got[i][1]["counters"] == s["counters"]
        assert s["counters"][17] > 0  # excitons were generated


@pytest.mark.gpu
@pytest.mark.parametrize("fused", [True, False])
def test_batch_replica_matches_oracle(oracle_mod, fused):
    params = uneven_params(3, seed=5)
    steps = 25
    with L.KMCBatch(params, replica0=7, fused_max_charges=None if fused else 0) as b:
        assert (b.fused_count == 3) == fused
        reps = [b.replica(i) for i in range(3)]
        orcs = []
        for i, r in enumerate(reps):
            st = r.stats()
            e0, h0 = r.carriers()
            world = independent_world(params[i], 7 + i)
            assert_same_world(r.world(), world)
            orcs.append(oracle_for(oracle_mod, params[i], world, e0, h0, st["max_electrons"],
                                   st["max_holes"], replica=7 + i))
        for _ in range(steps):
            for k in orcs:
                k.step()
            b.run(1)
        for r, k in zip(reps, orcs):
            e, h = r.carriers()
            e_o, h_o = k.carriers()
            np.testing.assert_array_equal(e, e_o)
            np.testing.assert_array_equal(h, h_o)
            np.testing.assert_array_equal(np.array(r.stats()["counters"], np.uint64), k.counters)


# ---- GPU: the step against the reference's own compiled code ---------------------------
REFERENCE_CASES = [n for n, k in CASES.items()
                   if not any(k.get(x) for x in ("image_charges", "site_disorder",
                                                  "morphology_confine", "generation_interface"))
                   and "morphology" not in k]


@pytest.mark.gpu
@pytest.mark.skipif(not refkmc.available(), reason="the compiled reference is not built")
@pytest.mark.parametrize("name", REFERENCE_CASES)
def test_gpu_step_matches_the_reference_engine(name):
    """The GPU replica and the reference's World + agents (oracle/_ref,
    compiled from its sources) from the same parameters: the same world, then
    the same outcomes and carrier lists after every step and the same flux
    counters -- no restatement in between."""
    keys = dict(CASES[name])
    steps = keys.pop("steps")
    p = make_params(**keys)
    ref = refkmc.RefKMC(p, 2)
    with L.KMC(p, device=0, replica=2) as g:
        w = ref.world()
        gw = g.world()
        np.testing.assert_array_equal(gw["site_energy"], w["site_energy"])
        np.testing.assert_array_equal(gw["defects"], w["defects"])
        for a, b in zip(g.carriers(), ref.carriers()):
            np.testing.assert_array_equal(a, b)
        for s in range(steps):
            n0 = sum(len(a) for a in ref.carriers())
            out_r, de_r = ref.step()
            g.run(1)
            out_g, de_g = g.last_outcomes(n0)
            np.testing.assert_array_equal(out_g, out_r, err_msg=f"{name}: outcomes, step {s}")
            for a, b in zip(g.carriers(), ref.carriers()):
                np.testing.assert_array_equal(a, b, err_msg=f"{name}: carriers, step {s}")
            met = (out_r == 1) | (out_r == 2)
            if met.any():
                assert np.abs(de_g[met] - de_r[met]).max() <= 1e-4
        np.testing.assert_array_equal(np.array(g.stats()["counters"], np.uint64), ref.counters)
