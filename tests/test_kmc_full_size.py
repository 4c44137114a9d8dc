"""The kMC step against the FP64 oracle at the sizes the measured workloads
use, and the FP64 guard band exercised on purpose (GPU).

The small cases of test_kmc.py rarely reach the guard band: with few charges
the error scale N of a potential is small and almost no decision lies within
guard_band * N of its threshold.  Here:

* the guard band is widened (lgm_params::guard_band) on small cases, so that
  most Metropolis decisions that reach the threshold test are queued and taken
  from FP64 sums; trajectories, outcomes and counters must still equal the
  oracle's bit for bit, and the run must equal the run with the default band;
* the 256x256x16 electron-hole world with images at both electrodes, the
  128x128x64 Gaussian solar cell and the three largest replicas of a batched
  draw are stepped against the oracle's FP64 step, with the default band; the
  large worlds must queue guard decisions (N is large there) and still match.

Parity bar as in test_kmc.py: outcomes, carrier lists and flux counters
bit-exact after every step under the shared Philox stream, |dE_gpu - dE_oracle|
<= 1e-4 (compareCoulomb, chargeagent.cpp:368).
"""
import numpy as np
import pytest

import bench
import langmuir_b200 as L
from oracle.kmc_setup import assert_same_world, independent_world, oracle_for
from tests.test_kmc import CASES, blob_phase, make_params

pytestmark = pytest.mark.gpu


def step_against_oracle(O, g, p, steps, replica=0, phase=None, threads=0):
    """Steps replica g and the oracle from g's initial state; returns
    (metropolis decisions, guard evaluations, worst |dE| difference)."""
    st = g.stats()
    e0, h0 = g.carriers()
    world = independent_world(p, replica)
    assert_same_world(g.world(), world)
    k = oracle_for(O, p, world, e0, h0, st["max_electrons"], st["max_holes"], replica,
                   step=st["step"], phase=phase)
    guard0 = st["guard_evaluations"]
    worst, metropolis = 0.0, 0
    for s in range(steps):
        n0 = sum(len(a) for a in k.carriers())
        out_o, de_o = k.step(threads=threads)
        g.run(1)
        out_g, de_g = g.last_outcomes(n0)
        np.testing.assert_array_equal(out_g, out_o, err_msg=f"outcomes, step {s}")
        e_g, h_g = g.carriers()
        e_o, h_o = k.carriers()
        np.testing.assert_array_equal(e_g, e_o, err_msg=f"electrons, step {s}")
        np.testing.assert_array_equal(h_g, h_o, err_msg=f"holes, step {s}")
        met = (out_o == 1) | (out_o == 2)
        metropolis += int(met.sum())
        if met.any():
            worst = max(worst, float(np.abs(de_g[met] - de_o[met]).max()))
    stg = g.stats()
    np.testing.assert_array_equal(np.array(stg["counters"], np.uint64), k.counters)
    assert worst <= 1e-4, f"max |dE_gpu - dE_oracle| = {worst:.3e}"
    return metropolis, stg["guard_evaluations"] - guard0, worst


@pytest.mark.parametrize("name", ["3d_eh_images_disorder", "gauss_cutoff30",
                                  "solar_3d_gauss_confined", "2d_128_holes_1pct"])
def test_widened_guard_band_takes_decisions_in_fp64(oracle_mod, name):
    keys = dict(CASES[name])
    steps = min(keys.pop("steps"), 60)
    morph = keys.pop("morphology", None)
    runs = []
    for band in (L.GUARD_BAND_MIN, 0.5):
        p = make_params(**keys, guard_band=band)
        with L.KMC(p, device=0) as g:
            phase = None
            if morph is not None:
                phase = blob_phase(p.grid_x, p.grid_y, p.grid_z, morph)
                g.set_morphology(phase)
            metropolis, guard, _ = step_against_oracle(oracle_mod, g, p, steps, phase=phase)
            runs.append((g.carriers(), metropolis, guard))
    (carriers_default, _, _), (carriers_wide, metropolis, guard) = runs
    # a uniform draw reaches the threshold test when it is below the coupling
    # (1/3 for nearest neighbours): a third of the Metropolis decisions
    assert guard > 0.2 * metropolis, (guard, metropolis)
    for a, b in zip(carriers_default, carriers_wide):
        np.testing.assert_array_equal(a, b)


def test_guard_band_below_the_error_bound_is_rejected():
    p = make_params(**{k: v for k, v in CASES["no_coulomb"].items() if k != "steps"})
    p.guard_band = 0.5 * L.GUARD_BAND_MIN
    with pytest.raises(L.LgmError) as e:
        L.KMC(p)
    assert "guard band" in str(e.value)


def test_cfg2_world_steps_match_oracle(oracle_mod):
    """256x256x16, 1% electrons + 1% holes (20,970 carriers), images at both
    electrodes, site disorder 0.05 eV, traps 2% at 0.2 eV, 1 V: the world of
    the measured kMC leg, four steps."""
    w = bench.WORKLOADS[bench.DEFAULT_WORKLOAD]
    p = bench.kmc_params(L, w, seed=2)
    with L.KMC(p, device=0) as g:
        metropolis, guard, worst = step_against_oracle(oracle_mod, g, p, 4)
    assert metropolis > 10000
    assert guard > 0, "the cfg2 world queues decisions in the guard band"


def test_config3_world_steps_match_oracle(oracle_mod):
    """128x128x64 Gaussian solar cell (sigma 1, cutoff 30) on a GRF
    morphology, 1% electrons on acceptor and 1% holes on donor sites,
    confinement, interface generation and recombination: three steps."""
    p = bench.cfg3_params(L, seed=13)
    X, Y, Z = p.grid_x, p.grid_y, p.grid_z
    phase = bench.grf_phase_3d(X, Y, Z, ell=8.0, seed=17)
    rng = np.random.default_rng(19)
    n1 = int(0.01 * X * Y * Z)
    e = rng.choice(np.flatnonzero(phase == 1), n1, replace=False).astype(np.int32)
    h = rng.choice(np.flatnonzero(phase == 0), n1, replace=False).astype(np.int32)
    with L.KMC(p, device=0) as g:
        g.set_morphology(phase)
        g.set_carriers(e, h)
        metropolis, guard, worst = step_against_oracle(oracle_mod, g, p, 3, phase=phase)
    assert metropolis > 5000
    assert guard > 0, "the config-3 world queues decisions in the guard band"


def test_largest_batched_replicas_match_oracle(oracle_mod):
    """The three largest replicas (by charge capacity) of the 512-replica
    batched draw, stepped as one per-phase batch against the oracle."""
    params = bench.batch_params(L, 512, seed=4)
    cap = [(p.grid_x * p.grid_y * p.grid_z) * (p.electron_percentage + p.hole_percentage)
           for p in params]
    pick = sorted(np.argsort(cap)[-3:])
    chosen = [params[i] for i in pick]
    steps = 5
    with L.KMCBatch(chosen, replica0=0, fused_max_charges=0) as b:
        reps = [b.replica(i) for i in range(len(chosen))]
        orcs = []
        for i, r in enumerate(reps):
            st = r.stats()
            e0, h0 = r.carriers()
            assert st["max_electrons"] + st["max_holes"] > 10000
            world = independent_world(chosen[i], i)
            assert_same_world(r.world(), world)
            orcs.append(oracle_for(oracle_mod, chosen[i], world, e0, h0, st["max_electrons"],
                                   st["max_holes"], replica=i))
        for s in range(steps):
            outs = [k.step()[0] for k in orcs]
            b.run(1)
            for r, k, out_o in zip(reps, orcs, outs):
                out_g, _ = r.last_outcomes(len(out_o))
                np.testing.assert_array_equal(out_g, out_o, err_msg=f"outcomes, step {s}")
                e, h = r.carriers()
                e_o, h_o = k.carriers()
                np.testing.assert_array_equal(e, e_o)
                np.testing.assert_array_equal(h, h_o)
        for r, k in zip(reps, orcs):
            np.testing.assert_array_equal(np.array(r.stats()["counters"], np.uint64), k.counters)
