"""The kMC oracle and the library's world set-up pinned to the reference's own
code (CPU).

oracle/_ref/librefkmc.so is the reference's World, Grid, Potential, Random and
agent classes compiled from its sources (oracle/refshim, make -C oracle ref),
driven by the Philox draws the GPU step and the FP64 oracle use.  Here:

* the world the library builds on the host (lgm_kmc_world_host, the set-up
  every GPU replica starts from) equals World::initialize's bit for bit: site
  energies, defects, traps and their potentials, seeded carriers;
* the FP64 oracle's step equals the reference's step -- ChargeAgent::
  chooseFuture/coulombCPU/decideFuture/completeTick, drains, sources and
  recombination, all compiled reference code -- bit for bit: outcomes,
  carrier lists, flux counters and the Coulomb energy changes;
* Grid::neighborsSite and the coupling table equal the oracle's.

Configurations are the reference's own features (no image charges, site
disorder, confinement or interface generation, which are extensions).
Skipped where the reference tree was not there to compile the checker.
"""
import numpy as np
import pytest

from langmuir_b200.kmc import world_host
from oracle import refkmc
from oracle.kmc_setup import oracle_for
from tests.test_kmc import CASES, make_params

pytestmark = pytest.mark.skipif(not refkmc.available(),
                                reason="the compiled reference (oracle/_ref) is not built")

EXTENSION_KEYS = ("image_charges", "site_disorder", "morphology_confine", "generation_interface")

EXTRA = {
    "grown_traps_gauss_defects_gate": dict(
        grid_x=40, grid_y=36, grid_z=4, electron_percentage=0.02, hole_percentage=0.03,
        trap_percentage=0.1, seed_percentage=0.2, gaussian_stdev=0.05, trap_potential=0.2,
        defect_percentage=0.03, defects_charge=-1, voltage_right=1.5, slope_z=0.1,
        h_source_l_rate=0.3, e_source_r_rate=0.2, h_drain_r_rate=0.9, e_drain_l_rate=0.7,
        steps=60),
    "solar_traps_range2": dict(
        simulation_type="solarcell", grid_x=30, grid_y=30, grid_z=5, electron_percentage=0.04,
        hole_percentage=0.04, seed_charges=0.5, trap_percentage=0.05, seed_percentage=0.5,
        voltage_right=0.5, generation_rate=0.3, source_scale_area=0, recombination_rate=0.2,
        recombination_range=2, hopping_range=2, steps=80),
}


def reference_cases():
    out = {}
    for name, keys in {**CASES, **EXTRA}.items():
        if any(keys.get(k) for k in EXTENSION_KEYS) or "morphology" in keys:
            continue
        out[name] = keys
    return out


@pytest.mark.parametrize("replica", [0, 5])
@pytest.mark.parametrize("name", list({**CASES, **EXTRA}))
def test_host_world_equals_the_reference_world(oracle_mod, name, replica):
    keys = {k: v for k, v in {**CASES, **EXTRA}[name].items() if k not in ("steps", "morphology")}
    keys["site_disorder"] = 0.0  # an extension: the reference has no such key
    p = make_params(**keys)
    ref = refkmc.RefKMC(p, replica)
    w = ref.world()
    e, h = ref.carriers()
    g = world_host(p, replica)
    np.testing.assert_array_equal(g["site_energy"], w["site_energy"])
    np.testing.assert_array_equal(g["site_energy"], w["hole_site_energy"])
    np.testing.assert_array_equal(g["defects"], w["defects"])
    np.testing.assert_array_equal(g["traps"], w["traps"])
    np.testing.assert_array_equal(g["trap_potentials"], w["trap_potentials"])
    np.testing.assert_array_equal(g["electrons"], e)
    np.testing.assert_array_equal(g["holes"], h)
    z = ref.sizes()
    assert (z["max_electrons"], z["max_holes"]) == (
        int(p.electron_percentage * z["volume"]), int(p.hole_percentage * z["volume"]))


@pytest.mark.parametrize("name", list(reference_cases()))
def test_oracle_step_equals_the_reference_step(oracle_mod, name):
    keys = dict(reference_cases()[name])
    steps = keys.pop("steps")
    p = make_params(**keys)
    ref = refkmc.RefKMC(p, 0)
    z = ref.sizes()
    e0, h0 = ref.carriers()
    k = oracle_for(oracle_mod, p, ref.world(), e0, h0, z["max_electrons"], z["max_holes"], 0)
    decisions = 0
    for s in range(steps):
        out_o, de_o = k.step()
        out_r, de_r = ref.step()
        np.testing.assert_array_equal(out_o, out_r, err_msg=f"{name}: outcomes, step {s}")
        for a, b in zip(k.carriers(), ref.carriers()):
            np.testing.assert_array_equal(a, b, err_msg=f"{name}: carriers, step {s}")
        met = (out_r == 1) | (out_r == 2)
        decisions += int(met.sum())
        # the same FP64 sums in the same order: equal to the last bits
        np.testing.assert_array_equal(de_o[met], de_r[met], err_msg=f"{name}: dE, step {s}")
    np.testing.assert_array_equal(k.counters, ref.counters)
    assert decisions > 0


@pytest.mark.parametrize("dims", [(9, 7, 1), (8, 6, 5)])
@pytest.mark.parametrize("hopping", [1, 2])
def test_neighbors_and_coupling_equal_the_reference(oracle_mod, dims, hopping):
    X, Y, Z = dims
    p = make_params(grid_x=X, grid_y=Y, grid_z=Z, electron_percentage=0.05, hole_percentage=0.0,
                    hopping_range=hopping, e_source_l_rate=0.5, e_drain_r_rate=0.5)
    ref = refkmc.RefKMC(p, 0)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=50, hopping_range=hopping)
    V = X * Y * Z
    for site in range(V):
        want = ref.neighbors(site, hopping)
        got = list(orc.neighbors(site, hopping))
        x = site % X
        if x == 0:
            got.append(V + 3)      # the electron grid's left drain
        if x == X - 1:
            got.append(V + 4)      # and its right drain
        np.testing.assert_array_equal(np.asarray(got, np.int32), want, err_msg=f"site {site}")
    np.testing.assert_array_equal(orc.coupling_table().reshape(-1), ref.coupling(hopping))


def test_reference_example_inputs_step_alike(oracle_mod):
    """Every example input of the reference (examples/*.inp, read where the
    reference tree is present) builds the same world in the library and in
    the reference's World::initialize, and the oracle's steps equal the
    reference engine's for a few steps."""
    import glob
    import os
    from oracle import oracle as O
    tree = O.reference_tree()
    files = sorted(glob.glob(os.path.join(tree, "examples", "*.inp"))) if tree else []
    if not files:
        pytest.skip("reference examples not present")
    from langmuir_b200 import Params
    for f in files:
        p = Params.from_text(open(f).read())
        if p.random_seed == 0:  # 0 means the clock to the reference: fix one
            p.random_seed = 1
        p.check()
        ref = refkmc.RefKMC(p, 0)
        g = world_host(p, 0)
        w = ref.world()
        np.testing.assert_array_equal(g["site_energy"], w["site_energy"], err_msg=f)
        z = ref.sizes()
        e0, h0 = ref.carriers()
        np.testing.assert_array_equal(g["electrons"], e0, err_msg=f)
        np.testing.assert_array_equal(g["holes"], h0, err_msg=f)
        k = oracle_for(oracle_mod, p, w, e0, h0, z["max_electrons"], z["max_holes"], 0)
        for s in range(3):
            out_o, _ = k.step()
            out_r, _ = ref.step()
            np.testing.assert_array_equal(out_o, out_r, err_msg=f"{f}: step {s}")
            for a, b in zip(k.carriers(), ref.carriers()):
                np.testing.assert_array_equal(a, b, err_msg=f"{f}: step {s}")
        np.testing.assert_array_equal(k.counters, ref.counters, err_msg=f)
