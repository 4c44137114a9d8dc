"""Checkpoints, out.dat / out.coulomb and the LangmuirPython analysis layer,
against the reference's own LangmuirPython test data (tests/golden/
langmuirpython_system0.json, made by make_lp_golden.py)."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "langmuirpython_system0.json")))


def _params(**keys):
    from langmuir_b200 import Params
    p = Params.default()
    for k, v in keys.items():
        p.set(k, v)
    return p


# ---- CPU -------------------------------------------------------------------------------------
def test_read_reference_checkpoint():
    """out.chk of LangmuirPython/test/system.0 (the file test.py:73-88 loads)."""
    from langmuir_b200 import checkpoint
    for part, step in (("part.0", 10), ("part.1", 20)):
        ck = checkpoint.read(GOLD[f"{part}/out.chk"])
        assert ck.electrons.tolist() == list(range(10))
        assert ck.traps.tolist() == list(range(10))
        assert ck.trap_potentials.tolist() == [1.0] * 10
        assert len(ck.holes) == 0 and len(ck.defects) == 0 and len(ck.flux) == 0
        p = ck.params
        assert (p.grid_x, p.grid_y, p.grid_z) == (128, 128, 1)
        assert p.current_step == step and p.iterations_print == 1 and p.voltage_right == 0.0


def test_read_checkpoint_sections_and_errors():
    from langmuir_b200 import checkpoint
    text = ("[FluxState]\n20\n" + "\n".join(str(i) for i in range(20)) + "\n"
            "[RandomState]\n1 2 3 4\n5 6\n[Holes]\n2\n7\n9\n[Defects]\n1\n4\n"
            "[Parameters]\ngrid.x = 16\nend\n[Electrons]\n1\n3\n")
    ck = checkpoint.read(text)
    assert ck.flux.tolist() == list(range(20)) and ck.had_random_state
    assert ck.holes.tolist() == [7, 9] and ck.defects.tolist() == [4]
    assert ck.electrons.tolist() == [3] and ck.params.grid_x == 16
    with pytest.raises(ValueError, match="invalid section"):
        checkpoint.read("[Bogus]\n0\n")
    with pytest.raises(ValueError, match="lists 1 of 2"):
        checkpoint.read("[Holes]\n2\n5\n")


def test_parameters_section_format_and_round_trip():
    """KeyValueParser's checkpoint format: key in 30 columns, '=' in 3 (2
    before a minus sign), doubles with 15 digits, True/False."""
    from langmuir_b200 import Params
    p = _params(grid_x=96, voltage_left=-1.25, voltage_right=7.5, coulomb_carriers=1,
                simulation_type="solarcell", random_seed=123456789012)
    text = p.format()
    lines = text.split("\n")
    assert lines[0] == "[Parameters]" and text.endswith("\n")
    assert "grid.x                        =  96" in lines
    assert "voltage.left                  = -1.250000000000000e+00" in lines
    assert "voltage.right                 =  7.500000000000000e+00" in lines
    assert "coulomb.carriers              =  True" in lines
    assert "simulation.type               =  solarcell" in lines
    assert "random.seed                   =  123456789012" in lines
    # constants and unset extension keys are not written
    assert not any(l.startswith(("electrostatic.prefactor", "inverse.kt", "site.disorder"))
                   for l in lines)
    q = Params.from_text(text)
    for name, _ in Params._fields_:
        a, b = getattr(p, name), getattr(q, name)
        if isinstance(a, float):
            assert a == pytest.approx(b, rel=1e-15, abs=0), name
        elif name not in ("electrostatic_prefactor", "inverse_kt"):
            assert a == b, name
    # an extension key is written once set
    p.site_disorder = 0.05
    assert any(l.startswith("site.disorder") for l in p.format().split("\n"))


class _FakeReplica:
    """The accessors checkpoint.write and FluxWriter use, without a GPU."""

    def __init__(self, params):
        self.params = params
        self.counters = list(range(100, 120))

    def stats(self):
        return dict(step=42, electrons=3, holes=2, counters=self.counters, defects=1, traps=2)

    def carriers(self):
        return np.array([5, 1, 9], np.int32), np.array([7, 2], np.int32)

    def world(self):
        return dict(defects=np.array([11], np.int32), traps=np.array([3, 4], np.int32),
                    trap_potentials=np.array([0.1, 0.2]))


def test_write_checkpoint_and_read_back():
    from langmuir_b200 import checkpoint
    fake = _FakeReplica(_params(grid_x=32, grid_y=16, output_chk_trap_potential=1))
    text = checkpoint.write(fake)
    heads = [l for l in text.split("\n") if l.startswith("[")]
    # CheckPointer::save order, no [RandomState]
    assert heads == ["[Electrons]", "[Holes]", "[Defects]", "[Traps]", "[TrapPotentials]",
                     "[FluxState]", "[Parameters]"]
    ck = checkpoint.read(text)
    assert ck.electrons.tolist() == [5, 1, 9] and ck.holes.tolist() == [7, 2]
    assert ck.defects.tolist() == [11] and ck.traps.tolist() == [3, 4]
    assert ck.trap_potentials.tolist() == [0.1, 0.2]
    assert ck.params.current_step == 42 and ck.params.grid_x == 32
    # flux in the reference's agent order: eSL eSR hSL hSR xSource eDL eDR hDL hDR xDrain
    c = fake.counters
    order = [0, 1, 2, 3, 8, 4, 5, 6, 7, 9]
    assert ck.flux.tolist() == sum(([c[2 * a], c[2 * a + 1]] for a in order), [])


def test_flux_writer_header_matches_reference_out_dat(tmp_path):
    """The header row of out.dat written by the reference engine."""
    from langmuir_b200.output import FluxWriter
    fake = _FakeReplica(_params())
    path = str(tmp_path / "out.dat")
    w = FluxWriter(fake, path)
    w.write()
    mine = open(path).read().split("\n")
    ref = GOLD["part.0/out.dat"].split("\n")
    assert mine[0] == ref[0]
    row = mine[1].split()
    assert len(row) == len(ref[1].split()) == 24
    assert row[0] == "42" and row[-3:-1] == ["3", "2"]
    assert all(len(mine[1][i:i + 23]) == 23 for i in range(0, 24 * 23, 23))


def test_load_dat_and_calculate_reference_output(tmp_path):
    """analyze.calculate on the engine's own out.dat (test.py:40-43)."""
    from langmuir_b200 import analysis
    path = tmp_path / "out.dat"
    path.write_text(GOLD["part.0/out.dat"])
    df = analysis.load_dat(str(path))
    assert len(df.columns) == 24 and len(df) == 10
    assert df["simulation:time"].tolist() == list(range(1, 11))
    out = analysis.calculate(df.copy())
    t = df["simulation:time"].astype(float)
    expect = (df["eDrainR:success"] - df["eDrainL:success"]) / t + \
             (df["hDrainL:success"] - df["hDrainR:success"]) / t
    assert np.allclose(out["drain:rate"], expect)
    assert np.allclose(out["drain:current"], expect * analysis.IFACTOR)
    assert (out["carrier:count"] == df["electron:count"] + df["hole:count"]).all()


# ---- GPU -------------------------------------------------------------------------------------
def _transistor(**keys):
    base = dict(simulation_type="transistor", grid_x=32, grid_y=24, grid_z=4, random_seed=9,
                electron_percentage=0.02, hole_percentage=0.02, seed_charges=1.0,
                defect_percentage=0.01, defects_charge=1, trap_percentage=0.03,
                trap_potential=0.1, gaussian_stdev=0.02, seed_percentage=0.5,
                voltage_right=1.0, coulomb_carriers=1, h_source_l_rate=0.3, h_drain_r_rate=0.9,
                iterations_real=1000, iterations_print=10)
    base.update(keys)
    return _params(**base).check()


@pytest.mark.gpu
def test_resume_from_checkpoint_continues_bit_for_bit():
    """A run checkpointed at step 60 and resumed continues exactly as the
    uninterrupted run (counter-based random stream; no generator state)."""
    from langmuir_b200 import KMC, checkpoint
    with KMC(_transistor(), replica=3) as a:
        a.run(60)
        text = checkpoint.write(a, trap_potentials=True)
        ck = checkpoint.read(text)
        ck.params.seed_charges = 0.0  # place exactly the checkpointed carriers
        with KMC(ck.params.check(), replica=3, world=ck.world()) as b:
            sa, sb = a.stats(), b.stats()
            assert sb["step"] == sa["step"] == 60 and sb["counters"] == sa["counters"]
            for x, y in zip(a.carriers(), b.carriers()):
                assert np.array_equal(x, y)
            wa, wb = a.world(), b.world()
            assert np.array_equal(wa["defects"], wb["defects"])
            assert np.array_equal(wa["traps"], wb["traps"])
            assert np.array_equal(wa["site_energy"], wb["site_energy"])
            a.run(80)
            b.run(80)
            assert a.stats()["counters"] == b.stats()["counters"]
            assert a.stats()["guard_evaluations"] - sa["guard_evaluations"] == \
                b.stats()["guard_evaluations"]
            for x, y in zip(a.carriers(), b.carriers()):
                assert np.array_equal(x, y)


@pytest.mark.gpu
def test_checkpointed_world_placement_rules():
    """Listed sites first, the rest drawn (placeDefects, placeElectrons,
    setPotentialTraps); a legacy 4-value transistor [FluxInfo]."""
    from langmuir_b200 import KMC
    p = _transistor(trap_percentage=0.02, gaussian_stdev=0.0)
    V = 32 * 24 * 4
    world = dict(defects=[5, 17], electrons=[40, 41, 42], holes=[40, 99],
                 traps=[200, 201], trap_potentials=[0.3, -0.2], flux=[11, 7, 13, 5])
    with KMC(p, replica=0, world=world) as k:
        s = k.stats()
        e, h = k.carriers()
        w = k.world()
        assert s["defects"] == int(0.01 * V) and w["defects"][:2].tolist() == [5, 17]
        assert e[:3].tolist() == [40, 41, 42] and len(e) == int(0.02 * V)
        assert h[:2].tolist() == [40, 99] and len(h) == int(0.02 * V)
        assert s["traps"] == int(0.02 * V) and w["traps"][:2].tolist() == [200, 201]
        assert w["trap_potentials"][:2].tolist() == [0.3, -0.2]
        assert np.all(w["trap_potentials"][2:] == 0.1)
        c = s["counters"]
        assert (c[0], c[1], c[10], c[11]) == (11, 7, 13, 5) and sum(c) == 36
    from langmuir_b200._native import LgmError
    with pytest.raises(LgmError, match="can not inject"):
        KMC(p, world=dict(defects=[5], electrons=[5]))  # a carrier on a defect
    with pytest.raises(LgmError, match="FluxInfo"):
        KMC(p, world=dict(flux=[1, 2, 3]))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["mesh_3x4x5", "mesh_9x7x4"])
def test_precalculated_mesh_coulomb_matches_reference(name):
    """grid.PrecalculatedMesh.coulomb (LangmuirPython/langmuir/grid.py:505-554)
    golden values, computed by the GPU pair kernel (tolerance 1e-6 of the sum
    of |terms|)."""
    from langmuir_b200.analysis import PrecalculatedMesh
    d = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    src, tgt = d["src"], d["tgt"]
    with PrecalculatedMesh(*d["dims"]) as mesh:
        v = mesh.coulomb(src[:, 0], src[:, 1], src[:, 2], tgt[:, 0], tgt[:, 1], tgt[:, 2], q=-1)
    norm = np.sum(d["ri"]) + 1.0
    assert np.all(np.abs(v - (-d["v"])) <= 1e-6 * norm)


@pytest.mark.gpu
def test_coulomb_dump_matches_kernel1(tmp_path, oracle_mod):
    """out.coulomb: every site, x slowest, the whole-grid potential of the
    replica's carriers and charged defects (checked against the oracle)."""
    from langmuir_b200 import KMC
    from langmuir_b200.output import coulomb_grid, write_coulomb
    p = _transistor(grid_x=16, grid_y=12, grid_z=3)
    with KMC(p, replica=1) as k:
        k.run(5)
        v = coulomb_grid(k)
        path = str(tmp_path / "out.coulomb")
        write_coulomb(k, path, v)
        e, h = k.carriers()
        d = k.world()["defects"]
    lines = open(path).read().split("\n")
    assert lines[0] == "s x y z v" and len(lines) == 16 * 12 * 3 + 2
    s0 = lines[2].split()
    assert s0[1:4] == ["0", "0", "1"] and int(s0[0]) == 16 * 12
    src = np.concatenate([e, h, d]).astype(np.int32)
    q = np.concatenate([-np.ones(len(e)), np.ones(len(h)), np.ones(len(d))]).astype(np.int32)
    O = oracle_mod.Oracle(16, 12, 3, cutoff=p.electrostatic_cutoff)
    ref = O.kernel1(src, q)
    norm = O.kernel1(src, np.abs(q)).max() + 1e-30
    assert np.all(np.abs(v - ref) <= 1e-6 * max(norm, 1.0))
