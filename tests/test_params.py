"""Input keys: defaults, the parser's rules and the validation, as the
reference's KeyValueParser / CheckPointer / checkSimulationParameters."""
import glob
import os

import pytest

import langmuir_b200 as L
from langmuir_b200 import _native as N


def test_struct_matches_library():
    import ctypes
    N.lib()
    assert ctypes.sizeof(L.Params) == N.lib().lgm_params_size()


def test_defaults_are_the_reference_defaults():
    p = L.Params.default()
    # parameters.h:285-378
    assert p.simulation_type == b"transistor"
    assert (p.grid_x, p.grid_y, p.grid_z) == (128, 128, 1)
    assert p.electron_percentage == 0.01 and p.hole_percentage == 0.0
    assert p.trap_potential == 0.1 and p.seed_percentage == 1.0
    assert p.source_rate == 0.9 and p.drain_rate == 0.9 and p.generation_rate == 0.001
    assert p.e_source_l_rate == -1.0 and p.h_drain_r_rate == -1.0
    assert p.work_size == 256 and p.opencl_threshold == 256 and p.hopping_range == 1
    assert p.electrostatic_cutoff == 50 and p.dielectric_constant == 3.5
    assert p.output_stub == b"out" and p.iterations_print == 10 and p.iterations_real == 1000
    assert p.source_scale_area == 65536 and p.max_threads == -1


def test_parse_and_derived_constants():
    text = ("[Parameters]\n"
            "simulation.type    = transistor   # comment\n"
            "GRID.X = 64\n"
            "grid.y = \"32\"\n"
            "grid.z = 4\n"
            "coulomb.carriers = TRUE\n"
            "use.opencl = 1\n"
            "hole.percentage = 0.02\n"
            "electrostatic.cutoff = 30\n"      # constant: ignored (variable.h:269-274)
            "trap.potential =\n"               # empty value: skipped
            "\n"
            "voltage.left = 1.5\n")
    p = L.Params.from_text(text)
    assert (p.grid_x, p.grid_y, p.grid_z) == (64, 32, 4)
    assert p.coulomb_carriers == 1 and p.use_opencl == 1
    assert p.hole_percentage == 0.02 and p.voltage_left == 1.5
    assert p.electrostatic_cutoff == 50 and p.trap_potential == 0.1
    p.check()
    assert p.electrostatic_prefactor == pytest.approx(0.4114184, rel=1e-6)
    assert p.inverse_kt == pytest.approx(38.6817, rel=1e-5)


def test_end_line_and_unterminated_last_line():
    p = L.Params.from_text("[Parameters]\ngrid.x = 10\nend\ngrid.y = 11\n")
    assert p.grid_x == 10 and p.grid_y == 128
    # a last line without '\n' is not read (std::getline at EOF, checkpointer.cpp:408-414)
    p = L.Params.from_text("[Parameters]\ngrid.x = 12\ngrid.y = 13")
    assert p.grid_x == 12 and p.grid_y == 128


@pytest.mark.parametrize("line,needle", [
    ("grid.x 12", "missing equal sign"),
    ("grid.x = 1 = 2", "missing equal sign"),
    (" = 5", "key is empty"),
    ("no.such.key = 1", "invalid key"),
    ("grid.x = twelve", "can not convert to int"),
    ("use.opencl = maybe", "can not convert to bool"),
    ("current.step = -3", "unsigned"),
])
def test_parse_errors(line, needle):
    with pytest.raises(L.LgmError) as e:
        L.Params.from_text(f"[Parameters]\n{line}\n")
    assert e.value.status == N.ERR_PARSE and needle in str(e.value)


def test_first_section_must_be_parameters():
    with pytest.raises(L.LgmError):
        L.Params.from_text("[Electrons]\n3\n1 2 3\n")


@pytest.mark.parametrize("key,value,needle", [
    ("simulation.type", "diode", "transistor or solarcell"),
    ("iterations.real", "15", "iterations.print"),
    ("electron.percentage", "1.5", "electron.pecentage"),
    ("defects.charge", "1", "defects.charge != 0"),
    ("hopping.range", "3", "hopping.range"),
    ("source.coulomb", "true", "source.metropolis = false"),
    ("recombination.rate", "0.1", "recombination.rate"),
    ("coulomb.gaussian.sigma", "1.0", "not 3D"),
])
def test_validation_messages(key, value, needle):
    p = L.Params.from_text(f"[Parameters]\n{key} = {value}\n")
    with pytest.raises(L.LgmError) as e:
        p.check()
    assert e.value.status == N.ERR_INVALID_ARGUMENT and needle in str(e.value)


def test_reference_example_inputs_parse():
    from oracle import oracle as O
    tree = O.reference_tree()
    files = sorted(glob.glob(os.path.join(tree, "examples", "*.inp"))) if tree else []
    if not files:
        pytest.skip("reference examples not present")
    for f in files:
        p = L.Params.from_text(open(f).read())
        p.check()
        assert p.grid_x >= 1
