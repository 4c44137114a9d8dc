"""The C++ drop-in for OpenClHelper (include/langmuir_b200_helper.hpp),
compiled against the library and driven like the reference engine drives its
helper."""
import os
import subprocess

import numpy as np
import pytest

from langmuir_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def shim_exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("shim") / "helper_shim_check")
    lib_dir = os.path.dirname(N.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "helper_shim_check.cpp"), "-o", out,
                    "-L", lib_dir, "-llangmuir_b200", f"-Wl,-rpath,{lib_dir}"], check=True)
    return out


def run_shim(exe, X, Y, Z, c, e, ef, h, hf, d, dq, *args):
    lines = [f"{X} {Y} {Z} {c} {len(e)} {len(h)} {len(d)} {dq}"]
    lines += [f"{s} {f}" for s, f in zip(list(e) + list(h), list(ef) + list(hf))]
    lines += [str(s) for s in d]
    p = subprocess.run([exe, *args], input="\n".join(lines) + "\n", capture_output=True,
                       text=True)
    return p.returncode, p.stdout


def test_shim_without_device_reports_okcl_false(shim_exe):
    from tests.conftest import HAS_GPU
    if HAS_GPU:
        pytest.skip("a GPU is present")
    rc, out = run_shim(shim_exe, 8, 8, 2, 5, [1], [2], [3], [4], [], 0)
    assert rc == 0
    assert out.startswith("okCL 0 use 0 status 4")  # LGM_ERR_NO_DEVICE, openCL stays off


@pytest.mark.gpu
def test_shim_kernel2_matches_oracle(shim_exe, oracle_mod):
    X, Y, Z, c = 40, 36, 6, 25
    rng = np.random.default_rng(4)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    sites = rng.choice(X * Y * Z, 330, replace=False)
    e, h, d = sites[:150], sites[150:310], sites[310:]
    ef = [int(rng.choice(orc.neighbors(int(s)))) for s in e]
    hf = [int(rng.choice(orc.neighbors(int(s)))) for s in h]
    rc, out = run_shim(shim_exe, X, Y, Z, c, e, ef, h, hf, d, 1)
    assert rc == 0, out
    rows = out.strip().splitlines()
    assert rows[0] == "okCL 1 use 1 status 0"
    src = np.concatenate([e, h, d]).astype(np.int32)
    q = np.concatenate([-np.ones(150), np.ones(160), np.ones(20)]).astype(np.int32)
    cur = np.concatenate([e, h]).astype(np.int32)
    fut = np.array(ef + hf, dtype=np.int32)
    want1, want2 = orc.potentials(src, q, cur), orc.potentials(src, q, fut)
    n1, n2 = orc.potentials(src, np.abs(q), cur), orc.potentials(src, np.abs(q), fut)
    for i, row in enumerate(rows[1:]):
        oid, p1, p2 = row.split()
        assert int(oid) == i
        assert abs(float(p1) - want1[i]) <= 1e-6 * n1[i] + 1e-13
        assert abs(float(p2) - want2[i]) <= 1e-6 * n2[i] + 1e-13


@pytest.mark.gpu
def test_shim_compare_host_and_device(shim_exe, oracle_mod):
    """compareHostAndDeviceForAllCarriers (openclhelper.cpp:546-558 with
    chargeagent.cpp:298-370): the FP64 side equals the oracle, the GPU side is
    the kernel-2 output, and each carrier's flag is the reference's rule."""
    X, Y, Z, c = 40, 36, 6, 25
    rng = np.random.default_rng(9)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    sites = rng.choice(X * Y * Z, 300, replace=False)
    e, h, d = sites[:140], sites[140:290], sites[290:]
    ef = [int(rng.choice(orc.neighbors(int(s)))) for s in e]
    hf = [int(rng.choice(orc.neighbors(int(s)))) for s in h]
    rc, out = run_shim(shim_exe, X, Y, Z, c, e, ef, h, hf, d, -1, "--compare")
    assert rc == 0, out
    rows = out.strip().splitlines()
    assert rows[0] == "okCL 1 use 1 status 0"
    failed = int(rows[1].split()[1])
    src = np.concatenate([e, h, d]).astype(np.int32)
    q = np.concatenate([-np.ones(140), np.ones(150), -np.ones(10)]).astype(np.int32)
    cur = np.concatenate([e, h]).astype(np.int32)
    fut = np.array(ef + hf, dtype=np.int32)
    pref = N.default_config().electrostatic_prefactor
    self_term = pref * q[:290]
    want1 = orc.potentials(src, q, cur)
    want2 = orc.potentials(src, q, fut) - self_term
    n1, n2 = orc.potentials(src, np.abs(q), cur), orc.potentials(src, np.abs(q), fut)
    vals = np.array([[float(x) for x in r.split()] for r in rows[2:]])
    assert len(vals) == 290 and np.array_equal(vals[:, 0], np.arange(290))
    gpu1, gpu2, cpu1, cpu2, gpu, cpu, flag = vals[:, 1:].T
    np.testing.assert_allclose(cpu1, want1, rtol=0, atol=1e-12 * n1.max())
    np.testing.assert_allclose(cpu2, want2, rtol=0, atol=1e-12 * n2.max())
    assert np.all(np.abs(gpu1 - want1) <= 1e-6 * n1 + 1e-13)
    assert np.all(np.abs(gpu2 - want2) <= 1e-6 * n2 + 1e-13)
    np.testing.assert_allclose(gpu, q[:290] * (gpu2 - gpu1), rtol=1e-15, atol=1e-15)

    def pdiff(a, b):
        with np.errstate(invalid="ignore", divide="ignore"):
            return np.abs(a - b) / (0.5 * (np.abs(b) + np.abs(a))) * 100.0
    rule = ((gpu - cpu) > 1e-4) | (pdiff(gpu1, cpu1) > 1e-4) | (pdiff(gpu2, cpu2) > 1e-4)
    assert np.array_equal(flag.astype(bool), rule)
    assert failed == int(rule.sum())


@pytest.mark.gpu
def test_shim_compare_flags_no_carrier_on_a_cfg2_world_with_fp64_terms(shim_exe, oracle_mod):
    """On a 256x256x16 world with 1% electrons and 1% holes, each with one
    proposed hop, compareHostAndDeviceForAllCarriers under the FP64-table
    accumulation (LGM_PATH_TABLE64) flags no carrier: every potential is within
    the reference's 1e-4 % of the FP64 sums (chargeagent.cpp:364-370).  The
    FP32 rsqrt path, run on the same world for contrast, stays within its
    stated 1e-6 N bound but may flag carriers whose potential nearly cancels."""
    X, Y, Z, c = 256, 256, 16, 50
    rng = np.random.default_rng(21)
    orc = oracle_mod.Oracle(X, Y, Z, cutoff=c)
    n = int(0.01 * X * Y * Z)
    sites = rng.choice(X * Y * Z, 2 * n, replace=False)
    e, h = sites[:n], sites[n:]
    ef = [int(rng.choice(orc.neighbors(int(s)))) for s in e]
    hf = [int(rng.choice(orc.neighbors(int(s)))) for s in h]
    failed = {}
    for path in (2, 0):
        rc, out = run_shim(shim_exe, X, Y, Z, c, e, ef, h, hf, [], 0, "--compare", str(path))
        assert rc == 0, out
        rows = out.strip().splitlines()
        assert rows[0] == "okCL 1 use 1 status 0"
        failed[path] = int(rows[1].split()[1])
        assert len(rows) == 2 + 2 * n
    assert failed[2] == 0
    print("carriers flagged: FP64 table", failed[2], "FP32 rsqrt", failed[0])
