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


def run_shim(exe, X, Y, Z, c, e, ef, h, hf, d, dq):
    lines = [f"{X} {Y} {Z} {c} {len(e)} {len(h)} {len(d)} {dq}"]
    lines += [f"{s} {f}" for s, f in zip(list(e) + list(h), list(ef) + list(hf))]
    lines += [str(s) for s in d]
    p = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True)
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
