"""Generate the golden fixtures from the reference's own code.

Run in a container that holds the reference tree (REFERENCE, default
/root/reference); the fixtures it writes are committed, so tests need no
reference tree.  Two sources of truth, both the reference's own code:

1. LangmuirPython/langmuir/grid.py (Python 2 module; imported here under
   Python 3 with stub modules for its ``import langmuir`` / ``StringIO`` and
   ``itertools.izip = zip``; only pure-numpy code of ``Grid`` and
   ``PrecalculatedMesh`` runs).  ``PrecalculatedMesh.coulomb`` sums 1/r over
   charges with no cutoff and no prefactor (grid.py:505-554); its r^2/r/1/r
   tables are the ones test.py:177-201 checks.
2. src/langmuirCore/kernel.cl compiled as C by oracle/Makefile (``make ref``)
   and run with work.size = 256 and work = 4x4x4 as OpenClHelper sets them
   (openclhelper.cpp:266-274, 434-437).

Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import importlib.util
import io
import itertools
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REFERENCE = os.environ.get("REFERENCE", "/root/reference")
sys.path.insert(0, ROOT)


def load_reference_grid_module():
    sys.modules.setdefault("langmuir", types.ModuleType("langmuir"))
    sio = types.ModuleType("StringIO")
    sio.StringIO = io.StringIO
    sys.modules.setdefault("StringIO", sio)
    if not hasattr(itertools, "izip"):
        itertools.izip = zip
    path = os.path.join(REFERENCE, "LangmuirPython", "langmuir", "grid.py")
    spec = importlib.util.spec_from_file_location("reference_grid", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def mesh_case(G, nx, ny, nz, n_src, n_tgt, seed):
    rng = np.random.default_rng(seed)
    grid = G.Grid(nx, ny, nz)
    mesh = G.PrecalculatedMesh(grid)
    src = rng.integers(0, [nx, ny, nz], size=(n_src, 3))
    tgt = rng.integers(0, [nx, ny, nz], size=(n_tgt, 3))
    v = mesh.coulomb(src[:, 0], src[:, 1], src[:, 2], tgt[:, 0], tgt[:, 1], tgt[:, 2], q=1)
    return dict(dims=np.array([nx, ny, nz]), src=src.astype(np.int32), tgt=tgt.astype(np.int32),
                v=np.asarray(v, dtype=np.float64), r2=mesh.r2.astype(np.float64),
                r1=mesh.r1.astype(np.float64), ri=mesh.ri.astype(np.float64))


def kernel_cases():
    from oracle import oracle as O
    O.build(ref=True)
    out = {}
    pref = O.electrostatic_prefactor()
    rng = np.random.default_rng(20261203)
    # kernel 2 packing: n sources (e, h, defects), then future sites of e, h
    for name, (X, Y, Z, cutoff, ne, nh, nd, dq, sigma) in {
        "k2_point_2d": (40, 32, 1, 50, 30, 25, 0, 0, 0.0),
        "k2_point_3d_cut": (24, 20, 12, 9, 60, 50, 10, 1, 0.0),
        "k2_gauss_3d": (20, 18, 10, 30, 40, 40, 0, 0, 1.0),
        "k2_gauss_3d_defects": (16, 16, 8, 7, 30, 20, 6, -1, 1.5),
    }.items():
        vol = X * Y * Z
        sites = rng.choice(vol, ne + nh + nd, replace=False).astype(np.int32)
        q = np.concatenate([-np.ones(ne), np.ones(nh), np.full(nd, dq)]).astype(np.int32)
        orc = O.Oracle(X, Y, Z, cutoff=cutoff, sigma=sigma)
        fut = []
        for s in sites[: ne + nh]:
            nb = orc.neighbors(int(s), 1)
            fut.append(nb[rng.integers(len(nb))])
        # one proposal onto a drain id (volume + k), as the reference packs it
        fut[0] = vol + 1
        n = ne + nh + nd
        s_all = np.concatenate([sites, np.asarray(fut, dtype=np.int32)])
        q_all = np.concatenate([q, q[: ne + nh]]).astype(np.int32)
        o = O.ref_kernel2(s_all, q_all, n, cutoff, X, Y, pref, sigma=sigma, gauss=sigma > 0,
                          work_size=256)
        out[name] = dict(dims=np.array([X, Y, Z]), cutoff=np.array(cutoff), sigma=np.array(sigma),
                         n=np.array(n), s=s_all, q=q_all, o=o, prefactor=np.array(pref))
    for name, (X, Y, Z, cutoff, m, sigma) in {
        "k1_point": (12, 10, 8, 6, 40, 0.0),
        "k1_gauss": (12, 12, 8, 50, 30, 1.0),
    }.items():
        vol = X * Y * Z
        sites = rng.choice(vol, m, replace=False).astype(np.int32)
        q = rng.choice([-1, 1], m).astype(np.int32)
        o = O.ref_kernel1(sites, q, cutoff, (X, Y, Z), pref, sigma=sigma, gauss=sigma > 0)
        out[name] = dict(dims=np.array([X, Y, Z]), cutoff=np.array(cutoff), sigma=np.array(sigma),
                         s=sites, q=q, o=o, prefactor=np.array(pref))
    return out


def main():
    G = load_reference_grid_module()
    cases = {
        "mesh_3x4x5": mesh_case(G, 3, 4, 5, 7, 11, 1),
        "mesh_9x7x4": mesh_case(G, 9, 7, 4, 25, 40, 2),
    }
    cases.update(kernel_cases())
    for name, d in cases.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **d)
        print(name, {k: v.shape for k, v in d.items()})


if __name__ == "__main__":
    main()
