"""The figures the bench derives its roofline from, checked on the CPU.

``pairs_in_cutoff`` counts the (target, source, term) pairs with
0 < r^2 < cutoff^2, the pairs that contribute (the 3 FLOP per pair of the
roofline's basis beyond the 8 of every pair tested); ``make_inputs`` draws the
kernel-2 packing of a workload (current sites, then one nearest-neighbour
proposal per carrier, reflected at the faces).
"""
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _brute_pairs(w, tgt, src, terms):
    X, Y = w["X"], w["Y"]
    c2 = w["cutoff"] ** 2

    def xyz(s):
        s = np.asarray(s, np.int64)
        return s % X, (s // X) % Y, s // (X * Y)
    xs, ys, zs = xyz(src)
    total = 0
    xg, yg, zg = xyz(tgt)
    for xt, yt, zt in zip(xg.tolist(), yg.tolist(), zg.tolist()):
        dyz = (yt - ys) ** 2 + (zt - zs) ** 2
        for bit, dx in ((1, xt - xs), (2, xt + xs + 1), (4, 2 * X - 1 - xt - xs)):
            if terms & bit:
                r2 = dx * dx + dyz
                total += int(((r2 > 0) & (r2 < c2)).sum())
    return total


def test_pairs_in_cutoff_matches_a_direct_count():
    w = dict(X=24, Y=20, Z=6, cutoff=9, e=0.02, h=0.02, terms=7, sigma=0.0)
    s_all, q_all, n = bench.make_inputs(w, seed=4)
    for terms in (1, 3, 7):
        got = bench.pairs_in_cutoff(w, s_all, s_all[:n], terms, torch.device("cpu"))
        assert got == _brute_pairs(w, s_all, s_all[:n], terms)


def test_make_inputs_packs_sites_then_neighbour_proposals():
    w = bench.WORKLOADS["cfg3_gauss"]
    s_all, q_all, n = bench.make_inputs(w, seed=1)
    X, Y, Z = w["X"], w["Y"], w["Z"]
    assert len(s_all) == 2 * n and len(q_all) == 2 * n
    assert n == int(w["e"] * X * Y * Z) + int(w["h"] * X * Y * Z)
    cur, fut = s_all[:n].astype(np.int64), s_all[n:].astype(np.int64)
    assert len(np.unique(cur)) == n  # one carrier per site
    assert fut.min() >= 0 and fut.max() < X * Y * Z
    d = np.abs(np.stack([cur % X - fut % X, (cur // X) % Y - (fut // X) % Y,
                         cur // (X * Y) - fut // (X * Y)], 1))
    assert np.all(d.sum(1) == 1)  # nearest neighbours only
    assert np.array_equal(q_all[:n], q_all[n:]) and set(np.unique(q_all)) <= {-1, 1}
