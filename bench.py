#!/usr/bin/env python
"""Coulomb pair-evaluation throughput of the B200 hot path.

One step = the potentials at the current and proposed sites of every carrier
(the kernel-2 packing of OpenClHelper::launchCoulombKernel2,
openclhelper.cpp:372-457) from all carriers, with the workload's image terms.
Default workload: 256x256x16 lattice, 2% occupancy split 50/50 electrons and
holes (20,970 charges, 41,940 targets), cutoff 50, image charges at both x
electrodes -- seeded synthetic placement.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 (under torchrun): independent replicas, one per GPU (the path does not
shard); value = pairs of all ranks / max over ranks of the timed span.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: lattice, cutoff, occupancy, image terms, sigma
    "cfg2_3d_eh_images": dict(X=256, Y=256, Z=16, cutoff=50, e=0.01, h=0.01, terms=7, sigma=0.0,
                              desc="256x256x16, 2% e/h 50/50, cutoff 50, images at both x "
                                   "electrodes"),
    "cfg1_2d_holes": dict(X=128, Y=128, Z=1, cutoff=50, e=0.0, h=0.01, terms=1, sigma=0.0,
                          desc="128x128x1, 1% holes, cutoff 50, no images"),
    "cfg3_gauss": dict(X=128, Y=128, Z=64, cutoff=30, e=0.01, h=0.01, terms=1, sigma=1.0,
                       desc="128x128x64, 1%+1% e/h, Gaussian sigma 1, cutoff 30"),
}
DEFAULT_WORKLOAD = "cfg2_3d_eh_images"

# The roofline counts the work the skip tiles cannot avoid: r^2 of every pair
# tested (8), and 1/r plus the accumulate (3) for a pair inside the cutoff.
FLOP_PER_TEST = 8
FLOP_PER_CONTRIB = 3
# DRAM bytes per launch of the pair kernel from one ncu capture of this
# workload: dram__bytes_read.sum + dram__bytes_write.sum.
PAIR_KERNEL_DRAM_BYTES = 2034176


def make_inputs(w, seed):
    """Seeded uniform placement and one nearest-neighbour proposal per carrier."""
    rng = np.random.default_rng(seed)
    X, Y, Z = w["X"], w["Y"], w["Z"]
    vol = X * Y * Z
    ne, nh = int(w["e"] * vol), int(w["h"] * vol)
    sites = rng.choice(vol, ne + nh, replace=False).astype(np.int64)
    q = np.concatenate([-np.ones(ne), np.ones(nh)]).astype(np.int32)
    x, y, z = sites % X, (sites // X) % Y, sites // (X * Y)
    coords = np.stack([x, y, z], 1)
    dims = np.array([X, Y, Z])
    axis = rng.integers(0, 3 if Z > 1 else 2, len(sites))
    step = rng.choice([-1, 1], len(sites))
    fut = coords.copy()
    fut[np.arange(len(sites)), axis] += step
    off = (fut < 0) | (fut >= dims)
    fut[off] = coords[off] - (fut[off] - coords[off])  # reflect at the faces
    fsites = fut[:, 0] + X * (fut[:, 1] + Y * fut[:, 2])
    s_all = np.concatenate([sites, fsites]).astype(np.int32)
    q_all = np.concatenate([q, q]).astype(np.int32)
    return s_all, q_all, ne + nh


def job_totals(dist, units, seconds):
    """Whole-job figures of one bench leg run as independent replicas: the
    units every rank processed, summed, and the longest rank's time (max over
    ranks).  Every rank calls this in the same order, leg by leg.  With no
    process group the rank's own figures come back unchanged."""
    if dist is None:
        return float(units), float(seconds)
    import torch
    dev = (torch.device("cuda", torch.cuda.current_device())
           if dist.get_backend() == "nccl" else torch.device("cpu"))
    u = torch.tensor([float(units)], dtype=torch.float64, device=dev)
    s = torch.tensor([float(seconds)], dtype=torch.float64, device=dev)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    dist.all_reduce(s, op=dist.ReduceOp.MAX)
    return float(u.item()), float(s.item())


def pairs_in_cutoff(w, tgt_sites, src_sites, terms, dev):
    """(target, source, term) pairs with 0 < r^2 < cutoff^2 -- the pairs that
    contribute -- counted on the GPU outside any timed region.  Image
    distances along x: x_t + x_s + 1 (left), 2X - 1 - x_t - x_s (right)."""
    import torch
    X, Y = w["X"], w["Y"]
    c2 = w["cutoff"] ** 2

    def xyz(sites):
        s = torch.as_tensor(np.asarray(sites, np.int32), device=dev)
        return s % X, (s // X) % Y, s // (X * Y)
    xs, ys, zs = xyz(src_sites)
    xt, yt, zt = xyz(tgt_sites)
    total = 0
    for t0 in range(0, len(tgt_sites), 2048):
        a, b, c = xt[t0:t0 + 2048, None], yt[t0:t0 + 2048, None], zt[t0:t0 + 2048, None]
        dyz = (b - ys) ** 2 + (c - zs) ** 2
        for bit, dx in ((1, a - xs), (2, a + xs + 1), (4, 2 * X - 1 - a - xs)):
            if terms & bit:
                r2 = dx * dx + dyz
                total += int(((r2 > 0) & (r2 < c2)).sum())
    return total


def accuracy_vs_oracle(w, src, q, tgt, got, terms):
    """FP32 sums against the FP64 oracle (the checker) on a sample of targets:
    max |V32 - V64| / N with N = sum_j |q_j| w(r_j) (the error scale of a
    target's potential), and the error relative to |V|."""
    from oracle import oracle as O
    orc = O.Oracle(w["X"], w["Y"], w["Z"], cutoff=w["cutoff"], sigma=w["sigma"])
    g = w["sigma"] > 0
    want = orc.potentials(src, q, tgt, g, terms)
    aq = np.abs(q).astype(np.int32)
    nrm = orc.potentials(src, aq, tgt, g, 1)
    for t in (2, 4):
        if terms & t:
            nrm -= orc.potentials(src, aq, tgt, g, t)  # image terms carry -|q|
    err = np.abs(np.asarray(got) - want)
    nrm = np.maximum(nrm, 1e-300)  # a target with no charge inside the cutoff has V = N = 0
    return {"targets_checked": len(tgt), "max_err_over_norm": float((err / nrm).max()),
            "max_rel_err": float((err / np.maximum(np.abs(want), 1e-3 * nrm)).max()),
            "tolerance_over_norm": 1e-6}


def grf_phase_3d(X, Y, Z, ell, seed):
    """Binary bulk-heterojunction morphology: white noise blurred by a
    Gaussian of standard deviation ``ell`` sites (in Fourier space, on a
    padded box so the blur does not wrap), thresholded at its median.
    phase[site] 0 donor, 1 acceptor, x fastest."""
    rng = np.random.default_rng(seed)
    pad = int(3 * ell)
    P = (Z + 2 * pad, Y + 2 * pad, X + 2 * pad)
    k2 = sum(np.fft.fftfreq(n)[tuple(slice(None) if a == i else None for a in range(3))] ** 2
             for i, n in enumerate(P))
    f = np.fft.irfftn(np.fft.rfftn(rng.standard_normal(P))
                      * np.exp(-2.0 * np.pi ** 2 * k2[:, :, : P[2] // 2 + 1] * ell ** 2), P)
    f = f[pad:pad + Z, pad:pad + Y, pad:pad + X]
    return (f > np.median(f)).astype(np.uint8).reshape(-1)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            os.remove(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def cpu_baseline_run(w, s_all, q_all, n, seconds, threads):
    """The oracle (C++ FP64 restatement of the reference's CPU Coulomb path) on a
    bounded sample of targets: pairs/s, threads used, sample description."""
    from oracle import oracle as O
    orc = O.Oracle(w["X"], w["Y"], w["Z"], cutoff=w["cutoff"], sigma=w["sigma"])
    src, q = s_all[:n], q_all[:n]
    nterms = bin(w["terms"]).count("1")
    probe = s_all[: min(64, len(s_all))]
    t0 = time.perf_counter()
    orc.potentials(src, q, probe, gauss=w["sigma"] > 0, terms=w["terms"], threads=threads)
    rate = len(probe) * n * nterms / max(time.perf_counter() - t0, 1e-6)
    k = int(np.clip(rate * seconds / (n * nterms), 64, len(s_all)))
    tgt = s_all[:k]
    passes = 0
    t0 = time.perf_counter()
    while True:  # whole passes over the sample until `seconds` of CPU work
        orc.potentials(src, q, tgt, gauss=w["sigma"] > 0, terms=w["terms"], threads=threads)
        passes += 1
        dt = time.perf_counter() - t0
        if dt >= seconds:
            break
    pairs = passes * k * n * nterms
    return pairs / dt, dt, (f"{passes} pass(es) over {k} of {len(s_all)} targets x {n} sources "
                            f"x {nterms} terms")


def reference_arm(args, w, rank):
    """--impl reference: the CPU path on the host cores, rank 0 only."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    s_all, q_all, n = make_inputs(w, seed=2)
    from oracle import oracle as O
    orc = O.Oracle(w["X"], w["Y"], w["Z"], cutoff=w["cutoff"], sigma=w["sigma"])
    nterms = bin(w["terms"]).count("1")
    # each step: a bounded slice of the targets (about 2 s of CPU work)
    probe = s_all[:64]
    t0 = time.perf_counter()
    orc.potentials(s_all[:n], q_all[:n], probe, w["sigma"] > 0, w["terms"], threads)
    rate = 64 * n * nterms / max(time.perf_counter() - t0, 1e-6)
    k = int(np.clip(rate * 2.0 / (n * nterms), 64, len(s_all)))
    times = []
    for i in range(args.warmup + args.steps):
        lo = (i * k) % max(1, len(s_all) - k)
        tgt = s_all[lo:lo + k]
        t0 = time.perf_counter()
        orc.potentials(s_all[:n], q_all[:n], tgt, w["sigma"] > 0, w["terms"], threads)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    pairs = k * n * nterms
    value = pairs * len(times) / sum(times)
    sample = (f"{k} of {len(s_all)} targets per step x {n} sources x {nterms} terms "
              "(C++ FP64 restatement of Potential::coulomb*/coulombImage*, table gathers)")
    line = {
        "impl": "reference", "metric": "Coulomb pair-evals/s", "value": value,
        "unit": "pair-evals/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": args.workload, "desc": w["desc"]},
        "cpu_baseline": {"value": value, "unit": "pair-evals/s", "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "pair-evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def kmc_params(L, w, seed):
    """The workload's lattice and occupancy as a Langmuir transistor run."""
    p = L.Params.default()
    for k, v in dict(grid_x=w["X"], grid_y=w["Y"], grid_z=w["Z"], electron_percentage=w["e"],
                     hole_percentage=w["h"], seed_charges=1.0, coulomb_carriers=1,
                     electrostatic_cutoff=w["cutoff"], coulomb_gaussian_sigma=w["sigma"],
                     trap_percentage=0.02, trap_potential=0.2, site_disorder=0.05,
                     image_charges=(1 if w["terms"] & 2 else 0) | (2 if w["terms"] & 4 else 0),
                     voltage_right=1.0, random_seed=seed).items():
        p.set(k, v)
    if w["e"] == 0:
        p.e_source_l_rate = 0.0
    if w["h"] > 0:
        p.h_source_r_rate = 0.9
        p.h_drain_l_rate = 0.9
    return p


def kmc_run(L, w, args, seed, replica):
    p = kmc_params(L, w, seed)
    with L.KMC(p, device=int(os.environ.get("LOCAL_RANK", "0")), replica=replica) as k:
        k.run(args.warmup)
        s0 = k.stats()
        t0 = time.perf_counter()
        k.run(args.kmc_steps)
        dt = time.perf_counter() - t0
        s1 = k.stats()
    hops = s1["proposals"] - s0["proposals"]
    return {"workload": w["desc"] + ", traps 2% at 0.2 eV, site disorder 0.05 eV, 1 V",
            "steps": args.kmc_steps, "ms_per_step": 1e3 * dt / args.kmc_steps,
            "hops": hops, "timed_s": dt, "hops_per_s": hops / dt, "accepted_per_s": (s1["accepted"] - s0["accepted"]) / dt,
            "guard_fp64_per_step": (s1["guard_evaluations"] - s0["guard_evaluations"])
            / args.kmc_steps,
            "carriers": s1["electrons"] + s1["holes"],
            "timing": "host wall clock around graph replays of the whole step"}


def _timed_kmc(k, warmup, steps):
    k.run(warmup)
    s0 = k.stats()
    t0 = time.perf_counter()
    k.run(steps)
    dt = time.perf_counter() - t0
    s1 = k.stats()
    return s0, s1, dt


def cfg1_params(L, seed):
    """Hole transport on 128x128x1: 1% holes seeded uniformly, traps on 5% of
    sites at 0.1 eV, cutoff 50, no image charges, 1 V across x with the hole
    source at x = 0 and the drain at x = 127."""
    p = L.Params.default()
    for k, v in dict(grid_x=128, grid_y=128, grid_z=1, hole_percentage=0.01,
                     electron_percentage=0.0, seed_charges=1.0, coulomb_carriers=1,
                     electrostatic_cutoff=50, trap_percentage=0.05, trap_potential=0.1,
                     voltage_left=1.0, e_source_l_rate=0.0, h_source_l_rate=0.9,
                     h_drain_r_rate=0.9, random_seed=seed).items():
        p.set(k, v)
    return p


def cfg3_params(L, seed):
    """Solar cell on 128x128x64 with Gaussian-smeared charges (sigma 1, cutoff
    30): holes confined to donor and electrons to acceptor sites, excitons
    split at donor-acceptor bonds with probability 1e-3 per step,
    recombination of interface pairs with probability 1e-3, 0.5 V across x
    (the engine's field axis), room for 1.25% electrons and holes."""
    p = L.Params.default()
    for k, v in dict(simulation_type="solarcell", grid_x=128, grid_y=128, grid_z=64,
                     electron_percentage=0.0125, hole_percentage=0.0125, seed_charges=0.0,
                     coulomb_carriers=1, coulomb_gaussian_sigma=1.0, electrostatic_cutoff=30,
                     voltage_right=0.5, generation_rate=1e-3, source_scale_area=0.0,
                     recombination_rate=1e-3, recombination_range=1, morphology_confine=1,
                     generation_interface=1, random_seed=seed).items():
        p.set(k, v)
    return p


def kmc_configs_run(L, args, rank, world):
    """The kMC step on config 1 (128x128 holes, with the oracle's FP64 step
    timed beside it on the host) and config 3 (3-D Gaussian solar cell on a
    GRF morphology, 1% electrons on acceptor and 1% holes on donor sites)."""
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    out = {}
    p = cfg1_params(L, seed=11 + rank)
    with L.KMC(p, device=dev, replica=rank) as k:
        s0, s1, dt = _timed_kmc(k, args.warmup, args.cfg1_steps)
        hops = s1["proposals"] - s0["proposals"]
        out["cfg1"] = {"workload": "128x128x1, 1% holes, traps 5% at 0.1 eV, cutoff 50, "
                                   "1 V across x",
                       "steps": args.cfg1_steps, "carriers": s1["holes"],
                       "ms_per_step": 1e3 * dt / args.cfg1_steps, "hops": hops, "timed_s": dt,
                       "hops_per_s": hops / dt,
                       "timing": "host wall clock around graph replays of the whole step"}
        e_single, h_single = k.carriers()
    # the same replica as a batch of one: 163 carriers fit the fused
    # one-block step, which runs many steps per launch instead of one graph
    # replay per step; same Philox key, so the same trajectory
    with L.KMCBatch([p], device=dev, replica0=rank) as b:
        r = b.replica(0)
        b.run(args.warmup)
        f0 = r.stats()
        t0 = time.perf_counter()
        b.run(args.cfg1_steps)
        fdt = time.perf_counter() - t0
        f1 = r.stats()
        e_f, h_f = r.carriers()
        out["cfg1"]["fused_batch_of_one"] = {
            "fused_replicas": b.fused_count, "ms_per_step": 1e3 * fdt / args.cfg1_steps,
            "hops_per_s": (f1["proposals"] - f0["proposals"]) / fdt,
            "same_carriers_as_single": bool(np.array_equal(e_f, e_single)
                                            and np.array_equal(h_f, h_single)),
            "timing": "host wall clock around the batch run (fused kernel launches)"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        with L.KMC(p, device=dev, replica=rank) as k:
            k.run(args.warmup + args.cfg1_steps)  # the state the timed leg ended in
            # the oracle's FP64 kMC step (one host thread) from the same world
            from oracle import oracle as O
            from oracle.kmc_setup import oracle_for
            st = k.stats()
            e, h = k.carriers()
            orc = oracle_for(O, p, k.world(), e, h, st["max_electrons"], st["max_holes"],
                             replica=rank, step=st["step"])
            n_cpu, h0 = 0, orc.counters.copy()
            props = 0
            t0 = time.perf_counter()
            while time.perf_counter() - t0 < args.cfg1_cpu_seconds:
                ne, nh = (len(a) for a in orc.carriers())
                orc.step(threads=1)
                props += ne + nh
                n_cpu += 1
            cdt = time.perf_counter() - t0
            out["cfg1"]["cpu_baseline"] = {
                "value": props / cdt, "unit": "hops/s", "cores": 1, "kind": "port",
                "sample": f"{n_cpu} steps of the oracle's FP64 kMC step (one proposal per "
                          f"carrier per step) from the GPU replica's world ({cdt:.1f} s)"}
    p = cfg3_params(L, seed=13 + rank)
    X, Y, Z = p.grid_x, p.grid_y, p.grid_z
    phase = grf_phase_3d(X, Y, Z, ell=8.0, seed=17 + rank)
    rng = np.random.default_rng(19 + rank)
    n1 = int(0.01 * X * Y * Z)
    e = rng.choice(np.flatnonzero(phase == 1), n1, replace=False).astype(np.int32)
    h = rng.choice(np.flatnonzero(phase == 0), n1, replace=False).astype(np.int32)
    with L.KMC(p, device=dev, replica=rank) as k:
        k.set_morphology(phase)
        k.set_carriers(e, h)
        s0, s1, dt = _timed_kmc(k, args.warmup, args.cfg3_steps)
        hops = s1["proposals"] - s0["proposals"]
        out["cfg3"] = {"workload": "128x128x64 solar cell, GRF morphology (blur 8 sites, median "
                                   "threshold), Gaussian charges sigma 1, cutoff 30, generation "
                                   "and recombination 1e-3 per step, 0.5 V across x, 1% e + 1% h",
                       "steps": args.cfg3_steps,
                       "carriers": s1["electrons"] + s1["holes"],
                       "ms_per_step": 1e3 * dt / args.cfg3_steps, "hops": hops, "timed_s": dt,
                       "hops_per_s": hops / dt,
                       "guard_fp64_per_step": (s1["guard_evaluations"] - s0["guard_evaluations"])
                       / args.cfg3_steps,
                       "timing": "host wall clock around graph replays of the whole step"}
    return out


def batch_params(L, n, seed=4):
    """Replicas drawn as the batched configuration draws them: square lattices
    of side {32,64,128,256} x depth {1,2,4,8}, occupancy U(0.5%, 3%) split
    between electrons and holes, voltage U(0.1, 2) V, traps U(0, 10%) at depth
    U(0.05, 0.3) eV, cutoff 50."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        xy = int(rng.choice([32, 64, 128, 256]))
        z = int(rng.choice([1, 2, 4, 8]))
        occ = float(rng.uniform(0.005, 0.03))
        p = L.Params.default()
        for k, v in dict(grid_x=xy, grid_y=xy, grid_z=z, electron_percentage=occ / 2,
                         hole_percentage=occ / 2, seed_charges=1.0, coulomb_carriers=1,
                         voltage_right=float(rng.uniform(0.1, 2.0)),
                         trap_percentage=float(rng.uniform(0.0, 0.10)),
                         trap_potential=float(rng.uniform(0.05, 0.3)),
                         h_source_r_rate=0.9, h_drain_l_rate=0.9, random_seed=seed).items():
            p.set(k, v)
        out.append(p)
    return out


def fp32_peak_derived(dev):
    """FP32 FMA peak from the SM count and the maximum SM clock: 128 lanes x
    2 FLOP per SM per cycle (TFLOP/s)."""
    import torch
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    return sms * 128 * 2 * float(measured_peaks().get("sm_max_mhz", 1965.0)) * 1e6 / 1e12


def batch_run(L, args, rank):
    """Batched replicas in one graph vs the same replicas stepped one by one."""
    import torch
    params = batch_params(L, args.batch_replicas, seed=4 + rank)
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    t0 = time.perf_counter()
    with L.KMCBatch(params, device=dev, replica0=1000 * rank) as b:
        build_s = time.perf_counter() - t0
        b.run(max(1, args.warmup))  # tunes the tile shape, records the graph
        reps = [b.replica(i) for i in range(len(params))]
        st0 = [r.stats() for r in reps]
        h0 = sum(st["proposals"] for st in st0)
        t0 = time.perf_counter()
        b.run(args.batch_steps)
        dt = time.perf_counter() - t0
        st1 = [r.stats() for r in reps]
        hops = sum(st["proposals"] for st in st1) - h0
        charges = sum(st["electrons"] + st["holes"] for st in st1)
        # pairs the step's Coulomb sums test: 2M targets x M sources per
        # replica, averaged over the carrier counts before and after
        m0 = np.array([st["electrons"] + st["holes"] for st in st0], dtype=np.float64)
        m1 = np.array([st["electrons"] + st["holes"] for st in st1], dtype=np.float64)
        pairs_per_step = float(np.sum(m0 * m0 + m1 * m1))
        # the pair sum alone (CUDA events), after one more step from these counts
        b.run(1)
        pair_ms = b.time_pair(7)
        m2 = np.array([r.stats()["electrons"] + r.stats()["holes"] for r in reps], np.float64)
        pairs_timed = float(np.sum(2.0 * m2 * m2))
        examined = b.count_pairs()
        # pairs inside the cutoff, estimated from the current sites: each
        # replica's 2M targets are its M current sites and M proposed sites
        # one hop away, so about twice the current-current pairs
        p_in = 0
        for i, r in enumerate(reps):
            e, h = r.carriers()
            sites = np.concatenate([e, h])
            p = params[i]
            w = {"X": p.grid_x, "Y": p.grid_y, "cutoff": p.electrostatic_cutoff}
            p_in += 2 * pairs_in_cutoff(w, sites, sites, 1, torch.device("cuda", dev))
        tuning = b.tuning()
        fused = b.fused_count
        culled = b.culled_count
    # the same replicas with every one on the per-phase kernels
    with L.KMCBatch(params, device=dev, replica0=1000 * rank, fused_max_charges=0) as b:
        b.run(max(1, args.warmup))
        reps = [b.replica(i) for i in range(len(params))]
        h0 = sum(r.stats()["proposals"] for r in reps)
        t0 = time.perf_counter()
        b.run(args.batch_steps)
        pp_dt = time.perf_counter() - t0
        pp_hops = sum(r.stats()["proposals"] for r in reps) - h0
    # the plain single-replica path on a stratified sample of the same replicas
    sample = list(range(0, len(params), max(1, len(params) // args.batch_sample)))
    s_hops, s_time = 0, 0.0
    for i in sample:
        with L.KMC(params[i], device=dev, replica=1000 * rank + i) as k:
            k.run(max(1, args.warmup))
            h = k.stats()["proposals"]
            t1 = time.perf_counter()
            k.run(args.batch_steps)
            s_time += time.perf_counter() - t1
            s_hops += k.stats()["proposals"] - h
    single = s_hops / s_time
    fp32_peak = fp32_peak_derived(torch.device("cuda", dev))
    ach = (FLOP_PER_TEST * examined + FLOP_PER_CONTRIB * p_in) / (pair_ms * 1e-3) / 1e12
    return {"workload": f"{len(params)} replicas, side {{32,64,128,256}} x depth {{1,2,4,8}}, "
                        "occupancy U(0.5%,3%) e/h, V U(0.1,2), traps U(0,10%) at U(0.05,0.3) eV, "
                        "cutoff 50",
            "steps": args.batch_steps, "charges": charges,
            "ms_per_step": 1e3 * dt / args.batch_steps, "hops": hops, "timed_s": dt,
            "hops_per_s": hops / dt,
            "single_replica_hops_per_s": single,
            "single_replica_sample": f"{len(sample)} of {len(params)} replicas stepped one by one",
            "speedup_vs_single": (hops / dt) / single, "tuning": tuning,
            "pairs_per_step": pairs_per_step,
            "pair_evals_per_s_in_step": pairs_per_step / (dt / args.batch_steps),
            "pair_kernel": {"ms": pair_ms, "pairs_reference": pairs_timed,
                            "pairs_examined": examined,
                            "pairs_inside_cutoff_estimate": p_in,
                            "pair_evals_per_s": pairs_timed / (pair_ms * 1e-3),
                            "examined_per_s": examined / (pair_ms * 1e-3),
                            "roofline": {"bound": "fp32", "achieved": ach,
                                         "peak": fp32_peak, "unit": "TFLOP/s",
                                         "frac": ach / fp32_peak,
                                         "basis": f"{FLOP_PER_TEST} FLOP per pair examined + "
                                                  f"{FLOP_PER_CONTRIB} per pair inside the "
                                                  "cutoff (estimated)"},
                            "timing": "CUDA events around the batched pair sum alone (culled "
                                      "replicas' boxes, culls and culled launch, then the "
                                      "work-item kernel), median of 7, over one step's charges"},
            "fused_replicas": fused, "culled_replicas": culled,
            "per_phase_only": {"ms_per_step": 1e3 * pp_dt / args.batch_steps,
                               "hops_per_s": pp_hops / pp_dt},
            "build_s": build_s}


def _kernel_leg(L, ctx, args, w, s_all, q_all, n, kind, terms, dev, st, fp32_peak,
                all_sites=False):
    """One timed pair-sum workload on a context: the autotuned tile variant,
    the pair kernel's own CUDA events (median over args.steps after
    args.warmup), one untimed call counting the pairs the culled kernel
    examines, the FP64 oracle's accuracy on 512 targets, and the roofline on
    the work done (8 FLOP per pair examined + 3 per pair inside the cutoff)."""
    import torch
    T = w["X"] * w["Y"] * w["Z"] if all_sites else len(s_all)
    d_s = torch.from_numpy(s_all[: (n if all_sites else T)].copy()).to(dev)
    d_q = torch.from_numpy(q_all[: (n if all_sites else T)].copy()).to(dev)
    d_o = torch.empty(T, dtype=torch.float64, device=dev)

    def call():
        if all_sites:
            ctx.kernel1_async(d_s.data_ptr(), d_q.data_ptr(), n, d_o.data_ptr(), kind,
                              st.cuda_stream)
        else:
            ctx.potentials_async(d_s.data_ptr(), d_q.data_ptr(), n, d_s.data_ptr(), T,
                                 d_o.data_ptr(), kind, terms, st.cuda_stream)
        ctx.sync(st.cuda_stream)
    v = ctx.autotune(n, T, kind, terms)
    ctx.set_variant(v)
    ctx.set_timing(True)
    ms = []
    for i in range(args.warmup + args.steps):
        call()
        if i >= args.warmup:
            ms.append(ctx.last_launch()["pair_kernel_ms"])
    ctx.set_timing(False)
    ctx.set_counting(True)
    call()
    examined = ctx.last_launch()["pairs_examined"]
    ctx.set_counting(False)
    pk = float(np.median(ms))
    nterms = bin(terms).count("1")
    pairs = nterms * n * T
    tgt = np.arange(T, dtype=np.int32) if all_sites else s_all
    idx = np.linspace(0, T - 1, 512).astype(int)
    acc = accuracy_vs_oracle(w, s_all[:n], q_all[:n], tgt[idx], d_o.cpu().numpy()[idx], terms)
    p_in = pairs_in_cutoff(w, tgt, s_all[:n], terms, dev)
    done = examined if examined >= 0 else pairs
    achieved = (FLOP_PER_TEST * done + FLOP_PER_CONTRIB * p_in) / (pk * 1e-3) / 1e12
    return {"pairs_reference": pairs, "pairs_examined": done, "pairs_inside_cutoff": p_in,
            "pair_kernel_ms": pk, "pair_evals_per_s": pairs / (pk * 1e-3),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                         "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                         "basis": f"{FLOP_PER_TEST} FLOP per pair examined + "
                                  f"{FLOP_PER_CONTRIB} per pair inside the cutoff"},
            "tile_variant": dict(ctx.variants()[v], id=v), "accuracy": acc}


def other_kernels_run(L, args, fp32_peak):
    """Rows a2 and a3 and the other accumulation paths: the Gaussian kernel-2
    sum on config 3 (128x128x64, sigma 1, cutoff 30), the cfg2 kernel-2 sum
    through the FP32 1/sqrt(k) table and through the FP64 table (TABLE64,
    FP64-accurate sums), and the whole-grid kernel 1 on config 1's lattice and
    on the 1,048,576 sites of the 256x256x16 lattice -- pair kernel time from
    the library's own CUDA events."""
    import torch
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    st = torch.cuda.Stream(dev)
    out = {}
    # gauss2, config 3, FP32 rsqrt path and FP64 table path
    w = WORKLOADS["cfg3_gauss"]
    s_all, q_all, n = make_inputs(w, 5)
    for key, path, what in (("gauss2_cfg3", L.PATH_RSQRT, ""),
                            ("gauss2_table64_cfg3", L.PATH_TABLE64,
                             ", FP64 w(k) table, every term added in FP64")):
        with L.Coulomb(w["X"], w["Y"], w["Z"], cutoff=w["cutoff"], sigma=w["sigma"],
                       device=dev.index, path=path) as ctx:
            out[key] = dict(workload=w["desc"] + what, **_kernel_leg(
                L, ctx, args, w, s_all, q_all, n, L.GAUSS, 1, dev, st, fp32_peak))
    # cfg2 through the FP32 1/sqrt(k) table and through the FP64 table
    w = WORKLOADS["cfg2_3d_eh_images"]
    s_all, q_all, n = make_inputs(w, 7)
    for key, path, what in (("table_cfg2", L.PATH_TABLE, "FP32 1/sqrt(k) table path"),
                            ("table64_cfg2", L.PATH_TABLE64,
                             "FP64 w(k) table, every term added in FP64")):
        with L.Coulomb(w["X"], w["Y"], w["Z"], cutoff=w["cutoff"], device=dev.index,
                       path=path) as ctx:
            leg = _kernel_leg(L, ctx, args, w, s_all, q_all, n, L.POINT, w["terms"], dev, st,
                              fp32_peak)
            # one table entry gathered from shared memory per pair examined
            # (4 B FP32, 8 B FP64)
            nb = 8 if path == L.PATH_TABLE64 else 4
            leg["shared_memory_gather_gbs"] = nb * leg["pairs_examined"] / (
                leg["pair_kernel_ms"] * 1e-3) / 1e9
            out[key] = dict(workload=w["desc"] + ", " + what, **leg)
    # kernel 1: every site of config 1's lattice (163 charges) and of the
    # 256x256x16 lattice (20,970 charges), point charges, cutoff 50
    w = WORKLOADS["cfg1_2d_holes"]
    s_all, q_all, n = make_inputs(w, 6)
    with L.Coulomb(w["X"], w["Y"], w["Z"], cutoff=w["cutoff"], device=dev.index) as ctx:
        leg = _kernel_leg(L, ctx, args, w, s_all, q_all, n, L.POINT, 1, dev, st, fp32_peak,
                          all_sites=True)
        out["kernel1_cfg1"] = dict(workload=f"every site of {w['desc']}", charges=n,
                                   note="163 charges: launch- and latency-bound; the "
                                        "reference runs this only for output.coulomb", **leg)
    w = dict(WORKLOADS["cfg2_3d_eh_images"], terms=1)
    s_all, q_all, n = make_inputs(w, 8)
    with L.Coulomb(w["X"], w["Y"], w["Z"], cutoff=w["cutoff"], device=dev.index) as ctx:
        leg = _kernel_leg(L, ctx, args, w, s_all, q_all, n, L.POINT, 1, dev, st, fp32_peak,
                          all_sites=True)
        out["kernel1_1M_sites"] = dict(
            workload="every site of 256x256x16 (1,048,576 sites), 1% electrons + 1% holes, "
                     "cutoff 50", charges=n,
            note="the output.coulomb dump (writer.cpp:545-581) at a size where it matters",
            **leg)
    return out


def cnn_layers(S, peaks):
    """Per-layer timing of the surrogate's conv kernels (1024 images, CUDA
    events): layer 1 against HBM, layer 2 against the measured bf16 GEMM peak."""
    import torch
    B = 1024
    ph, _, _ = S.grf_morphologies(B, seed=11)
    x16 = S.phases_to_input(ph)
    prm = S.init_params(0)
    w1, w2 = S.conv_weights_bf16(prm[0], 1), S.conv_weights_bf16(prm[2], 32)
    _, p1 = S.conv3x3(x16, w1, prm[1], 128, 128, keep_act=False)

    def timeit(fn, n=20):
        for _ in range(3):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n
    t1 = timeit(lambda: S.conv3x3(x16, w1, prm[1], 128, 128, keep_act=False))
    t2 = timeit(lambda: S.conv3x3(p1, w2, prm[3], 64, 64, keep_act=False))
    b1 = B * 128 * 128 * 2 + B * 64 * 64 * 32 * 2            # image in, pooled map out
    f2 = 2 * B * 64 * 64 * 32 * 288                            # layer-2 MACs x 2
    hbm, bf16 = float(peaks.get("hbm_gbs", 6650.0)), float(peaks.get("bf16_tflops", 1590.0))
    # the 32-channel layers on both tensor-core kernels (tcgen05 is the product path)
    compare = {}
    for size, pool in ((64, True), (32, True), (16, False)):
        xin = torch.randn(B, size, size, 32, device="cuda").to(torch.bfloat16)
        fl = 2 * B * size * size * 32 * 288
        ms = {name: timeit(lambda f=f: f(xin, w2, prm[3], size, size, keep_act=not pool, pool=pool))
              for name, f in (("tcgen05", S.conv3x3_tc), ("mma_sync", S.conv3x3_mma))}
        compare[f"{size}x{size}"] = {k + "_tflops": fl / (v * 1e-3) / 1e12 for k, v in ms.items()}
    return {"images": B, "conv32_tcgen05_vs_mma_sync": compare,
            "conv1_pool": {"ms": t1, "achieved": b1 / (t1 * 1e-3) / 1e9, "peak": hbm,
                           "unit": "GB/s", "frac": b1 / (t1 * 1e-3) / 1e9 / hbm, "bound": "hbm"},
            "conv2_pool": {"ms": t2, "achieved": f2 / (t2 * 1e-3) / 1e12, "peak": bf16,
                           "unit": "TFLOP/s", "frac": f2 / (t2 * 1e-3) / 1e12 / bf16,
                           "bound": "tensor",
                           "note": "tcgen05.mma M128 N32 K16 bf16, TMA-loaded patches; peak = "
                                   "measured cuBLAS bf16 GEMM"}}


def surrogate_run(args, rank):
    """Morphology screening: the CNN ensemble over fresh GRF candidates vs
    labelling the same kind of morphology with the batched solar-cell kMC."""
    import torch
    from langmuir_b200 import surrogate as S
    from langmuir_b200.kmc import KMCBatch
    n = args.surrogate_candidates
    t0 = time.perf_counter()
    cand, _, _ = S.grf_morphologies(n, seed=7 + rank)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    model = S.Surrogate(members=4, seed=rank)  # throughput does not depend on the weights
    for _ in range(args.warmup):
        S.screen(model, cand[:4096])
    S.screen(model, cand)  # the full size once: buffers of that size are cached after it
    torch.cuda.synchronize()
    times = []
    for _ in range(max(3, args.steps // 10)):
        t0 = time.perf_counter()
        S.screen(model, cand)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    screen_s = float(np.median(times))
    # kMC labels of the same morphologies: set-up, steady steps, teardown
    R, full = args.surrogate_label_replicas, 50000
    K = min(args.surrogate_label_steps, full - args.warmup)  # the rest of the label run
    ph = cand[:R].cpu().numpy()
    t0 = time.perf_counter()
    b = KMCBatch([S.solar_label_params(size=128, seed=1) for _ in range(R)], replica0=0,
                 fused_max_charges=0 if args.label_form == "per_phase" else None)
    reps = [b.replica(i) for i in range(R)]
    for i, r in enumerate(reps):
        r.set_morphology(ph[i].reshape(-1))
    b.run(args.warmup)
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    b.run(K)
    step_s = (time.perf_counter() - t0) / K
    t0 = time.perf_counter()
    b.close()
    teardown_s = time.perf_counter() - t0
    kmc_label_s = setup_s + teardown_s + (full - args.warmup) * step_s
    out = {"workload": f"{n} GRF candidates 128x128, l ~ U(2,16), donor fraction ~ U(0.4,0.6); "
                       "4-member CNN ensemble, BF16 tensor-core kernels",
           "surrogate_morphs_per_s": n / screen_s, "screen_ms": 1e3 * screen_s,
           "generate_ms": 1e3 * gen_s,
           "kmc_morphs_per_s": R / kmc_label_s,
           "kmc_label": {"replicas": R, "steps_per_label": full, "timed_steps": K,
                         "form": args.label_form,
                         "ms_per_batched_step": 1e3 * step_s, "setup_s": setup_s,
                         "teardown_s": teardown_s,
                         "note": (f"the whole {full}-step label run timed: set-up with "
                                  f"{args.warmup} steps, {K} steps, teardown"
                                  if K == full - args.warmup else
                                  f"{full}-step label cost = set-up with {args.warmup} steps + "
                                  f"teardown + {full - args.warmup} x the batched step time "
                                  f"measured over {K} steps")},
           "speedup_vs_kmc": (n / screen_s) / (R / kmc_label_s),
           "cnn_layers": cnn_layers(S, measured_peaks())}
    if rank == 0 and not args.no_cpu_baseline:
        # the reference's screening score (ga.py:83-141), restated, on the host
        from oracle import ga_score as G
        imgs = [G.phases_to_image(p) for p in ph[:64]]
        t0 = time.perf_counter()
        for im in imgs:
            G.score(im)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": len(imgs) / dt, "unit": "morphs/s", "cores": 1,
                               "kind": "port", "sample": f"ga.py score of {len(imgs)} candidates"}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=list(WORKLOADS))
    ap.add_argument("--path", type=int, default=0, help="0 MUFU rsqrt, 1 1/sqrt(k) table")
    ap.add_argument("--variant", type=int, default=-1, help="tile variant, -1 = autotune")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-kmc", action="store_true")
    ap.add_argument("--kmc-steps", type=int, default=50)
    ap.add_argument("--no-configs", action="store_true", help="skip the config 1 and 3 kMC legs")
    ap.add_argument("--cfg1-steps", type=int, default=2000)
    ap.add_argument("--cfg1-cpu-seconds", type=float, default=5.0)
    ap.add_argument("--cfg3-steps", type=int, default=50)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--batch-replicas", type=int, default=512)
    ap.add_argument("--batch-steps", type=int, default=20)
    ap.add_argument("--batch-sample", type=int, default=32)
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--no-other-kernels", action="store_true")
    ap.add_argument("--surrogate-candidates", type=int, default=100000)
    ap.add_argument("--surrogate-label-replicas", type=int, default=4096)
    ap.add_argument("--label-form", default="fused", choices=["fused", "per_phase"],
                    help="step form of the label batch")
    ap.add_argument("--surrogate-label-steps", type=int, default=50000,
                    help="label steps timed (past the warm-up; fewer are extrapolated)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    w = WORKLOADS[args.workload]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        reference_arm(args, w, rank)
        return

    import torch
    import langmuir_b200 as L

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    s_all, q_all, n = make_inputs(w, seed=2 + rank)
    T = len(s_all)
    nterms = bin(w["terms"]).count("1")
    pairs_per_step = nterms * T * n

    ctx = L.Coulomb(w["X"], w["Y"], w["Z"], cutoff=w["cutoff"], sigma=w["sigma"],
                    device=local_rank, path=args.path)
    kind = L.GAUSS if w["sigma"] > 0 else L.POINT
    dev = torch.device("cuda", local_rank)
    d_s = torch.from_numpy(s_all).to(dev)
    d_q = torch.from_numpy(q_all).to(dev)
    d_out = torch.empty(T, dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream(dev)  # a real stream: handle 0 would mean the context's own
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2

    def step():
        ctx.potentials_async(d_s.data_ptr(), d_q.data_ptr(), n, d_s.data_ptr(), T,
                             d_out.data_ptr(), kind, w["terms"], sp)

    variant = ctx.autotune(n, T, kind, w["terms"]) if args.variant < 0 else args.variant
    ctx.set_variant(variant)
    for _ in range(args.warmup):
        step()
    ctx.sync(sp)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    pair_ms = []
    launches = 0
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize(dev)
        for i in range(args.steps):
            flush.zero_()  # L2 flush between timed steps (outside the events)
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
            launches += ctx.last_launch()["kernel_launches"]
        torch.cuda.synchronize(dev)
    ctx.sync(sp)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    # the pair kernel alone: the same steps again, untimed, with its own
    # events on (events between the call's kernels hold back the launch
    # overlap, so the timed steps above run without them)
    ctx.set_timing(True)
    for i in range(args.steps):
        flush.zero_()
        step()
        pair_ms.append(ctx.last_launch()["pair_kernel_ms"])
    ctx.set_timing(False)
    ctx.sync(sp)
    # one more call, untimed, counting the pairs the culled kernel examines
    ctx.set_counting(True)
    step()
    ctx.sync(sp)
    examined = ctx.last_launch()["pairs_examined"]
    ctx.set_counting(False)
    job_pairs, span_s = job_totals(dist, pairs_per_step * args.steps, 1e-3 * sum(step_ms))
    if dist:
        dist.barrier()
    clocks = clk.summary()
    ms_per_step = 1e3 * span_s / args.steps
    value = job_pairs / span_s

    # accuracy on a sample of targets against the FP64 oracle (the checker)
    o = d_out.cpu().numpy()
    acc = None
    if rank == 0:
        idx = np.linspace(0, T - 1, 512).astype(int)
        acc = accuracy_vs_oracle(w, s_all[:n], q_all[:n], s_all[idx], o[idx], w["terms"])

    # end to end through the host-buffer ABI: H2D inputs, kernels, D2H result
    e2e = None
    if rank == 0:
        h_s = s_all.copy()
        h_q = q_all.copy()
        h_o = np.empty(T, dtype=np.float64)  # one result array, reused as a stepping caller does
        for _ in range(3):
            ctx.potentials(h_s[:n], h_q[:n], h_s, kind, w["terms"], out=h_o)
        t0 = time.perf_counter()
        k_e2e = max(3, args.steps // 2)
        for _ in range(k_e2e):
            ctx.potentials(h_s[:n], h_q[:n], h_s, kind, w["terms"], out=h_o)
        dt = (time.perf_counter() - t0) / k_e2e
        # host->device per call, one copy: the T int32 site ids (the sources are
        # their first n) and the n int32 charges; device->host, one copy: T
        # doubles and the device error word behind them (one more double)
        e2e = {"value": pairs_per_step / dt, "unit": "pair-evals/s",
               "h2d_bytes_per_step": int(4 * (n + T)), "d2h_bytes_per_step": int(8 * (T + 1))}

    # the fused kMC step on the same lattice and occupancy: hops per second
    kmc = None
    if not args.no_kmc and w["e"] + w["h"] > 0:
        kmc = kmc_run(L, w, args, seed=2 + rank, replica=rank)
        if dist:
            h, t = job_totals(dist, kmc["hops"], kmc["timed_s"])
            kmc["job_hops_per_s"] = h / t

    configs = None
    if not args.no_configs:
        configs = kmc_configs_run(L, args, rank, world)
        if dist:
            for key in ("cfg1", "cfg3"):
                h, t = job_totals(dist, configs[key]["hops"], configs[key]["timed_s"])
                configs[key]["job_hops_per_s"] = h / t

    batch = None
    if not args.no_batch:
        batch = batch_run(L, args, rank)
        if dist:
            h, t = job_totals(dist, batch["hops"], batch["timed_s"])
            batch["job_hops_per_s"] = h / t

    surrogate = None
    if not args.no_surrogate:
        surrogate = surrogate_run(args, rank)
        if dist:
            m, t = job_totals(dist, args.surrogate_candidates, 1e-3 * surrogate["screen_ms"])
            surrogate["job_morphs_per_s"] = m / t

    peaks = measured_peaks()
    props = torch.cuda.get_device_properties(dev)
    sms = props.multi_processor_count
    clk_max = float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak = fp32_peak_derived(dev)                         # TFLOP/s, derived
    sfu_peak = sms * 16 * clk_max * 1e6                        # rsqrt/s, derived
    pk = float(np.median(pair_ms))
    p_in = pairs_in_cutoff(w, s_all, s_all[:n], w["terms"], dev)
    # pairs whose r^2 the kernel computes: all of them for the grid tiles, the
    # live 32-source groups of each warp for the culled kernel
    done = examined if examined >= 0 else pairs_per_step
    achieved = (FLOP_PER_TEST * done + FLOP_PER_CONTRIB * p_in) / (pk * 1e-3) / 1e12
    roof = {
        "bound": "fp32", "kernel": "pair_kernel", "achieved": achieved, "peak": fp32_peak,
        "unit": "TFLOP/s", "frac": achieved / fp32_peak,
        "flop_basis": (f"{FLOP_PER_TEST} per pair examined (r^2) + {FLOP_PER_CONTRIB} per pair "
                       "inside the cutoff (1/r, q/r + acc)"),
        "pairs_reference": pairs_per_step, "pairs_examined": done, "pairs_inside_cutoff": p_in,
        "reference_pair_evals_per_s_in_kernel": pairs_per_step / (pk * 1e-3),
        "peak_source": (f"derived: {sms} SMs x 128 FP32 lanes x 2 x {clk_max:.0f} MHz "
                        "(sm_max_mhz of MEASURED_PEAKS.json); no measured FP32 figure exists"),
        "sfu_frac_lower_bound": (p_in / (pk * 1e-3)) / sfu_peak,
        "pair_kernel_ms": pk,
        "traffic": PAIR_KERNEL_DRAM_BYTES,
    }
    if clocks.get("sm_mhz"):
        roof["frac_at_sampled_clock"] = achieved / (sms * 256 * clocks["sm_mhz"] * 1e6 / 1e12)
    # measured FP32 FMA and MUFU rsqrt throughput of this device (lgm_probe_peaks)
    from langmuir_b200 import _native as LN
    probe = LN.probe_peaks(local_rank)
    fp32_measured = max(probe["ffma_tflops"], probe["ffma2_tflops"])
    roof["fp32_measured"] = {"tflops": fp32_measured, "ffma_tflops": probe["ffma_tflops"],
                             "ffma2_tflops": probe["ffma2_tflops"],
                             "rsqrt_per_s": probe["rsqrt_per_s"],
                             "frac_of_measured": achieved / fp32_measured,
                             "how": "FMA / FFMA2 / MUFU rsqrt chains, 8 per thread, 8 x 256 "
                                    "threads per SM, best of 5 launches (CUDA events)"}

    others = None if args.no_other_kernels else other_kernels_run(L, args, fp32_peak)
    if kmc is not None:
        # the reference's pair tests the step's Coulomb sums stand for, over the
        # whole step time (a rate of the reference's work, not a roofline)
        kp = kmc["carriers"] * 2 * kmc["carriers"] * nterms
        kmc["pair_evals_per_s_in_step"] = kp / (kmc["ms_per_step"] * 1e-3)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, dt, sample = cpu_baseline_run(w, s_all, q_all, n, args.cpu_seconds, threads)
        cpu = {"value": v, "unit": "pair-evals/s", "cores": threads, "kind": "port",
               "sample": sample + f" ({dt:.1f} s)"}

    if rank == 0:
        line = {
            "metric": "Coulomb pair-evals/s", "value": value, "unit": "pair-evals/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": {"workload": args.workload, "desc": w["desc"], "sources": n,
                       "targets": T, "terms": nterms, "pairs_per_step": pairs_per_step,
                       "path": "table" if args.path else "rsqrt", "l2": "flushed between steps",
                       "tile_variant": dict(ctx.variants()[variant], id=variant),
                       "parallelism": "replicas" if world > 1 else "single"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": launches, "accuracy": acc,
            "other_kernels": others, "surrogate": surrogate, "kmc_configs": configs,
            "kmc_batched": batch, "kmc": kmc,
        }
        # the hop rates last, where a tail of the output keeps them
        line["summary"] = {
            "pair_evals_per_s": value, "e2e_pair_evals_per_s": e2e and e2e["value"],
            "pair_kernel_frac_of_fp32": roof["frac"],
            "kmc_cfg2_hops_per_s": kmc and kmc["hops_per_s"],
            "kmc_cfg1_hops_per_s": configs and configs["cfg1"]["hops_per_s"],
            "kmc_cfg3_hops_per_s": configs and configs["cfg3"]["hops_per_s"],
            "kmc_batched_hops_per_s": batch and batch["hops_per_s"],
            "kmc_batched_speedup_vs_single": batch and batch["speedup_vs_single"],
            "surrogate_screen_speedup_vs_kmc": surrogate and surrogate.get("speedup_vs_kmc"),
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
