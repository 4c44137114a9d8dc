"""The N > 1 bench path on the CPU: two gloo ranks on 127.0.0.1.

bench.py runs N GPUs as independent replicas (the Coulomb path does not
shard): every rank draws its own seeded inputs, times its own steps, and the
whole-job figure is the units of all ranks over the longest rank's time.  No
data-path collective exists; ``job_totals`` is the only exchange.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, legs, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        res = [bench.job_totals(dist, u, s) for u, s in legs[rank]]
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


def _fake_label_slice(ph, replica_start, steps, burn_in, seed, device, chunk, setup):
    # a stand-in for the GPU labeller: each label a function of the replica id
    ids = replica_start + np.arange(len(ph), dtype=np.float64)
    return {"current": ids, "efficiency": 0.5 * ids, "generated": ids + 7.0,
            "recombined": ids % 3}


def _label_rank(rank, world, port, n, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from langmuir_b200 import surrogate as S
    S._label_slice = _fake_label_slice
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ph = np.zeros((n, 4, 4), np.uint8)
        got = S.kmc_labels(ph, steps=10, burn_in=2, replica0=100, group=dist.group.WORLD)
        out.put((rank, {k: got[k].tolist() for k in S.LABEL_KEYS}))
    finally:
        dist.destroy_process_group()


def _run(world, legs):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, legs, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return got


def test_job_totals_sum_units_and_max_time_over_two_ranks():
    # three legs in the same order on both ranks, as main() issues them
    legs = {0: [(1000, 0.50), (7, 2.0), (3.5e10, 1.25)],
            1: [(1200, 0.75), (9, 1.5), (3.5e10, 1.00)]}
    got = _run(2, legs)
    want = [(2200.0, 0.75), (16.0, 2.0), (7.0e10, 1.25)]
    for r in (0, 1):
        assert got[r] == want  # every rank sees the same whole-job figures


def test_job_totals_without_a_group_is_the_rank_itself():
    import bench
    assert bench.job_totals(None, 123, 0.5) == (123.0, 0.5)


def test_replica_inputs_differ_by_rank_with_equal_work():
    import bench
    w = bench.WORKLOADS[bench.DEFAULT_WORKLOAD]
    s0, q0, n0 = bench.make_inputs(w, seed=2)
    s1, q1, n1 = bench.make_inputs(w, seed=3)
    assert n0 == n1 and len(s0) == len(s1)          # pairs per step equal on every rank
    assert np.array_equal(q0, q1)                   # same charge split
    assert not np.array_equal(s0, s1)               # different placements
    for s, n in ((s0, n0), (s1, n1)):
        assert len(np.unique(s[:n])) == n           # no two carriers on one site
        assert s.min() >= 0 and s.max() < w["X"] * w["Y"] * w["Z"]


def test_reference_arm_under_torchrun_prints_one_line_from_rank_0(oracle_mod):
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--workload", "cfg1_2d_holes", "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] in ("port", "reference")


@pytest.mark.parametrize("n", [7, 1])
def test_sharded_labels_equal_unsharded(n):
    """Replica sharding of the label batch (surrogate.kmc_labels with a
    process group): each rank labels its slice, morphology i stays replica
    replica0 + i, and the gathered labels equal the one-GPU ones on every rank."""
    sys.path.insert(0, ROOT)
    from langmuir_b200 import surrogate as S
    want = _fake_label_slice(np.zeros((n, 4, 4)), 100, 10, 2, 1, 0, 4096, {})
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_label_rank, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        for k in S.LABEL_KEYS:
            np.testing.assert_array_equal(got[r][k], want[k])
