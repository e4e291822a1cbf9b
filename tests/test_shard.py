"""CPU, world size 2 over gloo: the multi-rank host logic.  Halos are
partitioned by LPT on a cost estimate (identically on every rank), each rank
computes its halos, and one host gather puts the per-particle outputs back in
catalogue order; the slowest rank's time and the summed work are reduced.
The per-halo computation here is the oracle's exact kNN density, so the
gathered result must equal the single-process one bit for bit.  Also runs
bench.py's reference arm under torchrun with two ranks (rank 0 alone
prints)."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

from galaxyfinder_b200 import shard, synth

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _catalogue():
    return synth.catalogue(seed=synth.SEED_BASE + 77, nhalo=24, nmin=40, nmax=1500)


def _halo_density(hb, h):
    from oracle.oracle import Restatement
    r = Restatement()
    a, b = int(hb.pstart[h]), int(hb.pstart[h + 1])
    p = np.stack([hb.x[a:b], hb.y[a:b], hb.z[a:b]], 1)
    p = (p - p.min(0)).astype(np.float32)
    k = min(32, b - a)
    idx, d2 = r.knn(p[:, 0], p[:, 1], p[:, 2], k, "brute")
    return r.sph_density(d2)


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        hb = _catalogue()
        owner = shard.lpt_partition(shard.halo_cost(hb.pstart), world)
        mine = np.nonzero(owner == rank)[0]
        dens = np.concatenate([_halo_density(hb, h) for h in mine]) if len(mine) else np.zeros(0, np.float32)
        out = shard.gather_particle_outputs({"dens": dens, "rank": np.full(len(dens), rank, np.int32)},
                                            mine, hb.pstart)
        t = shard.max_over_ranks(1.0 + rank)
        n = shard.sum_over_ranks(float(len(dens)))
        if rank == 0:
            q.put((out["dens"], out["rank"], owner, t, n))
    finally:
        dist.destroy_process_group()


def test_lpt_partition_balances_and_is_deterministic():
    cost = np.array([9.0, 7, 6, 5, 4, 3, 3, 1])
    o = shard.lpt_partition(cost, 3)
    load = np.bincount(o, weights=cost, minlength=3)
    assert load.max() - load.min() <= cost.min() + 3
    np.testing.assert_array_equal(o, shard.lpt_partition(cost, 3))
    assert np.all(shard.lpt_partition(cost, 1) == 0)


def test_take_halos_keeps_particles():
    hb = _catalogue()
    sub = shard.take_halos(hb, [3, 0, 7])
    assert sub.nhalo == 3
    a, b = int(hb.pstart[3]), int(hb.pstart[4])
    np.testing.assert_array_equal(sub.x[: b - a], hb.x[a:b])


def test_two_ranks_gather_matches_one_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    dens, ranks, owner, t, n = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    hb = _catalogue()
    want = np.concatenate([_halo_density(hb, h) for h in range(hb.nhalo)])
    np.testing.assert_array_equal(dens, want)
    # every particle came from its halo's owner, and both ranks had work
    np.testing.assert_array_equal(ranks, np.repeat(owner, np.diff(hb.pstart)))
    assert set(owner) == {0, 1}
    assert t == 2.0 and n == float(hb.n)


def test_bench_reference_arm_under_torchrun():
    env = dict(os.environ, OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--nhalo", "64"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference"
