"""Halo sharding across ranks (one process per GPU).

Halos are independent, as in the reference's MPI task farm
(NewGalFinder/gfind.c:394-540, which hands halos to idle ranks one at a
time), so the stage needs no collective on its data path: each rank runs its
own halos and the per-particle outputs are gathered once on the host.  The
farm's dynamic balance is replaced by a static longest-processing-time
partition on an estimate of each halo's cost (N log N for the tree walks plus
the mesh cells), computed identically on every rank.
"""
from __future__ import annotations

import numpy as np

from .synth import HaloBatch


def halo_cost(pstart, mesh_cells=None) -> np.ndarray:
    """Cost estimate per halo: N log2 N (+ mesh cells / 16 when given)."""
    n = np.diff(np.asarray(pstart, np.int64)).astype(np.float64)
    cost = n * np.log2(np.maximum(n, 2.0))
    if mesh_cells is not None:
        cost = cost + np.asarray(mesh_cells, np.float64) / 16.0
    return cost


def lpt_partition(cost, world: int) -> np.ndarray:
    """Owner rank of each halo: halos in decreasing cost (ties by index) go
    to the least-loaded rank (ties by rank).  Deterministic, so every rank
    computes the same partition without communicating."""
    cost = np.asarray(cost, np.float64)
    owner = np.empty(len(cost), np.int32)
    load = np.zeros(world, np.float64)
    for h in np.lexsort((np.arange(len(cost)), -cost)):
        r = int(np.argmin(load))
        owner[h] = r
        load[r] += cost[h]
    return owner


def take_halos(hb: HaloBatch, halos) -> HaloBatch:
    """The given halos of a batch, concatenated in the given order."""
    halos = np.asarray(halos, np.int64)
    ps = np.asarray(hb.pstart, np.int64)
    counts = ps[halos + 1] - ps[halos]
    idx = np.concatenate([np.arange(ps[h], ps[h + 1]) for h in halos]) if len(halos) else np.zeros(0, np.int64)
    f = {k: getattr(hb, k)[idx] for k in ("x", "y", "z", "vx", "vy", "vz", "mass", "type", "ids")}
    pstart = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    return HaloBatch(**f, pstart=pstart, meta=dict(hb.meta, halos=halos))


def gather_particle_outputs(local: dict, halos, pstart, group=None, dst: int = 0):
    """Gathers per-particle outputs of each rank's halos (arrays whose first
    axis runs over the rank's particles, halos in `halos` order) into the
    catalogue's particle order on rank dst (None elsewhere).  One host-side
    gather of Python objects over the process group (gloo or NCCL)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    parts = [None] * world if rank == dst else None
    dist.gather_object((np.asarray(halos, np.int64), {k: np.asarray(v) for k, v in local.items()}), parts,
                       dst=dst, group=group)
    if rank != dst:
        return None
    ps = np.asarray(pstart, np.int64)
    n = int(ps[-1])
    out = {}
    for hs, arrs in parts:
        off = 0
        for h in hs:
            a, b = int(ps[h]), int(ps[h + 1])
            for k, v in arrs.items():
                if k not in out:
                    out[k] = np.zeros((n,) + v.shape[1:], v.dtype)
                out[k][a:b] = v[off:off + (b - a)]
            off += b - a
    return out


def max_over_ranks(value: float, device="cpu", group=None) -> float:
    """The slowest rank's time (the job's time)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sum_over_ranks(value: float, device="cpu", group=None) -> float:
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())
