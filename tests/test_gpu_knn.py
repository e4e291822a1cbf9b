"""GPU parity of the octree kNN + SPH density against the reference's own
findsphdensity (golden fixture, INSERT-fixed build) and the exact oracle."""
import numpy as np
import pytest
import torch

from galaxyfinder_b200 import _lib, batch, dropin, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(cuda_device):
    c = batch.Context(0)
    yield c
    c.close()


def _recentred_fp32(hb, h):
    a, b = hb.pstart[h], hb.pstart[h + 1]
    p = np.stack([hb.x[a:b], hb.y[a:b], hb.z[a:b]], 1)
    for ax in range(3):
        c = p[:, ax]
        if c.max() - c.min() > 50:
            c[c < 50] += 100.0
    p = p - p.min(axis=0)
    return p.astype(np.float32)


def test_knn_bit_exact_vs_reference(golden, ctx):
    g = golden("knn")
    q = g["pos"].astype(np.float32)
    pos4 = np.concatenate([q, np.full((len(q), 1), 1e8, np.float32)], 1)
    near, dens = batch.knn_density(ctx, [0, len(q)], pos4, 32)
    np.testing.assert_array_equal(near.cpu().numpy(), g["idx_fixed"])
    np.testing.assert_array_equal(dens.cpu().numpy(), g["dens_fixed"])


def test_findsphdensity_dropin_bit_exact(golden, cuda_device):
    g = golden("knn")
    q = g["pos"]
    bp = np.zeros(len(q), _lib.BP_DTYPE)
    bp["x"], bp["y"], bp["z"] = q[:, 0], q[:, 1], q[:, 2]
    bp["mass"] = 1e8
    near, dens = dropin.findsphdensity(bp, 32)
    np.testing.assert_array_equal(near, g["idx_fixed"])
    np.testing.assert_array_equal(dens, g["dens_fixed"])


def test_batched_knn_vs_exact_oracle(restatement, ctx):
    """Many halos in one launch, including halos smaller than k."""
    hb = synth.catalogue(seed=91, nhalo=40, nmin=12, nmax=30000)
    pos = [_recentred_fp32(hb, h) for h in range(hb.nhalo)]
    pos4 = np.concatenate([np.concatenate([p, np.ones((len(p), 1), np.float32)], 1) for p in pos])
    k = 32
    near, dens = batch.knn_density(ctx, hb.pstart, pos4, k)
    near, dens = near.cpu().numpy(), dens.cpu().numpy()
    for h, p in enumerate(pos):
        a, b = hb.pstart[h], hb.pstart[h + 1]
        kk = min(k, len(p))
        idx, d2 = restatement.knn(p[:, 0], p[:, 1], p[:, 2], kk, "grid")
        np.testing.assert_array_equal(near[a:b, :kk], idx, err_msg=f"halo {h}")
        assert np.all(near[a:b, kk:] == -1)
        np.testing.assert_array_equal(dens[a:b], restatement.sph_density(d2), err_msg=f"halo {h}")


def test_knn_ties_broken_by_index(restatement, ctx):
    """Duplicate positions: equal distances are ordered by particle index."""
    rng = np.random.default_rng(3)
    base = rng.random((300, 3)).astype(np.float32) * 0.01
    p = np.concatenate([base, base[:150], base[:40]])  # many exact duplicates
    perm = rng.permutation(len(p))
    p = p[perm]
    pos4 = np.concatenate([p, np.ones((len(p), 1), np.float32)], 1)
    near, dens = batch.knn_density(ctx, [0, len(p)], pos4, 32)
    idx, d2 = restatement.knn(p[:, 0], p[:, 1], p[:, 2], 32, "brute")
    np.testing.assert_array_equal(near.cpu().numpy(), idx)


def test_knn_lattice_shells(restatement, ctx):
    """A cubic lattice with power-of-two spacing: every distance is exact and
    comes in shells of 6, 12, 8, ... equal distances, so the k-th place falls
    inside a tie group for almost every query (the float-key kernel cannot
    certify those and hands them to the exact kernel).  Batched with a random
    halo of the same size."""
    g = np.arange(12, dtype=np.float32) * np.float32(2.0 ** -7)
    lat = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    rng = np.random.default_rng(5)
    lat = lat[rng.permutation(len(lat))]
    rnd = (rng.random((len(lat), 3)) * 0.1).astype(np.float32)
    k = 32
    pos4 = np.concatenate([np.concatenate([p, np.ones((len(p), 1), np.float32)], 1) for p in (lat, rnd)])
    ps = [0, len(lat), 2 * len(lat)]
    near, dens = batch.knn_density(ctx, ps, pos4, k)
    near, dens = near.cpu().numpy(), dens.cpu().numpy()
    for h, p in enumerate((lat, rnd)):
        a, b = ps[h], ps[h + 1]
        idx, d2 = restatement.knn(p[:, 0], p[:, 1], p[:, 2], k, "brute")
        np.testing.assert_array_equal(near[a:b], idx, err_msg=f"halo {h}")
        np.testing.assert_array_equal(dens[a:b], restatement.sph_density(d2), err_msg=f"halo {h}")


def test_tree_structure_invariants(ctx):
    hb = synth.catalogue(seed=5, nhalo=6, nmin=100, nmax=50000)
    pos = [_recentred_fp32(hb, h) for h in range(hb.nhalo)]
    pos4 = np.concatenate([np.concatenate([p, hb.mass[hb.pstart[h]:hb.pstart[h + 1], None]
                                           .astype(np.float32)], 1) for h, p in enumerate(pos)])
    t = batch.tree_build_export(ctx, hb.pstart, pos4)
    kn, bh, tp = t["knn"], t["bh"], t["pos"]
    # the tree order is a permutation within each halo
    assert sorted(t["perm"].tolist()) == list(range(hb.n))
    for h in range(hb.nhalo):
        a, b = hb.pstart[h], hb.pstart[h + 1]
        assert np.all((t["perm"][a:b] >= a) & (t["perm"][a:b] < b))
        r, e = t["root"][h], t["rend"][h]
        assert kn[r]["skip"] == e and kn[r]["count"] == b - a and kn[r]["lstart"] == a
    np.testing.assert_array_equal(tp, pos4[t["perm"]])
    for i in range(t["nnode"]):
        s0, c = kn[i]["lstart"], kn[i]["count"]
        sub = tp[s0:s0 + c, :3]
        assert np.all(sub >= kn[i]["lo"]) and np.all(sub <= kn[i]["hi"])
        # reference node rule: every node holds at least MIN_CELL_PARTICLE_NUM particles
        # unless it is a halo root
        assert c >= 10 or i in set(t["root"].tolist())
        com = (sub.astype(np.float64) * tp[s0:s0 + c, 3:4]).sum(0) / tp[s0:s0 + c, 3].astype(np.float64).sum()
        assert np.allclose(bh[i]["com"], com, rtol=0, atol=1e-9)
