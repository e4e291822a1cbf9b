"""GPU parity of the Barnes-Hut potential: against an FP64 walk of the same
tree (<= 1e-6 relative), against FP64 direct sums, and against the
reference's own treeplumpotential / Self_Halo_Potent / External_Halo_Potent
(golden fixtures)."""
import numpy as np
import pytest

from galaxyfinder_b200 import batch, dropin, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(cuda_device):
    c = batch.Context(0)
    yield c
    c.close()


def _halos(seed, nhalo, nmin, nmax):
    hb = synth.catalogue(seed=seed, nhalo=nhalo, nmin=nmin, nmax=nmax)
    out = []
    for h in range(hb.nhalo):
        a, b = hb.pstart[h], hb.pstart[h + 1]
        p = np.stack([hb.x[a:b], hb.y[a:b], hb.z[a:b]], 1)
        for ax in range(3):
            c = p[:, ax]
            if c.max() - c.min() > 50:
                c[c < 50] += 100.0
        p = p - p.min(axis=0)
        out.append(np.concatenate([p, hb.mass[a:b, None]], 1).astype(np.float32))
    return hb, np.concatenate(out)


@pytest.mark.parametrize("theta2", [0.5, 0.25])
def test_potential_vs_fp64_same_tree(restatement, ctx, theta2):
    hb, pos4 = _halos(17, 10, 200, 40000)
    t = batch.tree_build_export(ctx, hb.pstart, pos4, theta2=theta2)
    _, raw = batch.self_potential(ctx, hb.pstart, pos4, theta2=theta2)
    raw = raw.cpu().numpy().astype(np.float64)
    # targets in batch order: tree position of batch particle i
    inv = np.empty_like(t["perm"])
    inv[t["perm"]] = np.arange(len(inv))
    halo = np.repeat(np.arange(hb.nhalo), np.diff(hb.pstart))
    phi = restatement.tree_potential(t["bh"], t["pos"], pos4[:, :3], t["root"][halo],
                                     t["rend"][halo])
    rel = np.abs(raw - phi) / np.abs(phi)
    assert rel.max() < 1e-6, rel.max()


def test_potential_small_theta_equals_direct_sum(restatement, ctx):
    hb, pos4 = _halos(23, 3, 300, 3000)
    _, raw = batch.self_potential(ctx, hb.pstart, pos4, theta2=1e-8)
    raw = raw.cpu().numpy().astype(np.float64)
    for h in range(hb.nhalo):
        a, b = hb.pstart[h], hb.pstart[h + 1]
        d = restatement.direct_potential(pos4[a:b], pos4[a:b, :3])
        assert np.max(np.abs(raw[a:b] - d) / np.abs(d)) < 1e-6


def test_direct_threshold_matches_direct_sum(restatement, ctx):
    """Halos below ndirect members are summed directly (Self_Halo_Potent, np < 100)."""
    hb, pos4 = _halos(29, 8, 20, 99)
    _, raw = batch.self_potential(ctx, hb.pstart, pos4, theta2=0.5, ndirect=100)
    raw = raw.cpu().numpy().astype(np.float64)
    for h in range(hb.nhalo):
        a, b = hb.pstart[h], hb.pstart[h + 1]
        d = restatement.direct_potential(pos4[a:b], pos4[a:b, :3])
        assert np.max(np.abs(raw[a:b] - d) / np.abs(d)) < 1e-6


def _errors(x, exact):
    e = np.abs(np.asarray(x, np.float64) - exact) / np.abs(exact)
    return e.mean(), np.median(e)


def test_tree_potential_vs_reference_treeplumpotential(golden, restatement, ctx):
    """Same tree rules as ost.c.  The reference adds its spline-table and float
    accumulation error and the q5 moment defect (ost.c:571); both are
    Barnes-Hut approximations of the FP64 direct sum, and ours must be at
    least as close to it as the reference's."""
    g = golden("potential")
    r = g["pos"].astype(np.float32)
    pos4 = np.concatenate([r, g["mass"][:, None]], 1)
    _, raw = batch.self_potential(ctx, [0, len(r)], pos4, theta2=0.5)
    direct = restatement.direct_potential(pos4, r)
    ours, ref = _errors(raw.cpu().numpy(), direct), _errors(g["phi_tree"], direct)
    assert ours[0] <= ref[0] and ours[1] <= ref[1], (ours, ref)


def _penergy_direct(restatement, r, m, targets):
    pos4 = np.concatenate([r.astype(np.float32), m[:, None].astype(np.float32)], 1)
    d = restatement.direct_potential(pos4, targets.astype(np.float32))
    ph = dropin.physics()
    return d * ph["potentfact"] + dropin.bg_potent(float(np.sum(m, dtype=np.float64)))


def test_self_halo_potent_dropin(golden, restatement, cuda_device):
    g = golden("potential")
    r, m = g["pos"], g["mass"]
    pe = dropin.Self_Halo_Potent(r, m)
    exact = _penergy_direct(restatement, r, m, r)
    ours, ref = _errors(pe, exact), _errors(g["self_pe"], exact)
    assert ours[0] <= ref[0] and ours[1] <= ref[1], (ours, ref)
    # below 100 members both sum directly: agreement to float rounding
    pe_small = dropin.Self_Halo_Potent(r[:80], m[:80])
    np.testing.assert_allclose(pe_small, g["self_small"], rtol=2e-6)
    exact_small = _penergy_direct(restatement, r[:80], m[:80], r[:80])
    np.testing.assert_allclose(pe_small, exact_small, rtol=1e-6)


def test_external_halo_potent_dropin(golden, restatement, cuda_device):
    g = golden("potential")
    r, m = g["pos"], g["mass"]
    tgt = r[::3][:1500]
    pe = dropin.External_Halo_Potent(tgt, m[::3][:1500], r, m)
    exact = _penergy_direct(restatement, r, m, tgt)
    ours, ref = _errors(pe, exact), _errors(g["ext_pe"], exact)
    assert ours[0] <= ref[0] and ours[1] <= ref[1], (ours, ref)
    # fewer than 1000 targets: direct sum (subhaloden.mod6.c:1545)
    pe_small = dropin.External_Halo_Potent(tgt[:500], m[:500], r, m)
    np.testing.assert_allclose(pe_small, exact[:500], rtol=1e-6)
