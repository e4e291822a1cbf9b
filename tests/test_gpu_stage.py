"""The whole batched stage (gf_stage_run) on a small catalogue with periodic
straddlers, checked output by output against the oracle."""
import numpy as np
import pytest
import torch

from galaxyfinder_b200 import _lib, batch, dropin, synth
from parity import assert_final_rounding

pytestmark = pytest.mark.gpu


def _recentre(hb):
    """Dump2BP after a periodic unwrap, in numpy FP64 (same operations)."""
    xs = []
    for h in range(hb.nhalo):
        a, b = hb.pstart[h], hb.pstart[h + 1]
        p = np.stack([hb.x[a:b], hb.y[a:b], hb.z[a:b]], 1).copy()
        for ax in range(3):
            c = p[:, ax]
            cs = np.where(c < 50.0, c + 100.0, c)
            if c.max() - c.min() > 50.0 and cs.max() - cs.min() < c.max() - c.min():
                p[:, ax] = cs
        p = p - p.min(axis=0)
        xs.append(p)
    return np.concatenate(xs)


@pytest.fixture(scope="module")
def run(cuda_device):
    hb = synth.catalogue(seed=4242, nhalo=24, nmin=40, nmax=40000, straddle_frac=0.3)
    ctx = batch.Context(0)
    db = batch.DeviceBatch.from_halobatch(hb)
    cfg = batch.stage_config(count_work=True)
    out, stats = batch.stage_run(ctx, db, cfg, stats=True)
    torch.cuda.synchronize()
    t = {}
    nn = stats["nnode"]
    t["bh"] = np.zeros(nn, _lib.BH_NODE_DTYPE)
    t["pos"] = np.zeros((hb.n, 4), np.float32)
    t["root"] = np.zeros(hb.nhalo, np.int32)
    t["rend"] = np.zeros(hb.nhalo, np.int32)
    _lib.check(_lib.lib().gf_tree_export(ctx.handle, _lib.ptr(t["bh"]), None, _lib.ptr(t["pos"]),
                                         None, _lib.ptr(t["root"]), _lib.ptr(t["rend"])))
    res = dict(hb=hb, out=out, stats=stats, tree=t, cfg=cfg)
    yield res
    ctx.close()


def test_recentring_bit_exact(run):
    hb, out = run["hb"], run["out"]
    p = _recentre(hb)
    np.testing.assert_array_equal(out.xr.cpu().numpy(), p[:, 0])
    np.testing.assert_array_equal(out.yr.cpu().numpy(), p[:, 1])
    np.testing.assert_array_equal(out.zr.cpu().numpy(), p[:, 2])


def test_stage_knn_and_sph_density(run, restatement):
    hb, out = run["hb"], run["out"]
    p = _recentre(hb).astype(np.float32)
    near = out.nearindex.cpu().numpy()
    dens = out.dens_sph.cpu().numpy()
    for h in range(hb.nhalo):
        a, b = hb.pstart[h], hb.pstart[h + 1]
        kk = min(32, b - a)
        idx, d2 = restatement.knn(p[a:b, 0], p[a:b, 1], p[a:b, 2], kk)
        np.testing.assert_array_equal(near[a:b, :kk], idx)
        np.testing.assert_array_equal(dens[a:b], restatement.sph_density(d2))


def test_stage_mesh_density(run, restatement):
    hb, out = run["hb"], run["out"]
    p = _recentre(hb)
    ext = np.array([p[hb.pstart[h]:hb.pstart[h + 1]].max(0) for h in range(hb.nhalo)])
    mesh, _ = batch.plan_meshes(ext, run["cfg"].mesh)
    got = out.dens_mesh.cpu().numpy()
    beyond = total = 0
    for h in range(hb.nhalo):
        a, b = hb.pstart[h], hb.pstart[h + 1]
        m = mesh[h]
        n3 = (int(m["nx"]), int(m["ny"]), int(m["nz"]))
        o, cell, rg = float(m["xmin"]), float(m["cellsize"]), float(m["rg"])
        d = restatement.tsc(p[a:b, 0], p[a:b, 1], p[a:b, 2], hb.mass[a:b], hb.type[a:b], *n3,
                            o, o, o, cell, 5, acc_double=True)
        _, s64 = restatement.smooth(d, *n3, cell, rg)
        ref = restatement.find_den(p[a:b, 0], p[a:b, 1], p[a:b, 2], s64.astype(np.float32), *n3,
                                   o, o, o, cell).astype(np.float64)
        sel = ref > 1e-3 * ref.max()
        assert np.max(np.abs(got[a:b][sel] - ref[sel]) / ref[sel]) < 1e-5, h
        pos = ref > 0
        beyond += int(np.sum(np.abs(got[a:b][pos] - ref[pos]) > 1e-5 * ref[pos]))
        total += int(pos.sum())
    print(f"mesh density vs FP64 over all {total} particles: {beyond / total:.2e} beyond 1e-5")


def test_stage_potential_vs_fp64_same_tree(run, restatement):
    hb, out, t = run["hb"], run["out"], run["tree"]
    p = _recentre(hb).astype(np.float32)
    halo = np.repeat(np.arange(hb.nhalo), np.diff(hb.pstart))
    counts = np.diff(hb.pstart)
    topen = (counts < 100).astype(np.int32)[halo]  # Self_Halo_Potent's direct branch
    phi = restatement.tree_potential(t["bh"], t["pos"], p, t["root"][halo], t["rend"][halo], topen)
    # the raw tree potential: within 1e-6 of an FP64 walk of the same tree
    raw = out.phi.cpu().numpy().astype(np.float64)
    rel = np.abs(raw - phi) / np.abs(phi)
    assert rel.max() < 1e-6, rel.max()
    # penergy = (float)(phi * potentfact + bg): the only further error is
    # that final rounding to float (half an ulp of penergy), with bg from
    # the reference's formula
    ph = dropin.physics()
    m32 = hb.mass.astype(np.float32)
    bg = np.array([dropin.bg_potent(float(np.sum(m32[hb.pstart[h]:hb.pstart[h + 1]], dtype=np.float64)))
                   for h in range(hb.nhalo)])
    e64 = raw * ph["potentfact"] + bg[halo]
    got = out.penergy.cpu().numpy()
    assert_final_rounding(got, e64)


def test_device_background_term_vs_host(run):
    """GetBGpotent (subhaloden.mod6.c:1093-1101) as the potential kernels
    evaluate it (double) against the host's long double restatement."""
    m = np.exp(np.random.default_rng(3).uniform(np.log(1e9), np.log(1e16), 2000))
    m[:3] = [1e8 * 100, 1e8 * 131072, 2e6 * 1e8]
    md = torch.as_tensor(m, device="cuda:0")
    bg = torch.empty_like(md)
    ctx = batch.Context(0)
    _lib.check(_lib.lib().gf_bg_potent_device(ctx.handle, len(m), _lib.ptr(md), _lib.ptr(bg)))
    torch.cuda.synchronize()
    ctx.close()
    host = np.array([dropin.bg_potent(float(v)) for v in m])
    rel = np.abs(bg.cpu().numpy() - host) / np.abs(host)
    print(f"device vs host background term: max rel {rel.max():.2e}, identical {np.mean(rel == 0):.3f}")
    assert rel.max() < 1e-14


def test_stage_stats(run):
    st = run["stats"]
    assert st["nparticle"] == run["hb"].n and st["nhalo"] == run["hb"].nhalo
    assert st["pp_interactions"] > 0 and st["pc_interactions"] > 0
    assert st["mesh_cells"] > 0 and st["nnode"] > 0


def test_onchip_meshes_match_device_meshes(run):
    """The 64^3 meshes kept in a cluster's shared memory give the mesh density
    of the device-memory path (same arithmetic; float atomics sum the deposit
    in another order)."""
    hb = run["hb"]
    ctx = batch.Context(0)
    db = batch.DeviceBatch.from_halobatch(hb)
    on = batch.stage_run(ctx, db, batch.stage_config(knn_k=0, do_potential=False, mesh_onchip=True))
    off = batch.stage_run(ctx, db, batch.stage_config(knn_k=0, do_potential=False))
    torch.cuda.synchronize()
    a, b = on.dens_mesh.cpu().numpy(), off.dens_mesh.cpu().numpy()
    ps = hb.pstart
    for h in range(hb.nhalo):
        sa, sb = a[ps[h]:ps[h + 1]], b[ps[h]:ps[h + 1]]
        assert np.abs(sa - sb).max() <= 2e-6 * np.abs(sb).max(), h
    r = np.stack([on.xr.cpu().numpy(), on.yr.cpu().numpy(), on.zr.cpu().numpy()], 1)
    ext = np.array([r[ps[h]:ps[h + 1]].max(0) for h in range(hb.nhalo)])
    mesh, _ = batch.plan_meshes(ext, run["cfg"].mesh)
    n64 = int(np.sum(mesh["nx"] == 64))
    assert n64 >= 5  # the catalogue exercises the on-chip path
    ctx.close()
