"""The plain FP64 stage (gf_stage_run with plain_fp64): every phase in FP64,
the baseline the batched FP32 stage is compared with.  Against FP64
references on the same recentred positions: exact kNN lists from FP64
distances, mesh density of the FP64 chain (oracle/adjoint.py: TSC, spectral
smoothing, findDen in FP64), and the direct-sum potential."""
import numpy as np
import pytest
import torch

from galaxyfinder_b200 import batch, synth
from oracle import adjoint as A

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def run(cuda_device):
    hb = synth.catalogue(seed=77, nhalo=6, nmin=150, nmax=12000, straddle_frac=0.3)
    ctx = batch.Context(0)
    db = batch.DeviceBatch.from_halobatch(hb)
    cfg = batch.stage_config(plain_fp64=True)
    out, st = batch.stage_run(ctx, db, cfg, stats=True)
    cfg_direct = batch.stage_config(plain_fp64=True, ndirect=1 << 30, knn_k=0, do_mesh=False)
    out_direct = batch.stage_run(ctx, db, cfg_direct)
    torch.cuda.synchronize()
    yield dict(hb=hb, out=out, st=st, cfg=cfg, direct=out_direct, ctx=ctx, db=db)
    ctx.close()


def _pos(out):
    return np.stack([out.xr.cpu().numpy(), out.yr.cpu().numpy(), out.zr.cpu().numpy()], 1)


def test_fp64_knn_exact(run):
    hb, out = run["hb"], run["out"]
    p = _pos(out)
    near = out.nearindex.cpu().numpy()
    dens = out.dens_sph.cpu().numpy()
    for h in range(hb.nhalo):
        a, b = hb.pstart[h], hb.pstart[h + 1]
        q = p[a:b]
        n = b - a
        for i in range(0, n, max(1, n // 300)):
            d = q - q[i]
            dd = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
            o = np.lexsort((np.arange(n), dd))[:32]
            np.testing.assert_array_equal(near[a + i], o)
            # W4 density (nnost.c:536-555) in FP64 with h = r_k/2
            r = np.sqrt(dd[o])
            hk = r[-1] / 2
            u = r / hk
            w = np.where(u < 1, 1 - 1.5 * u ** 2 + 0.75 * u ** 3, np.where(u < 2, 0.25 * (2 - u) ** 3, 0.0))
            assert abs(dens[a + i] - np.sum(w) / (np.pi * hk ** 3)) <= 2e-7 * abs(dens[a + i])


def test_fp64_mesh_density(run):
    hb, out = run["hb"], run["out"]
    p = _pos(out)
    ext = np.array([p[hb.pstart[h]:hb.pstart[h + 1]].max(0) for h in range(hb.nhalo)])
    mesh, _ = batch.plan_meshes(ext, run["cfg"].mesh)
    got = out.dens_mesh.cpu().numpy().astype(np.float64)
    for h in range(hb.nhalo):
        a, b = hb.pstart[h], hb.pstart[h + 1]
        M = A.Mesh.from_desc(mesh[h])
        den = A.tsc(p[a:b], hb.mass[a:b], M)
        rho = A.find_den(p[a:b], A.smooth(den, M), M)
        # float output of FP64 arithmetic: within float rounding of the FP64 chain
        assert np.max(np.abs(got[a:b] - rho) / np.abs(rho).max()) < 1e-6, h
        pos = rho > 1e-3 * rho.max()
        assert np.max(np.abs(got[a:b][pos] - rho[pos]) / rho[pos]) < 2e-7, h


def test_fp64_potential(run):
    hb, out, dr = run["hb"], run["out"], run["direct"]
    p = _pos(out)
    raw = dr.phi.cpu().numpy().astype(np.float64)
    tree = out.phi.cpu().numpy().astype(np.float64)
    m = hb.mass.astype(np.float32).astype(np.float64)
    rng = np.random.default_rng(0)
    for h in range(hb.nhalo):
        a, b = hb.pstart[h], hb.pstart[h + 1]
        for i in rng.choice(np.arange(a, b), 20, replace=False):
            d = np.sqrt(((p[a:b] - p[i]) ** 2).sum(1))
            ok = d > 0
            want = -np.sum(m[a:b][ok] / d[ok])
            # direct sums in FP64: the float rounding of the result only
            assert abs(raw[i] - want) <= 1e-6 * abs(want)
            # the tree walk (theta2 = 0.5) within the usual Barnes-Hut error
            assert abs(tree[i] - want) <= 2e-2 * abs(want)


def test_fp64_stage_one_halo_per_call_equals_batch(run):
    """The plain path one halo per call gives the batched call's FP64 results."""
    hb, out = run["hb"], run["out"]
    ctx, db, cfg = run["ctx"], run["db"], run["cfg"]
    bufs = batch.StageBuffers(hb.n, 32, db.x.device)
    views = batch.HaloViews(db, bufs, 32, hb.pstart)
    views.run(ctx, cfg)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(bufs.nearindex.cpu().numpy(), out.nearindex.cpu().numpy())
    a, b = bufs.dens_mesh.cpu().numpy(), out.dens_mesh.cpu().numpy()
    assert np.max(np.abs(a - b) / np.abs(b).max()) < 1e-6
