"""The single-halo workload at full size: 131072 equal-mass particles in an
NFW halo with two subhalos, k = 32, a fixed 128^3 TSC mesh over the bounding
cube, Gaussian smoothing of 2 cells, Barnes-Hut theta^2 = 0.5.  Every output
of gf_stage_run against the oracle on the same recentred positions."""
import numpy as np
import pytest
import torch

from galaxyfinder_b200 import _lib, batch, dropin, synth
from parity import assert_final_rounding

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1(cuda_device):
    hb = synth.config1()
    ctx = batch.Context(0)
    db = batch.DeviceBatch.from_halobatch(hb)
    rule = batch.mesh_rule(mode=_lib.MESH_FIXED, nfixed=128, rg=2.0, rg_in_cells=True)
    cfg = batch.stage_config(mesh=rule, knn_k=32)
    out, st = batch.stage_run(ctx, db, cfg, stats=True)
    torch.cuda.synchronize()
    t = {"bh": np.zeros(st["nnode"], _lib.BH_NODE_DTYPE), "pos": np.zeros((hb.n, 4), np.float32),
         "root": np.zeros(1, np.int32), "rend": np.zeros(1, np.int32)}
    _lib.check(_lib.lib().gf_tree_export(ctx.handle, _lib.ptr(t["bh"]), None, _lib.ptr(t["pos"]),
                                         None, _lib.ptr(t["root"]), _lib.ptr(t["rend"])))
    p = np.stack([hb.x, hb.y, hb.z], 1)
    p = p - p.min(0)
    yield dict(hb=hb, out=out, st=st, rule=rule, p=p, tree=t)
    ctx.close()


def test_c1_recentring_and_knn_bit_exact(c1, restatement):
    out, p = c1["out"], c1["p"]
    np.testing.assert_array_equal(out.xr.cpu().numpy(), p[:, 0])
    q = p.astype(np.float32)
    idx, d2 = restatement.knn(q[:, 0], q[:, 1], q[:, 2], 32)
    np.testing.assert_array_equal(out.nearindex.cpu().numpy(), idx)
    np.testing.assert_array_equal(out.dens_sph.cpu().numpy(), restatement.sph_density(d2))


def test_c1_mesh_density(c1, restatement):
    hb, out, p = c1["hb"], c1["out"], c1["p"]
    mesh, _ = batch.plan_meshes(p.max(0)[None, :], c1["rule"])
    m = mesh[0]
    n3 = (int(m["nx"]), int(m["ny"]), int(m["nz"]))
    assert n3 == (128, 128, 128)
    o, cell, rg = float(m["xmin"]), float(m["cellsize"]), float(m["rg"])
    d = restatement.tsc(p[:, 0], p[:, 1], p[:, 2], hb.mass, hb.type, *n3, o, o, o, cell, 5,
                        acc_double=True)
    _, s64 = restatement.smooth(d, *n3, cell, rg)
    ref = restatement.find_den(p[:, 0], p[:, 1], p[:, 2], s64.astype(np.float32), *n3, o, o, o,
                               cell).astype(np.float64)
    got = out.dens_mesh.cpu().numpy()
    rel = np.abs(got - ref) / ref
    # pointwise 1e-5 wherever rho > 1e-2 rho_max
    hi = ref > 1e-2 * ref.max()
    assert hi.mean() > 0.4
    assert rel[hi].max() < 1e-5
    # between 1e-3 and 1e-2 of the maximum the FP32 FFT's roundoff (~2e-7 of
    # the mesh maximum) sets the floor: no worse than a library
    # single-precision FFT of the same FP64 mesh (pocketfft via scipy, the
    # stand-in for the reference's FFTW single precision)
    lo = (ref > 1e-3 * ref.max()) & ~hi
    lib32 = _library_fp32_smoothing(d, n3, cell, rg)
    ref_lib = restatement.find_den(p[:, 0], p[:, 1], p[:, 2], lib32, *n3, o, o, o, cell)
    rel_lib = np.abs(ref_lib.astype(np.float64) - ref) / ref
    assert rel[lo].max() <= 1.5 * rel_lib[lo].max(), (rel[lo].max(), rel_lib[lo].max())
    assert np.abs(got - ref).max() < 1e-6 * ref.max()
    # over every particle: the fraction beyond 1e-5 relative (all of them in
    # the sparse outskirts, where the FP32 mesh's absolute roundoff dominates)
    # is no larger than a library FP32 FFT's
    pos = ref > 0
    frac = np.mean(rel[pos] > 1e-5)
    frac_lib = np.mean(rel_lib[pos] > 1e-5)
    print(f"mesh density vs FP64, all {pos.sum()} particles: {frac:.2e} beyond 1e-5 "
          f"(library FP32 FFT: {frac_lib:.2e}); p99 {np.quantile(rel[pos], 0.99):.2e}")
    assert frac <= max(1.2 * frac_lib, 1e-4)


def _library_fp32_smoothing(d, n3, cell, rg):
    import scipy.fft as sf
    nx, ny, nz = n3
    mx = 2 * (nx // 2 + 1)
    a = np.asarray(d, np.float32).reshape(nz, ny, mx)[:, :, :nx]
    kz, ky = np.fft.fftfreq(nz) * nz, np.fft.fftfreq(ny) * ny
    kx = np.arange(nx // 2 + 1)
    fac = (np.pi * float(np.float32(float(np.float32(rg)) / cell))) ** 2  # gsmooth.c:14,67
    filt = np.exp(-fac * (kz[:, None, None] ** 2 / nz ** 2 + ky[None, :, None] ** 2 / ny ** 2
                          + kx[None, None, :] ** 2 / nx ** 2)).astype(np.float32)
    s = sf.irfftn(sf.rfftn(a) * filt, s=(nz, ny, nx), axes=(0, 1, 2)).astype(np.float32)
    full = np.zeros((nz, ny, mx), np.float32)
    full[:, :, :nx] = s
    return full.ravel()


def test_c1_potential(c1, restatement):
    out, p, t = c1["out"], c1["p"], c1["tree"]
    n = len(p)
    phi = restatement.tree_potential(t["bh"], t["pos"], p.astype(np.float32),
                                     np.zeros(n, np.int32) + t["root"][0],
                                     np.zeros(n, np.int32) + t["rend"][0], None)
    raw = out.phi.cpu().numpy().astype(np.float64)
    rel = np.abs(raw - phi) / np.abs(phi)
    print(f"raw potential vs FP64 walk of the same tree: max rel {rel.max():.2e}, "
          f"median {np.median(rel):.2e}")
    assert rel.max() < 1e-6, rel.max()
    ph = dropin.physics()
    m32 = c1["hb"].mass.astype(np.float32)
    bg = dropin.bg_potent(float(np.sum(m32, dtype=np.float64)))
    assert_final_rounding(out.penergy.cpu().numpy(), raw * ph["potentfact"] + bg)
