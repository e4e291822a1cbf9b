"""Differentiable density on the GPU (galaxyfinder_b200.autograd over the
adjoint kernels of gf.h) against the FP64 restatement in oracle/adjoint.py:
the analytic FP64 gradient and FP64 central finite differences (h = 1e-6
Mpc/h).  The loss is the sum of the smoothed TSC density at the 64 highest
mesh peaks plus the kNN (k = 32) W4 density at probe particles."""
import numpy as np
import pytest
import torch

from galaxyfinder_b200 import _lib, autograd, batch, synth
from oracle import adjoint as A

pytestmark = pytest.mark.gpu


def _setup(n, nclump, mesh_n, nprobe, seed):
    hb = synth.config4(seed=seed, n=n, nclump=nclump)
    p = np.stack([hb.x, hb.y, hb.z], 1)
    p = p - p.min(0)
    ctx = batch.Context(0)
    rule = batch.mesh_rule(mode=_lib.MESH_FIXED, nfixed=mesh_n, rg=1.5, rg_in_cells=True)
    plan = autograd.MeshPlan.for_positions(ctx, [0, n], p, rule)
    rng = np.random.default_rng(seed + 1)
    probes = np.sort(rng.choice(n, nprobe, replace=False))
    dev = torch.device("cuda", 0)
    t = [torch.tensor(a, dtype=torch.float64, device=dev, requires_grad=True)
         for a in (p[:, 0], p[:, 1], p[:, 2], hb.mass)]
    return dict(p=p, mass=hb.mass, ctx=ctx, plan=plan, probes=probes, t=t, rng=rng, n=n)


def _check_loss_gradient(s, nparts):
    p, mass, plan, probes = s["p"], s["mass"], s["plan"], s["probes"]
    x, y, z, m = s["t"]
    q = torch.as_tensor(probes, device=x.device)
    loss, cells = autograd.peak_and_probe_loss(x, y, z, m, plan, q, k=32, npeak=64)
    loss.backward()
    mesh = A.Mesh.from_desc(plan.mesh[0])
    ind = mesh.zeros().ravel()
    ind[cells.cpu().numpy()] = 1.0
    G = A.smooth(ind, mesh)
    near, _ = autograd.knn_query(plan.ctx, [0, s["n"]], x.detach(), y.detach(), z.detach(), probes, 32)
    nbr = near.cpu().numpy().astype(np.int64)
    # particles to check: half among the probes' neighbours, half anywhere
    rng = s["rng"]
    parts = np.unique(np.concatenate([rng.choice(nbr.ravel(), nparts // 2, replace=False),
                                      rng.choice(s["n"], nparts // 2, replace=False)]))
    sel = np.zeros(s["n"], bool)
    sel[parts] = True
    gp_mesh, gm_mesh = A.tsc_grad(p, mass, mesh, G, select=sel)
    ref = gp_mesh[parts] + A.knn_density_grad(p, probes, nbr)[parts]
    fd_p, fd_m = A.fd_mesh_term(p, mass, mesh, G, parts)
    fd_k, fd_k2, kink = A.fd_knn_term(p, probes, nbr, parts)
    fd = fd_p + fd_k                      # central differences, h = 1e-6
    rich = fd_p + (4 * fd_k - fd_k2) / 3  # Richardson of h and 2h (the mesh term is quadratic)
    trunc = np.abs(fd_k - fd_k2) / 3      # truncation-error estimate of fd
    got = torch.stack([x.grad, y.grad, z.grad], 1).cpu().numpy()[parts]
    gotm = m.grad.cpu().numpy()[parts]
    scale = np.abs(ref).max()
    # components whose +-2h stencil changes a probe's farthest neighbour sit
    # on a kink of r_k: no derivative there, so no finite-difference check
    smooth = ~kink
    assert kink.sum() <= max(2, 0.02 * kink.size), kink.sum()
    big = smooth & (np.abs(fd) > 1e-3 * scale)
    assert big.sum() >= len(parts) // 3
    # the FP64 analytic gradient against the extrapolated differences
    assert np.abs(ref - rich)[smooth].max() <= 1e-7 * scale
    # the GPU adjoint against the FP64 analytic gradient ...
    assert np.abs(got - ref).max() <= 1e-5 * scale
    # ... against the extrapolated differences ...
    assert np.max(np.abs(got[big] - rich[big]) / np.abs(rich[big])) <= 1e-4
    # ... and against plain h = 1e-6 central differences wherever those are
    # themselves accurate (truncation estimate below 2e-5 relative)
    exact_fd = big & (trunc <= 2e-5 * np.abs(fd))
    # the counts behind these bars (shown with pytest -s)
    print(f"adjoint check: {kink.size} components, {int(kink.sum())} on a kink of r_k (excluded), "
          f"{int(big.sum())} above 1e-3 of the largest, {int(exact_fd.sum())} of those with plain h = 1e-6 "
          f"differences accurate to 2e-5; max rel err vs Richardson "
          f"{np.max(np.abs(got[big] - rich[big]) / np.abs(rich[big])):.2e}")
    assert exact_fd.sum() >= 0.5 * big.sum()
    assert np.max(np.abs(got[exact_fd] - fd[exact_fd]) / np.abs(fd[exact_fd])) <= 1e-4
    np.testing.assert_allclose(gotm, gm_mesh[parts], rtol=1e-5, atol=1e-6 * np.abs(gm_mesh[parts]).max())
    np.testing.assert_allclose(gotm, fd_m, rtol=1e-4, atol=1e-6 * np.abs(fd_m).max())
    return nbr


@pytest.fixture(scope="module")
def small(cuda_device):
    s = _setup(n=200_000, nclump=16, mesh_n=64, nprobe=512, seed=101)
    yield s
    s["ctx"].close()


def test_mesh_peaks_match_numpy(small):
    plan, x, y, z, m = small["plan"], *small["t"]
    S = plan.density_mesh(x.detach(), y.detach(), z.detach(), m.detach())
    h, c, v = plan.peaks(S, margin=1)
    mesh = A.Mesh.from_desc(plan.mesh[0])
    d = S.cpu().numpy().reshape(mesh.nz, mesh.ny, mesh.mx)[:, :, :mesh.nx]
    core = d[1:-1, 1:-1, 1:-1]
    peak = core > 0
    for dk in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for di in (-1, 0, 1):
                if dk or dj or di:
                    nb = d[1 + dk:mesh.nz - 1 + dk, 1 + dj:mesh.ny - 1 + dj, 1 + di:mesh.nx - 1 + di]
                    peak &= core > nb
    kk, jj, ii = np.nonzero(peak)
    want = np.sort((ii + 1) + mesh.mx * ((jj + 1) + mesh.ny * (kk + 1)))
    np.testing.assert_array_equal(np.sort(c), want)
    assert np.all(np.diff(v) <= 0) and np.all(h == 0)


def test_knn_query_matches_full_search(small, restatement):
    p, probes = small["p"], small["probes"]
    x, y, z, _ = small["t"]
    near, dens = autograd.knn_query(small["plan"].ctx, [0, small["n"]], x.detach(), y.detach(), z.detach(),
                                    probes, 32)
    q = p.astype(np.float32)
    idx, d2 = restatement.knn(q[:, 0], q[:, 1], q[:, 2], 32)
    np.testing.assert_array_equal(near.cpu().numpy(), idx[probes])
    np.testing.assert_array_equal(dens.cpu().numpy(), restatement.sph_density(d2)[probes])


def test_smoothing_is_self_adjoint(small):
    plan = small["plan"]
    rng = np.random.default_rng(5)
    mesh = A.Mesh.from_desc(plan.mesh[0])
    u = mesh.zeros()
    v = mesh.zeros()
    u[:, :, :mesh.nx] = rng.random((mesh.nz, mesh.ny, mesh.nx))
    v[:, :, :mesh.nx] = rng.random((mesh.nz, mesh.ny, mesh.nx))
    tu = torch.tensor(u.ravel(), dtype=torch.float32, device="cuda")
    tv = torch.tensor(v.ravel(), dtype=torch.float32, device="cuda")
    su = plan.smooth_(tu.clone()).double().cpu().numpy()
    sv = plan.smooth_(tv.clone()).double().cpu().numpy()
    a, b = np.dot(su, v.ravel()), np.dot(u.ravel(), sv)
    assert abs(a - b) <= 1e-6 * abs(a)


def test_loss_gradient_small(small):
    nbr = _check_loss_gradient(small, nparts=64)
    assert nbr.shape == (512, 32)


def test_mesh_density_at_particles_gradient(cuda_device):
    s = _setup(n=60_000, nclump=8, mesh_n=64, nprobe=8, seed=202)
    p, mass, plan = s["p"], s["mass"], s["plan"]
    x, y, z, m = s["t"]
    w = s["rng"].random(s["n"])
    rho = autograd.MeshDensityAt.apply(x, y, z, m, plan)
    (rho.double() * torch.as_tensor(w, device=x.device)).sum().backward()
    mesh = A.Mesh.from_desc(plan.mesh[0])
    S = A.smooth(A.tsc(p, mass, mesh), mesh)
    gdir, gS = A.find_den_grad(p, S, mesh, w)
    gp, gm = A.tsc_grad(p, mass, mesh, A.smooth(gS, mesh))
    ref = gdir + gp
    got = torch.stack([x.grad, y.grad, z.grad], 1).cpu().numpy()
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 1e-5 * scale
    np.testing.assert_allclose(m.grad.cpu().numpy(), gm, rtol=1e-4, atol=1e-6 * np.abs(gm).max())
    s["ctx"].close()


def test_loss_gradient_full_size(cuda_device):
    """1e7 particles in 64 clumps, 256^3 mesh, 4096 probes, FD on 256 particles."""
    s = _setup(n=10_000_000, nclump=64, mesh_n=256, nprobe=4096, seed=synth.SEED_BASE + 4)
    _check_loss_gradient(s, nparts=256)
    s["ctx"].close()
