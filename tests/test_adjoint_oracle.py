"""CPU: the FP64 restatement of the differentiable density (oracle/adjoint.py)
checked against itself (analytic gradient vs central differences) and its
smoothing and TSC against the C restatement that is pinned to the reference
(oracle/gf_oracle.c)."""
import numpy as np

from oracle import adjoint as A


def _scene(seed=3, n=3000):
    rng = np.random.default_rng(seed)
    p = np.concatenate([0.2 + 0.02 * rng.standard_normal((n // 2, 3)),
                        0.25 + 0.03 * rng.standard_normal((n - n // 2, 3))])
    p -= p.min(0)
    mass = 10 ** rng.uniform(7, 8.5, n)
    cell = 0.006
    nmesh = int(p.max() / cell) + 12
    mesh = A.Mesh(nmesh, nmesh + 2, nmesh + 1, -5 * cell, -5 * cell, -5 * cell, cell, 1.5 * cell)
    return rng, p, mass, mesh


def test_smooth_and_tsc_match_the_c_restatement(restatement):
    rng, p, mass, mesh = _scene()
    den = A.tsc(p, mass, mesh)
    ref = restatement.tsc(p[:, 0], p[:, 1], p[:, 2], mass, np.full(len(p), 2), mesh.nx, mesh.ny, mesh.nz,
                          *mesh.o, mesh.cell, 5, acc_double=True)
    np.testing.assert_allclose(den.ravel(), ref, rtol=1e-6, atol=1e-7 * np.abs(ref).max())
    d32 = den.ravel().astype(np.float32)
    _, s64 = restatement.smooth(d32, mesh.nx, mesh.ny, mesh.nz, mesh.cell, mesh.rg)
    s = A.smooth(d32.astype(np.float64), mesh).ravel()
    assert np.abs(s - s64).max() <= 1e-12 * np.abs(s64).max()


def test_mesh_gradient_vs_central_differences():
    rng, p, mass, mesh = _scene()
    G = A.smooth(rng.random(mesh.zeros().shape), mesh)
    parts = rng.choice(len(p), 40, replace=False)
    sel = np.zeros(len(p), bool)
    sel[parts] = True
    gp, gm = A.tsc_grad(p, mass, mesh, G, select=sel)
    fp, fm = A.fd_mesh_term(p, mass, mesh, G, parts)
    assert np.abs(gp[parts] - fp).max() <= 1e-7 * np.abs(fp).max()
    np.testing.assert_allclose(gm[parts], fm, rtol=1e-8)


def test_knn_gradient_vs_central_differences():
    rng, p, _, _ = _scene(n=2000)
    q = rng.choice(len(p), 50, replace=False)
    d2 = ((p[q][:, None, :] - p[None, :, :]) ** 2).sum(-1)
    nbr = np.argsort(d2, axis=1, kind="stable")[:, :32]
    parts = np.unique(np.concatenate([q[:10], nbr[:5].ravel()]))
    g = A.knn_density_grad(p, q, nbr)
    fd, fd2, kink = A.fd_knn_term(p, q, nbr, parts)
    ok = ~kink
    assert kink.sum() <= 2
    assert np.abs(g[parts] - fd)[ok].max() <= 1e-6 * np.abs(fd).max()
    # Richardson extrapolation of the two step sizes is closer still
    rich = (4 * fd - fd2) / 3
    assert np.abs(g[parts] - rich)[ok].max() <= np.abs(g[parts] - fd)[ok].max() + 1e-9 * np.abs(fd).max()


def test_find_den_gradient_vs_central_differences():
    rng, p, mass, mesh = _scene(n=800)
    w = rng.random(len(p))
    S = A.smooth(A.tsc(p, mass, mesh), mesh)
    gdir, gS = A.find_den_grad(p, S, mesh, w)
    # at fixed S, d/dx_p of sum_q w_q rho_q is w_p * grad rho_p
    parts = rng.choice(len(p), 20, replace=False)
    h = 1e-6
    for i in parts:
        for a in range(3):
            e = np.zeros(3)
            e[a] = h
            up = A.find_den((p[i] + e)[None, :], S, mesh)[0]
            dn = A.find_den((p[i] - e)[None, :], S, mesh)[0]
            assert abs(w[i] * (up - dn) / (2 * h) - gdir[i, a]) <= 1e-6 * np.abs(gdir).max()
    # dL/dS is the transpose of the gather: <gS, S> = sum_p w_p rho_p
    assert np.isclose((gS * S).sum(), (w * A.find_den(p, S, mesh)).sum(), rtol=1e-12)
