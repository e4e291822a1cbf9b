"""FP64 restatement of the differentiable density stage and of its gradient
(test infrastructure only; tests/ check results against it).

Everything here is plain FP64 numpy, with no float rounding anywhere, so
that central finite differences with h = 1e-6 are meaningful:

* ``tsc`` — the TSC deposit of tsc_omp2.c:166-506 (quadratic B-spline
  weights, tsc_omp2.c:335-343, times the mass, times volfact = (0.001/0.004)^3,
  tsc_omp2.c:188) into a padded mesh den[k, j, i], mx = 2(nx/2 + 1);
* ``smooth`` — gsmooth.c:14-115: multiply the 3-D r2c spectrum by
  exp(-(pi R_G / cell)^2 (kz^2/nz^2 + ky^2/ny^2 + kx^2/nx^2)) and invert,
  with R_G and R_G/cell rounded to float as the reference stores them;
* ``find_den`` — tsc_omp2.c:40-163, the TSC-weighted gather;
* ``knn_density`` — nnost.c:536-630: rho_i = sum_j W4(d_ij, r_k/2) over a
  given neighbour list (r_k = the largest distance in the list);
* ``*_grad`` — the analytic gradients of the above (product rule over the
  stencil; W4's r and h derivatives), the "plain FP64 reference gradient";
* ``fd_*`` — central finite differences of the same FP64 functions;
* ``centre_ascent`` — the gradient ascent of galaxy centres on a smoothed
  mesh, in the operation order of the GPU kernel (gf_cores.cu), so the two
  agree bit for bit on the same mesh.
"""
from __future__ import annotations

import math

import numpy as np

VOLFACT = (0.001 / 0.004) ** 3
A1, A2 = -0.2387324, 0.07957747  # AMPW41, AMPW42 (nnost.c:534-535)


class Mesh:
    def __init__(self, nx, ny, nz, xmin, ymin, zmin, cell, rg):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.mx = 2 * (self.nx // 2 + 1)
        self.o = np.array([xmin, ymin, zmin], np.float64)
        self.cell, self.rg = float(cell), float(rg)

    @classmethod
    def from_desc(cls, d):
        return cls(d["nx"], d["ny"], d["nz"], d["xmin"], d["ymin"], d["zmin"], d["cellsize"], d["rg"])

    def zeros(self):
        return np.zeros((self.nz, self.ny, self.mx), np.float64)


def _axis(pos, origin, cell):
    """Cells i0..i0+2 (i0 = nearest - 1), weights and d(weight)/d(pos)."""
    xp = (np.asarray(pos, np.float64) - origin) / cell
    nr = np.rint(xp)
    r = xp - nr
    w = np.stack([0.5 * (0.5 - r) ** 2, 0.75 - r * r, 0.5 * (0.5 + r) ** 2], -1)
    dw = np.stack([(r - 0.5) / cell, -2.0 * r / cell, (0.5 + r) / cell], -1)
    return nr.astype(np.int64) - 1, w, dw


def _stencil(pos, mesh):
    ax = [_axis(pos[:, a], mesh.o[a], mesh.cell) for a in range(3)]
    (i0, wx, dx), (j0, wy, dy), (k0, wz, dz) = ax
    for lo, n in ((i0, mesh.nx), (j0, mesh.ny), (k0, mesh.nz)):
        if np.any(lo < 0) or np.any(lo + 2 >= n):
            raise ValueError("TSC stencil outside the mesh")
    return i0, j0, k0, wx, wy, wz, dx, dy, dz


def tsc(pos, mass, mesh, select=None):
    pos = np.asarray(pos, np.float64)
    m = np.asarray(mass, np.float64)
    if select is not None:
        pos, m = pos[select], m[select]
    i0, j0, k0, wx, wy, wz, _, _, _ = _stencil(pos, mesh)
    den = mesh.zeros()
    for c in range(3):
        for b in range(3):
            for a in range(3):
                np.add.at(den, (k0 + c, j0 + b, i0 + a), VOLFACT * m * wx[:, a] * wy[:, b] * wz[:, c])
    return den


def _filter(mesh):
    kz = np.fft.fftfreq(mesh.nz) * mesh.nz
    ky = np.fft.fftfreq(mesh.ny) * mesh.ny
    kx = np.arange(mesh.nx // 2 + 1)
    # gsmooth.c:14,67: RG arrives as a float and RG/cellsize is stored in a float
    rg_cells = float(np.float32(float(np.float32(mesh.rg)) / mesh.cell))
    fac = (np.pi * rg_cells) ** 2
    return np.exp(-fac * (kz[:, None, None] ** 2 / mesh.nz ** 2 + ky[None, :, None] ** 2 / mesh.ny ** 2
                          + kx[None, None, :] ** 2 / mesh.nx ** 2))


def smooth(den, mesh):
    a = np.asarray(den, np.float64).reshape(mesh.nz, mesh.ny, mesh.mx)[:, :, :mesh.nx]
    s = np.fft.irfftn(np.fft.rfftn(a) * _filter(mesh), s=(mesh.nz, mesh.ny, mesh.nx), axes=(0, 1, 2))
    out = mesh.zeros()
    out[:, :, :mesh.nx] = s
    return out


def find_den(pos, S, mesh):
    pos = np.asarray(pos, np.float64)
    S = np.asarray(S, np.float64).reshape(mesh.nz, mesh.ny, mesh.mx)
    i0, j0, k0, wx, wy, wz, _, _, _ = _stencil(pos, mesh)
    rho = np.zeros(len(pos))
    for c in range(3):
        for b in range(3):
            for a in range(3):
                rho += S[k0 + c, j0 + b, i0 + a] * wx[:, a] * wy[:, b] * wz[:, c]
    return rho


def tsc_grad(pos, mass, mesh, G, select=None):
    """(dL/dpos (n, 3), dL/dmass (n,)) for L = <G, tsc(pos, mass)>."""
    pos = np.asarray(pos, np.float64)
    m = np.asarray(mass, np.float64)
    G = np.asarray(G, np.float64).reshape(mesh.nz, mesh.ny, mesh.mx)
    gp = np.zeros((len(pos), 3))
    gm = np.zeros(len(pos))
    idx = np.arange(len(pos)) if select is None else np.flatnonzero(select)
    i0, j0, k0, wx, wy, wz, dx, dy, dz = _stencil(pos[idx], mesh)
    for c in range(3):
        for b in range(3):
            for a in range(3):
                g = G[k0 + c, j0 + b, i0 + a]
                gm[idx] += VOLFACT * g * wx[:, a] * wy[:, b] * wz[:, c]
                gp[idx, 0] += VOLFACT * m[idx] * g * dx[:, a] * wy[:, b] * wz[:, c]
                gp[idx, 1] += VOLFACT * m[idx] * g * wx[:, a] * dy[:, b] * wz[:, c]
                gp[idx, 2] += VOLFACT * m[idx] * g * wx[:, a] * wy[:, b] * dz[:, c]
    return gp, gm


def find_den_grad(pos, S, mesh, g):
    """For L = sum_p g_p find_den(pos, S)_p: (dL/dpos at fixed S (n, 3),
    dL/dS (padded mesh))."""
    pos = np.asarray(pos, np.float64)
    g = np.asarray(g, np.float64)
    S = np.asarray(S, np.float64).reshape(mesh.nz, mesh.ny, mesh.mx)
    i0, j0, k0, wx, wy, wz, dx, dy, dz = _stencil(pos, mesh)
    gp = np.zeros((len(pos), 3))
    gS = mesh.zeros()
    for c in range(3):
        for b in range(3):
            for a in range(3):
                v = S[k0 + c, j0 + b, i0 + a]
                gp[:, 0] += g * v * dx[:, a] * wy[:, b] * wz[:, c]
                gp[:, 1] += g * v * wx[:, a] * dy[:, b] * wz[:, c]
                gp[:, 2] += g * v * wx[:, a] * wy[:, b] * dz[:, c]
                np.add.at(gS, (k0 + c, j0 + b, i0 + a), g * wx[:, a] * wy[:, b] * wz[:, c])
    return gp, gS


def w4(r, h):
    q = r / h
    out = np.where(q < 1.0, A1 * ((2.0 - q) * q * q - 1.333333) / h ** 3, 0.0)
    return np.where((q >= 1.0) & (q < 2.0), A2 * ((2.0 - q) / h) ** 3, out)


def _w4_r(r, h):
    q = r / h
    out = np.where(q < 1.0, A1 * (4.0 * q - 3.0 * q * q) / h ** 4, 0.0)
    return np.where((q >= 1.0) & (q < 2.0), -3.0 * A2 * (2.0 - q) ** 2 / h ** 4, out)


def knn_density(pos, qidx, nbr):
    """rho for queries qidx with neighbour lists nbr (nq, k) of global indices."""
    pos = np.asarray(pos, np.float64)
    d = np.linalg.norm(pos[np.asarray(qidx)][:, None, :] - pos[nbr], axis=-1)
    h = d.max(axis=1) / 2.0
    return w4(d, h[:, None]).sum(axis=1)


def knn_density_grad(pos, qidx, nbr, g=None):
    """d(sum_q g_q rho_q)/dpos, (n, 3)."""
    pos = np.asarray(pos, np.float64)
    qidx = np.asarray(qidx)
    nq, k = nbr.shape
    g = np.ones(nq) if g is None else np.asarray(g, np.float64)
    diff = pos[qidx][:, None, :] - pos[nbr]                  # (nq, k, 3)
    d = np.linalg.norm(diff, axis=-1)
    kth = np.argmax(d, axis=1)
    rk = d[np.arange(nq), kth]
    h = rk / 2.0
    w = w4(d, h[:, None])
    wr = _w4_r(d, h[:, None])
    wh = -(3.0 * w + d * wr) / h[:, None]
    with np.errstate(invalid="ignore", divide="ignore"):
        unit = np.where(d[..., None] > 0, diff / d[..., None], 0.0)
    pair = (g[:, None] * wr)[..., None] * unit                # d rho / d x_i per pair
    out = np.zeros_like(pos)
    np.add.at(out, qidx, pair.sum(axis=1))
    np.add.at(out, nbr.ravel(), -pair.reshape(-1, 3))
    dirk = diff[np.arange(nq), kth] / (2.0 * rk)[:, None]     # dh/dx_i
    hterm = (g * wh.sum(axis=1))[:, None] * dirk
    np.add.at(out, qidx, hterm)
    np.add.at(out, nbr[np.arange(nq), kth], -hterm)
    return out


def fd_mesh_term(pos, mass, mesh, G, parts, h=1e-6, select=None):
    """Central differences of L = <G, tsc(pos, mass)> for the particles
    `parts`: (len(parts), 3) position derivatives and (len(parts),) mass
    derivatives.  Only the moved particle's own 27 cells change, so each
    difference is taken over its stencil."""
    pos = np.asarray(pos, np.float64)
    m = np.asarray(mass, np.float64)
    G = np.asarray(G, np.float64).reshape(mesh.nz, mesh.ny, mesh.mx)
    sel = np.ones(len(pos), bool) if select is None else np.asarray(select, bool)

    def contrib(p, mp):
        i0, j0, k0, wx, wy, wz, _, _, _ = _stencil(p[None, :], mesh)
        tot = 0.0
        for c in range(3):
            for b in range(3):
                for a in range(3):
                    tot += G[k0[0] + c, j0[0] + b, i0[0] + a] * VOLFACT * mp * wx[0, a] * wy[0, b] * wz[0, c]
        return tot

    gp = np.zeros((len(parts), 3))
    gm = np.zeros(len(parts))
    for n, p in enumerate(parts):
        if not sel[p]:
            continue
        for a in range(3):
            e = np.zeros(3)
            e[a] = h
            gp[n, a] = (contrib(pos[p] + e, m[p]) - contrib(pos[p] - e, m[p])) / (2 * h)
        gm[n] = (contrib(pos[p], m[p] * (1 + 1e-6)) - contrib(pos[p], m[p] * (1 - 1e-6))) / (2e-6 * m[p])
    return gp, gm


def fd_knn_term(pos, qidx, nbr, parts, h=1e-6):
    """Central differences of sum_q rho_q (fixed neighbour lists) with
    respect to the positions of `parts`, with steps h and 2h.

    Returns (D_h, D_2h, kink), each (len(parts), 3).  The truncation error of
    D_h is about (D_h - D_2h)/3.  r_k is the largest distance of a list, so
    the density has a kink where the farthest neighbour changes; kink marks
    the components whose +-2h stencil crosses such a point (there a central
    difference does not estimate a derivative)."""
    pos = np.array(pos, np.float64)
    qidx = np.asarray(qidx)
    d1 = np.zeros((len(parts), 3))
    d2 = np.zeros((len(parts), 3))
    kink = np.zeros((len(parts), 3), bool)

    def far(rows):
        d = np.linalg.norm(pos[qidx[rows]][:, None, :] - pos[nbr[rows]], axis=-1)
        return np.argmax(d, axis=1)

    def total(rows):
        return knn_density(pos, qidx[rows], nbr[rows]).sum(), far(rows)

    for n, p in enumerate(parts):
        rows = np.flatnonzero((qidx == p) | np.any(nbr == p, axis=1))
        if len(rows) == 0:
            continue
        f0 = far(rows)
        for a in range(3):
            keep = pos[p, a]
            vals, crossed = {}, False
            for s in (-2, -1, 1, 2):
                pos[p, a] = keep + s * h
                vals[s], f = total(rows)
                crossed |= bool(np.any(f != f0))
            pos[p, a] = keep
            d1[n, a] = (vals[1] - vals[-1]) / (2 * h)
            d2[n, a] = (vals[2] - vals[-2]) / (4 * h)
            kink[n, a] = crossed
    return d1, d2, kink


def density_and_gradient(S, mesh, x):
    """Smoothed density at x (3,) and its gradient: FP64 TSC weights, sums in
    the order z, y, x of the 27 cells; None outside the mesh."""
    S = np.asarray(S, np.float32).reshape(mesh.nz, mesh.ny, mesh.mx)
    ax = [_axis(np.array([x[a]]), mesh.o[a], mesh.cell) for a in range(3)]
    (i0, wx, dx), (j0, wy, dy), (k0, wz, dz) = ax
    i0, j0, k0 = int(i0[0]), int(j0[0]), int(k0[0])
    if i0 < 0 or i0 + 2 >= mesh.nx or j0 < 0 or j0 + 2 >= mesh.ny or k0 < 0 or k0 + 2 >= mesh.nz:
        return None
    wx, wy, wz, dx, dy, dz = (a[0].tolist() for a in (wx, wy, wz, dx, dy, dz))
    rho = gx = gy = gz = 0.0
    for c in range(3):
        for b in range(3):
            wyz, dyz, ydz = wy[b] * wz[c], dy[b] * wz[c], wy[b] * dz[c]
            for a in range(3):
                v = float(S[k0 + c, j0 + b, i0 + a])
                rho += v * wx[a] * wyz
                gx += v * dx[a] * wyz
                gy += v * wx[a] * dyz
                gz += v * wx[a] * ydz
    return rho, gx, gy, gz


def centre_ascent(S, mesh, start, max_steps=20, step_frac=0.1):
    """(centre (3,), density, moves): up to max_steps moves of step_frac *
    R_G along the gradient; a move that does not raise the density is not
    taken and halves the step."""
    x = [float(v) for v in start]
    e = density_and_gradient(S, mesh, x)
    if e is None:
        raise ValueError("start outside the mesh")
    step = step_frac * mesh.rg
    moves = 0
    for _ in range(max_steps):
        gn = math.sqrt(e[1] * e[1] + e[2] * e[2] + e[3] * e[3])
        if not gn > 0.0:
            break
        nx = [x[a] + step * (e[1 + a] / gn) for a in range(3)]
        f = density_and_gradient(S, mesh, nx)
        if f is not None and f[0] > e[0]:
            x, e = nx, f
            moves += 1
        else:
            step *= 0.5
    return np.array(x), e[0], moves
