"""CPU check of the box-restricted smoothing schedule of the stage (the rule
gf_smooth.cu's smooth_box_kernel follows): with only the deposit box D
zeroed, the x pass over rows D_y x D_z reading x in D_x and writing x in E_x,
the y pass over columns E_x x D_z reading y in D_y and writing y in E_y, and
the z pass over columns E_x x E_y reading z in D_z and writing z in E_z, every
address stays inside the mesh, no unwritten cell is ever read, and the
evaluation box E (where findDen reads) holds exactly what three full passes
over a zeroed mesh give.  Pencils are filtered one at a time in FP64 (numpy
FFT), so equality is exact; tiles of P pencils are cut as the kernel cuts
them."""
import numpy as np
import pytest


def _gauss(n, rg=2.0):
    k = np.arange(n)
    ks = np.where(k > n // 2, k - n, k)
    return np.exp(-(np.pi * rg) ** 2 * ks ** 2 / n ** 2)


def _filt(v, g):
    return np.real(np.fft.ifft(np.fft.fft(v) * g))


def _boxes(near, dep):
    def rng3(sel):
        if not sel.any():
            return [1, 0, 1, 0, 1, 0]
        lo, hi = near[sel].min(0) - 1, near[sel].max(0) + 1
        return [lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]]
    return [int(v) for v in rng3(dep) + rng3(np.ones(len(near), bool))]


def _geom(axis, bx, nx, ny, mx):
    L = lambda lo, hi: hi - lo + 1 if hi >= lo else 0  # noqa: E731
    if axis == 0:
        g = (bx[2], L(bx[2], bx[3]), bx[4], L(bx[4], bx[5]), mx, mx * ny, 1, bx[0], bx[1], bx[6], bx[7])
    elif axis == 1:
        g = (bx[6], L(bx[6], bx[7]), bx[4], L(bx[4], bx[5]), 1, mx * ny, mx, bx[2], bx[3], bx[8], bx[9])
    else:
        g = (bx[6], L(bx[6], bx[7]), bx[8], L(bx[8], bx[9]), 1, mx, mx * ny, bx[4], bx[5], bx[10], bx[11])
    if bx[0] > bx[1]:
        g = (g[0], 0, g[2], 0) + g[4:]
    return g


@pytest.mark.parametrize("shape,npart,spread,dep_frac,P", [
    ((16, 16, 16), 50, 3.0, 1.0, 4),
    ((16, 12, 20), 200, 3.0, 1.0, 8),
    ((24, 16, 16), 30, 3.0, 0.0, 4),    # nothing deposited: E zeroed, no pass
    ((16, 16, 16), 300, 6.0, 0.3, 4),   # D inside a larger E
    ((20, 16, 12), 5, 0.5, 1.0, 4),
])
def test_box_passes_equal_full_passes_on_the_evaluation_box(shape, npart, spread, dep_frac, P):
    rng = np.random.default_rng(npart)
    nx, ny, nz = shape
    mx = 2 * (nx // 2 + 1)
    cells = mx * ny * nz
    pos = np.array(shape) / 2 + rng.normal(0, spread, (npart, 3))
    near = np.rint(pos).astype(int)
    near = near[np.all((near >= 1) & (near + 1 < np.array(shape)), axis=1)]
    dep = rng.random(len(near)) < dep_frac
    bx = _boxes(near, dep)
    full = np.zeros(cells)
    for p in np.nonzero(dep)[0]:
        for d in np.ndindex(3, 3, 3):
            i, j, k = near[p] + np.array(d) - 1
            full[i + mx * (j + ny * k)] += rng.random()
    new = np.full(cells, np.nan)  # never-written cells hold garbage
    o = 0 if bx[0] <= bx[1] else 6
    for z in range(bx[o + 4], bx[o + 5] + 1):
        for y in range(bx[o + 2], bx[o + 3] + 1):
            new[bx[o] + mx * (y + ny * z): bx[o + 1] + 1 + mx * (y + ny * z)] = 0.0
    new[full != 0] = full[full != 0]
    ref = full.reshape(nz, ny, mx).copy()
    ref[:, :, :nx] = np.apply_along_axis(_filt, 2, ref[:, :, :nx], _gauss(nx))
    ref[:, :, :nx] = np.apply_along_axis(_filt, 1, ref[:, :, :nx], _gauss(ny))
    ref[:, :, :nx] = np.apply_along_axis(_filt, 0, ref[:, :, :nx], _gauss(nz))
    ref = ref.ravel()
    for axis, n in ((0, nx), (1, ny), (2, nz)):
        u0, nu, v0, nv, us, vs, ss, l0, l1, s0, s1 = _geom(axis, bx, nx, ny, mx)
        for t in range((nu * nv + P - 1) // P):
            for f in range(t * P, min(t * P + P, nu * nv)):
                v, u = divmod(f, nu)
                pb = (u0 + u) * us + (v0 + v) * vs
                vec = np.zeros(n)
                for s in range(l0, l1 + 1):
                    assert 0 <= pb + s * ss < cells
                    assert not np.isnan(new[pb + s * ss]), "read a cell nothing wrote"
                    vec[s] = new[pb + s * ss]
                out = _filt(vec, _gauss(n))
                for s in range(s0, s1 + 1):
                    assert 0 <= pb + s * ss < cells
                    new[pb + s * ss] = out[s]
    E = np.array([x + mx * (y + ny * z) for z in range(bx[10], bx[11] + 1)
                  for y in range(bx[8], bx[9] + 1) for x in range(bx[6], bx[7] + 1)], int)
    assert not np.isnan(new[E]).any()
    assert np.array_equal(new[E], ref[E])
