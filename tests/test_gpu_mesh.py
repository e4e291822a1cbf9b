"""GPU parity of the mesh path (TSC deposit, Gaussian smoothing, findDen)
against the reference's own outputs (golden fixtures) and the oracle."""
import numpy as np
import pytest

from galaxyfinder_b200 import _lib, dropin

pytestmark = pytest.mark.gpu


def _bp_from(g):
    bp = np.zeros(len(g["pos"]), _lib.BP_DTYPE)
    bp["x"], bp["y"], bp["z"] = g["pos"][:, 0], g["pos"][:, 1], g["pos"][:, 2]
    bp["mass"] = g["mass"]
    bp["type"] = g["type"]
    return bp


def _logical(a, nx, ny, nz):
    mx = 2 * (nx // 2 + 1)
    return np.asarray(a).reshape(nz, ny, mx)[:, :, :nx]


@pytest.mark.parametrize("tag,ptype", [("all", 5), ("star", 1)])
def test_tsc_dropin_vs_reference(golden, cuda_device, tag, ptype):
    g = golden("mesh_chain")
    (nx, ny, nz), o, cell = g["dims"], float(g["origin"]), float(g["cell"])
    before = _lib.lib().gf_kernel_launch_count()
    den = dropin.assign_density_TSC(_bp_from(g), nx, ny, nz, o, o, o, cell, ptype)
    assert _lib.lib().gf_kernel_launch_count() > before
    ref = g[f"tsc_{tag}"]
    # identical per-particle weights; only the float summation order of the
    # contributions to a cell differs (atomics vs the reference's slab order)
    np.testing.assert_allclose(den, ref, rtol=2e-6, atol=1e-7 * ref.max())
    assert abs(den.sum(dtype=np.float64) / ref.sum(dtype=np.float64) - 1) < 1e-6


@pytest.mark.parametrize("tag", ["all", "star"])
def test_find_den_dropin_bit_exact(golden, cuda_device, tag):
    g = golden("mesh_chain")
    (nx, ny, nz), o, cell = g["dims"], float(g["origin"]), float(g["cell"])
    out = dropin.findDen(_bp_from(g), g[f"smooth_{tag}"], nx, ny, nz, o, o, o, cell)
    np.testing.assert_array_equal(out, g[f"findden_{tag}"])


@pytest.mark.parametrize("tag", ["all", "star"])
def test_smoothing_dropin_vs_reference(golden, restatement, cuda_device, tag):
    g = golden("mesh_chain")
    (nx, ny, nz), cell, rg = g["dims"], float(g["cell"]), float(g["rg"])
    den = g[f"tsc_{tag}"].copy()
    dropin.gaussian_Smoothing(den, nx, ny, nz, cell, rg)
    a, b = _logical(den, nx, ny, nz), _logical(g[f"smooth_{tag}"], nx, ny, nz)
    err = np.abs(a - b).max() / np.abs(b).max()
    assert err < 2e-6, err
    _, exact = restatement.smooth(g[f"tsc_{tag}"], nx, ny, nz, cell, rg)
    e64 = _logical(exact, nx, ny, nz)
    assert np.abs(a - e64).max() / np.abs(e64).max() < 2e-6


def test_smoothing_odd_and_prime_sizes(golden, cuda_device):
    g = golden("smooth_sizes")
    for key in [k for k in g if k.startswith("in_")]:
        a, b, c = map(int, key.split("_")[1:])
        den = g[key].copy()
        dropin.gaussian_Smoothing(den, a, b, c, 0.004, 0.006)
        x, y = _logical(den, a, b, c), _logical(g["out" + key[2:]], a, b, c)
        assert np.abs(x - y).max() / np.abs(y).max() < 2e-6, key


def test_mesh_chain_density_vs_fp64(golden, restatement, cuda_device):
    """TSC -> smoothing -> findDen on the GPU against the FP64 oracle chain:
    particle densities agree to 1e-5 relative wherever the density exceeds
    1e-3 of the halo maximum (below that FP32 rounding of the mesh dominates)."""
    g = golden("mesh_chain")
    (nx, ny, nz), o, cell, rg = g["dims"], float(g["origin"]), float(g["cell"]), float(g["rg"])
    bp = _bp_from(g)
    den = dropin.assign_density_TSC(bp, nx, ny, nz, o, o, o, cell, 5)
    dropin.gaussian_Smoothing(den, nx, ny, nz, cell, rg)
    gpu = dropin.findDen(bp, den, nx, ny, nz, o, o, o, cell)
    p = g["pos"]
    d64 = restatement.tsc(p[:, 0], p[:, 1], p[:, 2], g["mass"], g["type"], nx, ny, nz, o, o, o,
                          cell, 5, acc_double=True)
    _, s64 = restatement.smooth(d64, nx, ny, nz, cell, rg)
    ref = restatement.find_den(p[:, 0], p[:, 1], p[:, 2], s64.astype(np.float32), nx, ny, nz,
                               o, o, o, cell).astype(np.float64)
    sel = ref > 1e-3 * ref.max()
    rel = np.abs(gpu[sel] - ref[sel]) / ref[sel]
    assert rel.max() < 1e-5, rel.max()


def test_tsc_out_of_mesh_reports_range_error(cuda_device):
    bp = np.zeros(4, _lib.BP_DTYPE)
    bp["x"] = [0.01, 0.02, 0.03, 5.0]  # the last particle lies far outside a 16^3 mesh
    bp["y"] = bp["z"] = 0.02
    bp["mass"] = 1.0
    with pytest.raises(_lib.GFError) as e:
        dropin.assign_density_TSC(bp, 16, 16, 16, -0.02, -0.02, -0.02, 0.004, 5)
    assert e.value.status == _lib.GF_ERANGE


def test_batched_mesh_stage_vs_oracle(restatement, cuda_device):
    """Many halos of different sizes in one call of the batched mesh stage."""
    from galaxyfinder_b200 import batch, synth
    hb = synth.catalogue(seed=77, nhalo=12, nmin=200, nmax=20000)
    xs, ys, zs, ext = [], [], [], []
    for h in range(hb.nhalo):
        a, b = hb.pstart[h], hb.pstart[h + 1]
        p = np.stack([hb.x[a:b], hb.y[a:b], hb.z[a:b]], 1)
        for ax in range(3):  # unwrap the periodic box, then recentre (Dump2BP)
            c = p[:, ax]
            if c.max() - c.min() > 50:
                c[c < 50] += 100.0
        p = p - p.min(axis=0)
        xs.append(p[:, 0]); ys.append(p[:, 1]); zs.append(p[:, 2])
        ext.append(p.max(axis=0))
    x, y, z = map(np.concatenate, (xs, ys, zs))
    rule = batch.mesh_rule(mode=_lib.MESH_POW2, rg=2.0, rg_in_cells=True)
    mesh, total = batch.plan_meshes(np.array(ext), rule)
    ctx = batch.Context(0)
    db = batch.DeviceBatch.from_arrays(x, y, z, hb.mass, hb.type, hb.pstart)
    den, dens = batch.mesh_stage(ctx, db, mesh, total)
    den, dens = den.cpu().numpy(), dens.cpu().numpy()
    for h in range(hb.nhalo):
        a, b = hb.pstart[h], hb.pstart[h + 1]
        m = mesh[h]
        n3 = (int(m["nx"]), int(m["ny"]), int(m["nz"]))
        o, cell, rg = float(m["xmin"]), float(m["cellsize"]), float(m["rg"])
        d = restatement.tsc(x[a:b], y[a:b], z[a:b], hb.mass[a:b], hb.type[a:b], *n3, o, o, o, cell,
                            5, acc_double=True)
        sm, s64 = restatement.smooth(d, *n3, cell, rg)
        ref = restatement.find_den(x[a:b], y[a:b], z[a:b], s64.astype(np.float32), *n3, o, o, o,
                                   cell).astype(np.float64)
        got = dens[a:b]
        sel = ref > 1e-3 * ref.max()
        assert np.max(np.abs(got[sel] - ref[sel]) / ref[sel]) < 1e-5, h
        mine = den[m["off"]:m["off"] + len(sm)]
        assert np.abs(_logical(mine, *n3) - _logical(sm, *n3)).max() < 2e-6 * np.abs(sm).max()
    ctx.close()


@pytest.mark.parametrize("dims", [(64, 128, 256), (512, 16, 8), (40, 64, 512), (32, 1024, 12)])
def test_smoothing_every_fft_length_vs_fp64(restatement, cuda_device, dims):
    """Stockham radix-8/4/2 lengths 64..512, the radix-2 path (32, 1024) and
    the direct convolution (40, 12, 8...) against the FP64 spectral filter."""
    nx, ny, nz = dims
    mx = 2 * (nx // 2 + 1)
    rng = np.random.default_rng(sum(dims))
    den = np.zeros((nz, ny, mx), np.float32)
    den[:, :, :nx] = (rng.random((nz, ny, nx)) ** 6 * 1e3).astype(np.float32)
    den = den.ravel()
    _, exact = restatement.smooth(den, nx, ny, nz, 0.004, 0.008)
    got = den.copy()
    dropin.gaussian_Smoothing(got, nx, ny, nz, 0.004, 0.008)
    a, b = _logical(got, nx, ny, nz), _logical(exact, nx, ny, nz)
    assert np.abs(a - b).max() / np.abs(b).max() < 2e-6


def test_smoothing_odd_direct_axis_before_fft_axes(restatement, cuda_device):
    """A 37-cell (direct convolution) axis ahead of FFT axes: the FFT twiddle
    tables that follow an odd-length table must stay 8-byte aligned."""
    nx, ny, nz = 37, 64, 128
    mx = 2 * (nx // 2 + 1)
    rng = np.random.default_rng(5)
    den = np.zeros((nz, ny, mx), np.float32)
    den[:, :, :nx] = (rng.random((nz, ny, nx)) ** 6 * 1e3).astype(np.float32)
    den = den.ravel()
    _, exact = restatement.smooth(den, nx, ny, nz, 0.005, 0.0075)
    got = den.copy()
    dropin.gaussian_Smoothing(got, nx, ny, nz, 0.005, 0.0075)
    a, b = _logical(got, nx, ny, nz), _logical(exact, nx, ny, nz)
    assert np.abs(a - b).max() / np.abs(b).max() < 2e-6
