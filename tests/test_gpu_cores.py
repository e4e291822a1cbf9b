"""GPU parity of core finding on the kNN graph: gf_density_peaks /
gf_core_density and the finddenpeak / FindCoreDensity drop-ins against the
reference's own functions (golden fixture; the reference compiled into the
oracle for larger halos; the reference program linked with libgf for the
drop-in that works on the reference's working-particle array).  Peaks, core
densities, member and star counts, member ids and flags are exact; star
masses agree to float rounding (the reference adds them in float in its
search order)."""
import numpy as np
import pytest
import torch

from galaxyfinder_b200 import _lib, batch, dropin, synth
from oracle import cores
from oracle.oracle import Reference

pytestmark = pytest.mark.gpu

FIELDS = ("coredensity", "nummem", "numstar", "haloid", "flag")


@pytest.fixture(scope="module")
def ctx(cuda_device):
    c = batch.Context(0)
    yield c
    c.close()


def _dev(a, dt, dev="cuda:0"):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)


def _gpu_cores(ctx, den, nb, typ, mass, peak):
    out = batch.core_density(ctx, _dev(den, torch.float32), _dev(nb, torch.int32), _dev(typ, torch.int32),
                             _dev(mass, torch.float64), _dev(peak, torch.int32))
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


def _check(got, want):
    for f in FIELDS:
        np.testing.assert_array_equal(got[f], want[f], err_msg=f)
    np.testing.assert_allclose(got["starmass"], want["starmass"], rtol=1e-6)


def test_native_vs_golden(golden, ctx):
    g = golden("cores")
    den, nb = g["den"], g["neighbor"].astype(np.int32)
    pk = batch.density_peaks(ctx, _dev(den, torch.float32), _dev(nb, torch.int32)).cpu().numpy()
    np.testing.assert_array_equal(pk, g["peak"])
    spk = batch.density_peaks(ctx, _dev(den, torch.float32), _dev(nb, torch.int32),
                              _dev(g["type"], torch.int32)).cpu().numpy()
    np.testing.assert_array_equal(spk, g["star_peak"])
    got = _gpu_cores(ctx, den, nb, g["type"], g["mass"], g["peak"])
    _check(got, {f: g[f"core_{f}"] for f in FIELDS + ("starmass",)})
    # a second call on the same context (scratch reused) gives the same
    again = _gpu_cores(ctx, den, nb, g["type"], g["mass"], g["peak"])
    for f in FIELDS + ("starmass",):
        np.testing.assert_array_equal(again[f], got[f])


def test_finddenpeak_dropin_vs_golden(golden):
    g = golden("cores")
    bp = np.zeros(len(g["den"]), _lib.BP_DTYPE)
    bp["x"], bp["y"], bp["z"] = g["pos"][:, 0], g["pos"][:, 1], g["pos"][:, 2]
    bp["mass"], bp["type"] = g["mass"], g["type"]
    nb = g["neighbor"].astype(np.int64)
    for jflag, key in ((0, "peak"), (1, "star_peak")):
        c = dropin.finddenpeak(g["den"], nb, bp, jflag)
        np.testing.assert_array_equal(c["peak"], g[key])
        xyzd = g[f"{key}_xyzd"]
        np.testing.assert_array_equal(np.stack([c["cx"], c["cy"], c["cz"], c["density"]], 1), xyzd)


def test_no_cores_and_isolated_peaks(ctx):
    rng = np.random.default_rng(4)
    n, k = 500, 8
    den = rng.uniform(1e3, 1e5, n).astype(np.float32)
    nb = np.stack([np.arange(n)] + [rng.integers(0, n, n) for _ in range(k - 1)], 1).astype(np.int32)
    got = _gpu_cores(ctx, den, nb, np.full(n, 2), np.ones(n), np.zeros(0, np.int32))
    assert np.all(got["haloid"] == cores.NOT_HALO_MEMBER) and np.all(got["flag"] == 0)
    peak = cores.density_peaks(den, nb)
    got = _gpu_cores(ctx, den, nb, np.full(n, 1), np.ones(n), peak)
    want = cores.core_density(den, nb, np.full(n, 1), np.ones(n), peak)
    _check(got, want)


@pytest.mark.parametrize("seed,ndm,nsat", [(3, 30000, 6), (5, 120000, 10)])
def test_galaxy_group_vs_reference(ctx, seed, ndm, nsat):
    """A halo with satellites: kNN lists and SPH densities from libgf (bit-exact
    with the reference's findsphdensity), then peaks and cores on the GPU
    against the reference's own finddenpeak and FindCoreDensity (one thread)."""
    ref = Reference("fixed")
    hb = synth.galaxy_group(seed=seed, ndm=ndm, nsat=nsat, star_frac=0.2)
    p = np.stack([hb.x, hb.y, hb.z], 1)
    p = (p - p.min(0)).astype(np.float32)
    pos4 = np.concatenate([p, np.ones((len(p), 1), np.float32)], 1)
    near, dens = batch.knn_density(ctx, [0, len(p)], pos4, 32)
    nb, den = near.cpu().numpy(), dens.cpu().numpy()
    q = p.astype(np.float64)
    pk0, _ = ref.finddenpeak(den, nb.astype(np.int64), hb.type, q[:, 0], q[:, 1], q[:, 2], 0)
    pk = batch.density_peaks(ctx, dens, near).cpu().numpy()
    np.testing.assert_array_equal(pk, pk0)
    want = ref.FindCoreDensity(den, nb.astype(np.int64), hb.type, hb.mass, pk0)
    got = _gpu_cores(ctx, den, nb, hb.type, hb.mass, pk0)
    _check(got, want)
    assert (want["nummem"] > 100).sum() >= nsat // 2


def test_find_core_density_dropin_inside_the_reference(golden):
    """FindCoreDensity linked into the reference program: it reads and writes
    the reference's working-particle array (wp) like the reference's own."""
    g = golden("cores")
    lnk = Reference("linked")
    got = lnk.FindCoreDensity(g["den"], g["neighbor"].astype(np.int64), g["type"], g["mass"], g["peak"])
    _check(got, {f: g[f"core_{f}"] for f in FIELDS + ("starmass",)})
