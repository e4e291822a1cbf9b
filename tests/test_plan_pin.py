"""The numpy mesh plan (oracle/plan.py), which the benchmark's CPU legs use so
that they never load libgf, against libgf's own host planner gf_plan_meshes:
every field identical for the three mesh rules over random extents."""
import numpy as np
import pytest

from oracle import plan as oplan


@pytest.mark.parametrize("mode,kw", [
    (oplan.MESH_POW2, dict(nmin=64, nmax=256, rg=2.0, rg_in_cells=True)),
    (oplan.MESH_REFERENCE, dict()),
    (oplan.MESH_FIXED, dict(nfixed=128, rg=2.0, rg_in_cells=True)),
])
def test_numpy_plan_equals_libgf(gf, mode, kw):
    from galaxyfinder_b200 import batch
    rng = np.random.default_rng(5 + mode)
    ext = np.exp(rng.uniform(np.log(0.02), np.log(1.5), (300, 3)))
    ext[:5] = [[0.01, 0.01, 0.01], [0.256, 0.1, 0.1], [0.216, 0.216, 0.216], [1.0, 0.5, 0.25],
               [0.9959, 0.1, 0.2]]
    if mode == oplan.MESH_REFERENCE:
        ext *= 0.3  # meshes of extent/0.004 + 10 cells stay small
    rule = batch.mesh_rule(mode=mode, **kw)
    ref, total = batch.plan_meshes(ext, rule)
    mine, mtotal = oplan.plan(ext, mode=mode, **kw)
    assert mtotal == total
    for r, m in zip(ref, mine):
        for f in ("off", "nx", "ny", "nz", "cellsize", "xmin", "rg"):
            assert r[f] == m[f], (f, r[f], m[f])
        assert r["ymin"] == m["xmin"] and r["zmin"] == m["xmin"]


def test_fftw_standin_matches_reference_smoothing():
    """The scipy.fft stand-in that times gaussian_Smoothing's FFTs in the CPU
    baseline computes the reference's smoothing (its own gsmooth.c on the
    FP64 fftw3f shim) to FP32 roundoff."""
    from oracle import fftw_standin
    from oracle.oracle import Reference
    ref = Reference("fixed")
    rng = np.random.default_rng(2)
    for nx, ny, nz in ((64, 64, 64), (40, 36, 30)):
        mx = 2 * (nx // 2 + 1)
        den = np.zeros(mx * ny * nz, np.float32)
        den.reshape(nz, ny, mx)[:, :, :nx] = rng.random((nz, ny, nx), dtype=np.float32) ** 6
        want = ref.gaussian_Smoothing(den, nx, ny, nz, 0.004, 0.008)
        got = fftw_standin.gaussian_smoothing(den.copy(), nx, ny, nz, 0.004, 0.008, workers=1)
        w = want.reshape(nz, ny, mx)[:, :, :nx]
        g = got.reshape(nz, ny, mx)[:, :, :nx]
        assert np.abs(g - w).max() < 1e-6 * np.abs(w).max()
