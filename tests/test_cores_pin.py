"""CPU: the core-finding restatement (oracle/cores.py) pinned to the
reference's own finddenpeak and FindCoreDensity (tests/golden/cores.npz, made
by the reference compiled from its sources, one thread), and the argument
checks of the new entry points (no device work)."""
import ctypes

import numpy as np
import pytest

from galaxyfinder_b200 import _lib
from oracle import cores


@pytest.fixture(scope="module")
def g(golden):
    return golden("cores")


def test_peaks_restated(g):
    nb = g["neighbor"].astype(np.int64)
    np.testing.assert_array_equal(cores.density_peaks(g["den"], nb), g["peak"])
    np.testing.assert_array_equal(cores.density_peaks(g["den"], nb, g["type"]), g["star_peak"])
    assert len(g["peak"]) > 5 and len(g["star_peak"]) > 0
    # the float copies of the peak positions and their densities
    p = g["pos"][g["peak"]].astype(np.float32)
    np.testing.assert_array_equal(g["peak_xyzd"][:, :3], p)
    np.testing.assert_array_equal(g["peak_xyzd"][:, 3], g["den"][g["peak"]])


def test_core_density_restated(g):
    out = cores.core_density(g["den"], g["neighbor"].astype(np.int64), g["type"], g["mass"], g["peak"])
    for f in ("coredensity", "nummem", "numstar", "haloid", "flag"):
        np.testing.assert_array_equal(out[f], g[f"core_{f}"], err_msg=f)
    # the reference adds star masses in float in its search order
    np.testing.assert_allclose(out["starmass"], g["core_starmass"], rtol=1e-6)
    assert (g["core_nummem"] > 0).sum() >= 5 and (g["core_haloid"] >= 0).sum() > 50


def test_core_entry_points_reject_bad_arguments():
    L = _lib.lib()
    n = ctypes.c_int32()
    assert L.gf_density_peaks(None, 10, 32, None, None, None, 2000.0, 10, None, ctypes.byref(n)) == _lib.GF_EINVAL
    assert L.gf_core_density(None, 10, 32, None, None, None, None, 1, None, None, None, None, None, None,
                             None) == _lib.GF_EINVAL


@pytest.mark.parametrize("seed,n,nsub", [(31, 2500, 3), (32, 6000, 6)])
def test_restatement_vs_reference_functions(seed, n, nsub):
    """The restatement against the reference's own finddenpeak and
    FindCoreDensity (compiled into the oracle) on more clustered halos, with
    the stellar peaks as cores too."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    from make_golden import blob
    from oracle.oracle import Reference
    ref = Reference("fixed")
    p = blob(seed, n, 0.02, nsub=nsub)
    rng = np.random.default_rng(seed)
    mass = 10 ** rng.uniform(6, 8, n)
    typ = np.where(rng.random(n) < 0.3, 1, 2).astype(np.int32)
    idx, den = ref.findsphdensity(p[:, 0], p[:, 1], p[:, 2], mass, 32)
    for jflag in (0, 1):
        pk, _ = ref.finddenpeak(den, idx, typ, p[:, 0], p[:, 1], p[:, 2], jflag)
        np.testing.assert_array_equal(cores.density_peaks(den, idx, typ if jflag else None), pk)
        want = ref.FindCoreDensity(den, idx, typ, mass, pk)
        got = cores.core_density(den, idx, typ, mass, pk)
        for f in ("coredensity", "nummem", "numstar", "haloid", "flag"):
            np.testing.assert_array_equal(got[f], want[f], err_msg=f"{f} jflag={jflag}")
        np.testing.assert_allclose(got["starmass"], want["starmass"], rtol=1e-6)
