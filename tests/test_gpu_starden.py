"""starfindsphdensity (NewGalFinder/nnost.c:632-744) through the drop-in
against the reference's own function (the INSERT-fixed build, compiled from
its source into oracle/_ref): stellar densities (W4 of the 10 nearest stars
times their mass, summed in float in distance order) and the 32-neighbour
lists.  Positions are rounded to float first, as in the other kNN parity
tests (the lists of the findsphdensity drop-in are exact on the float
positions; the stellar search runs in FP64 on the positions as given)."""
import numpy as np
import pytest

from galaxyfinder_b200 import _lib, dropin, synth
from oracle.oracle import Reference

pytestmark = pytest.mark.gpu


def _halo(seed, n, star_frac):
    hb = synth.catalogue(seed=seed, nhalo=1, nmin=n, nmax=n + 1)
    a, b = int(hb.pstart[0]), int(hb.pstart[1])
    p = np.stack([hb.x[a:b], hb.y[a:b], hb.z[a:b]], 1)
    p = (p - p.min(0)).astype(np.float32).astype(np.float64)  # recentred, float-representable
    rng = np.random.default_rng(seed)
    typ = np.where(rng.random(b - a) < star_frac, 1, 2).astype(np.int32)
    mass = np.where(typ == 1, 10.0 ** rng.uniform(6, 7, b - a), 1e8)
    return p, mass, typ


@pytest.mark.parametrize("seed,n,star_frac", [(5, 3000, 0.2), (6, 20000, 0.05), (7, 500, 0.01)])
def test_starfindsphdensity_matches_reference(cuda_device, seed, n, star_frac):
    p, mass, typ = _halo(seed, n, star_frac)
    bp = np.zeros(len(p), _lib.BP_DTYPE)
    bp["x"], bp["y"], bp["z"] = p[:, 0], p[:, 1], p[:, 2]
    bp["mass"], bp["type"] = mass, typ
    near, dens = dropin.starfindsphdensity(bp, 32)
    ref_near, ref_dens = Reference("fixed").starfindsphdensity(p[:, 0], p[:, 1], p[:, 2], mass, typ, 32)
    np.testing.assert_array_equal(near, ref_near)
    # the stellar lists are exact in FP64; equal distances (none in these
    # halos) would be ordered differently
    np.testing.assert_array_equal(dens, ref_dens)
    assert np.all(dens > 0)


def test_starfindsphdensity_without_stars(cuda_device):
    p, mass, _ = _halo(8, 400, 0.0)
    bp = np.zeros(len(p), _lib.BP_DTYPE)
    bp["x"], bp["y"], bp["z"] = p[:, 0], p[:, 1], p[:, 2]
    bp["mass"], bp["type"] = mass, 2
    near, dens = dropin.starfindsphdensity(bp, 32)
    assert np.all(dens == 0)
    ref_near, _ = Reference("fixed").findsphdensity(p[:, 0], p[:, 1], p[:, 2], mass, 32)
    np.testing.assert_array_equal(near, ref_near)
