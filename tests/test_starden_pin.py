"""Pins the oracle's restatement of starfindsphdensity (NewGalFinder/nnost.c:
632-744) against the reference's own function (golden fixture made by
tests/golden/make_golden.py): the 10 nearest stars of every particle by
exact FP64 distance, W4 times the star's float mass summed in float in
distance order, and the 32-neighbour lists of all particles.  CPU only."""
import numpy as np
import pytest


def _nearest(q, c, k):
    """k nearest rows of c to every row of q: exact FP64 (dx*dx + dy*dy) + dz*dz,
    equal distances ordered by index (none occur in these inputs)."""
    d = q[:, None, :] - c[None, :, :]
    d2 = d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1] + d[..., 2] * d[..., 2]
    k = min(k, len(c))
    order = np.lexsort((np.broadcast_to(np.arange(len(c)), d2.shape), d2), axis=1)[:, :k]
    return order, np.take_along_axis(d2, order, axis=1)


@pytest.mark.parametrize("tag", ["a", "b"])
def test_star_density_bit_exact_vs_reference(golden, restatement, tag):
    g = golden("starden")
    p, mass, typ = g[f"pos_{tag}"], g[f"mass_{tag}"], g[f"type_{tag}"]
    stars = np.flatnonzero(typ == 1)
    sidx, d2 = _nearest(p, p[stars], 10)
    cnt = np.full(len(p), sidx.shape[1], np.int32)
    dens = restatement.star_density(d2, sidx, cnt, mass[stars].astype(np.float32))
    np.testing.assert_array_equal(dens, g[f"dens_{tag}"])
    assert np.all(dens > 0)
    if tag == "b":
        assert len(stars) < 10  # the list is every star


@pytest.mark.parametrize("tag", ["a", "b"])
def test_neighbour_lists_match_brute_force(golden, tag):
    g = golden("starden")
    p = g[f"pos_{tag}"]
    idx, _ = _nearest(p, p, 32)
    np.testing.assert_array_equal(idx, g[f"idx_{tag}"])
