"""CPU: the exactness argument of the float-key kNN kernel, on its arithmetic
emulated in numpy.  The kernel keeps each query's k smallest keys
(float d^2, index), where float d^2 is evaluated from float differences of
float positions; it accepts the list only when the largest exact FP64 d^2 of
the kept particles is below frej (1 - 2e-6), frej being the smallest float
d^2 of everything not kept.  Whenever that certificate holds, the kept set
must be the exact k nearest by (FP64 d^2, index).  Checked on random clouds,
near-degenerate shells, lattices with exact ties and duplicated positions,
with both the separately rounded and the fused float evaluations."""
import numpy as np
import pytest

K = 32


def _float_d2(q, p, fused):
    d = (p - q).astype(np.float32)  # float differences of float inputs
    if not fused:
        return (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
    # fma(dx, dx, fma(dy, dy, dz*dz)): products exact in FP64, one rounding each step
    dd = d.astype(np.float64)
    inner = (dd[:, 1] * dd[:, 1] + (dd[:, 2] * dd[:, 2]).astype(np.float32)).astype(np.float32)
    return (dd[:, 0] * dd[:, 0] + inner).astype(np.float32)


def _exact_d2(q, p):
    d = p.astype(np.float64) - q.astype(np.float64)
    return (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]


def _check(points, queries, fused):
    ids = np.arange(len(points))
    certified = 0
    for qi in queries:
        q = points[qi]
        f = _float_d2(q, points, fused)
        keep = np.lexsort((ids, f))[:K]  # the k smallest (f, index)
        rest = np.setdiff1d(ids, keep)
        frej = f[rest].min() if len(rest) else np.inf
        e = _exact_d2(q, points)
        if not (e[keep].max() < np.float64(frej) * (1.0 - 2e-6)):
            continue  # the kernel hands this query to the exact kernel
        certified += 1
        exact = np.lexsort((ids, e))[:K]
        assert set(keep.tolist()) == set(exact.tolist())
    return certified


@pytest.mark.parametrize("fused", [False, True])
def test_certificate_implies_exact_lists(fused):
    rng = np.random.default_rng(1)
    cloud = (rng.random((3000, 3)) * 0.05 + 10.0).astype(np.float32)
    assert _check(cloud, rng.choice(len(cloud), 60, replace=False), fused) > 50
    # particles on thin shells around a centre: many distances agree to ~1e-7
    r = (1e-3 * (1 + 1e-7 * rng.integers(0, 4, 600))).astype(np.float64)
    v = rng.normal(size=(600, 3))
    shell = (10.0 + r[:, None] * v / np.linalg.norm(v, axis=1)[:, None]).astype(np.float32)
    shell = np.concatenate([shell, np.float32([[10.0, 10.0, 10.0]])])
    _check(shell, [len(shell) - 1] + list(rng.choice(600, 10, replace=False)), fused)
    # a lattice (exact ties in shells) and duplicated positions
    g = np.arange(8, dtype=np.float32) * np.float32(2.0 ** -7)
    lat = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    _check(lat, rng.choice(len(lat), 30, replace=False), fused)
    dup = np.concatenate([cloud[:200], cloud[:120], cloud[:40]])
    _check(dup, rng.choice(len(dup), 30, replace=False), fused)
