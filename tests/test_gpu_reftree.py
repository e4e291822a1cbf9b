"""The reference's per-particle tree API on the GPU: new_Make_Tree_Near +
Find_Near (NewGalFinder/nnost.c:199,375) and Make_Tree + treeplumpotential
(ost.c:642,226), called through libgf's C ABI with the reference's own
TStruct/TPtlStruct/particle layouts.

* Find_Near against the reference's own Find_Near on its own tree (the oracle
  build with the INSERT bound fixed): identical squared distances, identical
  indices wherever a row has no tied distances.
* The tree libgf writes is a valid tree in the reference's layout: every
  particle threaded once, node sizes bounding their particles, and the
  reference's own Find_Near and treeplumpotential walking it give the exact
  neighbours and the reference's potential.
* treeplumpotential agrees with libgf's batched self potential of the same
  particles (the same build and walk), and is closer to an FP64 direct sum
  than the reference's spline-table walk.
* Points that are not particles of the tree, many threads at once, and a tree
  built by the reference's own code."""
import ctypes
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from galaxyfinder_b200 import _lib, batch, synth

pytestmark = pytest.mark.gpu

K = 32


def _halo(n=20000, seed=3):
    hb = synth.config1(n=n, seed=seed)
    p = np.stack([hb.x, hb.y, hb.z], 1)
    p = p - p.min(0)
    p[-40:] = p[:40]  # exact duplicates: ties at equal distance
    return p, hb.mass.copy()


def _ptl(p, m):
    ptl = np.zeros(len(p), _lib.TPTL_DTYPE)
    ptl["x"], ptl["y"], ptl["z"], ptl["mass"] = p[:, 0], p[:, 1], p[:, 2], m
    ptl["indx"] = np.arange(len(p))
    return ptl


def _points(p):
    pt = np.zeros(len(p), _lib.PARTICLE_DTYPE)
    pt["x"], pt["y"], pt["z"] = p[:, 0], p[:, 1], p[:, 2]
    return pt


def _addr(a, i=0):
    return ctypes.c_void_p(int(a.ctypes.data) + int(i) * a.dtype.itemsize)


def _find_near(fn, pts, T, ptl, i, k=K):
    idx = np.zeros(k, np.int64)
    d2 = np.zeros(k, np.float64)
    mass = np.zeros(k, np.float32)
    maxr = ctypes.c_float()
    n = fn(_addr(pts, i), k, _addr(T), _addr(ptl), ctypes.byref(maxr), _addr(idx), _addr(d2), _addr(mass))
    return n, idx[:n], d2[:n], mass[:n], maxr.value


def _ref_lib():
    from oracle.oracle import Reference
    ref = Reference("fixed")
    L = ref.L
    L.Find_Near.restype = ctypes.c_int
    L.Find_Near.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 6
    L.treeplumpotential.restype = ctypes.c_float
    L.treeplumpotential.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p]
    L.new_Make_Tree_Near.restype = None
    L.new_Make_Tree_Near.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                                     ctypes.c_int]
    return ref


def _walk(T, ptl):
    """Follows the threads of an exported tree: every particle once, node by node."""
    tb, pb = T.ctypes.data, ptl.ctypes.data
    seen = np.zeros(len(ptl), np.int32)
    ptr, steps = tb, 0
    while ptr:
        steps += 1
        assert steps < 10 * (len(ptl) + len(T))
        if tb <= ptr < tb + T.nbytes:
            i = (ptr - tb) // T.dtype.itemsize
            assert T[i]["type"] == 0
            ptr = int(T[i]["daughter"])
        else:
            j = (ptr - pb) // ptl.dtype.itemsize
            assert 0 <= j < len(ptl) and ptl[j]["type"] == 1
            seen[j] += 1
            ptr = int(ptl[j]["sibling"])
    return seen


def _row_equal(ia, da, ib, db):
    """Same squared distances; the same indices at every distance, except in a
    group of tied distances that the k-th place cuts (the reference keeps its
    walk order among equals, libgf the index order)."""
    np.testing.assert_array_equal(da, db)
    for v in np.unique(da):
        sel = da == v
        if v == da[-1]:
            continue
        assert set(ia[sel]) == set(ib[sel])


@pytest.fixture(scope="module")
def tree(cuda_device):
    p, m = _halo()
    ptl = _ptl(p, m)
    T = np.zeros(len(p), _lib.TSTRUCT_DTYPE)
    _lib.lib().new_Make_Tree_Near(_addr(T), len(T), _addr(ptl), len(ptl), 1)
    assert _lib.lib().gf_last_status() == 0, _lib.lib().gf_last_error()
    return dict(p=p, m=m, ptl=ptl, T=T, pts=_points(p))


def test_exported_tree_is_threaded_in_the_reference_layout(tree):
    T, ptl, p = tree["T"], tree["ptl"], tree["p"]
    assert np.all(_walk(T, ptl) == 1)
    nn = int(np.count_nonzero(T["Nparticle"]))
    assert T[0]["Nparticle"] == len(p) and T[0]["sibling"] == 0
    # node sizes bound their particles: check the root and a sample of nodes
    com = np.array([T[0]["monox"], T[0]["monoy"], T[0]["monoz"]])
    assert np.sqrt(((p - com) ** 2).sum(1)).max() <= T[0]["dist"] * (1 + 1e-15)
    assert abs(T[0]["mass"] - np.sum(tree["m"].astype(np.float32), dtype=np.float64)) <= 1e-12 * T[0]["mass"]
    assert nn > len(p) / 40


def test_find_near_matches_the_reference(tree):
    ref = _ref_lib()
    p, m = tree["p"], tree["m"]
    ridx, rd2, rmaxr = ref.find_near_all(p[:, 0], p[:, 1], p[:, 2], m, K)
    fn = _lib.lib().Find_Near
    for i in range(len(p)):
        n, idx, d2, mass, maxr = _find_near(fn, tree["pts"], tree["T"], tree["ptl"], i)
        assert n == K
        _row_equal(idx, d2, ridx[i], rd2[i])
        assert maxr == rmaxr[i]
        np.testing.assert_array_equal(mass, m[idx].astype(np.float32))


def test_reference_walks_the_exported_tree(tree):
    """The reference's own Find_Near on the tree libgf wrote."""
    ref = _ref_lib()
    fn = _lib.lib().Find_Near
    rng = np.random.default_rng(1)
    for i in rng.choice(len(tree["p"]), 500, replace=False):
        n, idx, d2, _, _ = _find_near(fn, tree["pts"], tree["T"], tree["ptl"], i)
        rn, ridx, rd2, _, _ = _find_near(ref.L.Find_Near, tree["pts"], tree["T"], tree["ptl"], i)
        assert rn == n
        _row_equal(idx, d2, ridx, rd2)


def test_find_near_off_particle_points_and_threads(tree):
    p, T, ptl = tree["p"], tree["T"], tree["ptl"]
    fn = _lib.lib().Find_Near
    rng = np.random.default_rng(2)
    q = p[rng.choice(len(p), 64)] + rng.normal(0, 1e-3, (64, 3))
    qp = _points(q)
    for i in range(len(q)):
        n, idx, d2, _, _ = _find_near(fn, qp, T, ptl, i)
        d = p - q[i]
        dd = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        o = np.lexsort((np.arange(len(p)), dd))[:K]
        np.testing.assert_array_equal(idx, o)
        np.testing.assert_array_equal(d2, dd[o])
    # many threads at once (ctypes releases the GIL): the same rows
    rows = list(range(0, len(p), 7))
    with ThreadPoolExecutor(8) as ex:
        got = list(ex.map(lambda i: _find_near(fn, tree["pts"], T, ptl, i), rows))
    for i, g in zip(rows, got):
        want = _find_near(fn, tree["pts"], T, ptl, i)
        np.testing.assert_array_equal(g[1], want[1])
        np.testing.assert_array_equal(g[2], want[2])


def test_find_near_on_a_tree_built_by_the_reference(tree):
    ref = _ref_lib()
    p, m = tree["p"][:3000], tree["m"][:3000]
    ptl = _ptl(p, m)
    T = np.zeros(4000, _lib.TSTRUCT_DTYPE)
    ref.L.new_Make_Tree_Near(_addr(T), len(T), _addr(ptl), len(ptl), 1)
    pts = _points(p)
    fn = _lib.lib().Find_Near
    for i in range(0, len(p), 11):
        n, idx, d2, _, _ = _find_near(fn, pts, T, ptl, i)
        rn, ridx, rd2, _, _ = _find_near(ref.L.Find_Near, pts, T, ptl, i)
        assert n == rn
        _row_equal(idx, d2, ridx, rd2)


def test_make_tree_and_treeplumpotential(cuda_device):
    ref = _ref_lib()
    p, m = _halo(n=30000, seed=5)
    ptl = _ptl(p, m)
    T = np.zeros(len(p), _lib.TSTRUCT_DTYPE)
    L = _lib.lib()
    L.Make_Tree(_addr(T), len(T), _addr(ptl), len(ptl), 0.5, 1)
    assert L.gf_last_status() == 0, L.gf_last_error()
    assert np.all(_walk(T, ptl) == 1)
    nn = int(np.count_nonzero(T["Nparticle"]))
    np.testing.assert_array_equal(T["dist_over_thetasq"][:nn], T["dist2"][:nn] / 0.5)
    pts = _points(p)
    phi = np.array([L.treeplumpotential(_addr(pts, i), 0.5, _addr(T), _addr(ptl)) for i in range(len(p))],
                   np.float32)
    # the batched self potential of the same FP32 particles: the same build
    # and walk (a centre of mass summed by FP64 atomics in another order may
    # move an opening decision of a rare particle)
    pos4 = np.concatenate([p.astype(np.float32), m.astype(np.float32)[:, None]], 1)
    ctx = batch.Context(0)
    _, raw = batch.self_potential(ctx, [0, len(p)], pos4, theta2=0.5, ndirect=0)
    raw = raw.cpu().numpy().astype(np.float64)
    rel = np.abs(phi - raw) / np.abs(raw)
    assert np.mean(rel <= 1e-6) > 0.999 and rel.max() < 2e-3, (np.mean(rel <= 1e-6), rel.max())
    # the reference's own walk (spline tables) on the tree libgf wrote, and
    # both against an FP64 direct sum
    rng = np.random.default_rng(4)
    sel = rng.choice(len(p), 200, replace=False)
    rphi = np.array([ref.L.treeplumpotential(_addr(pts, i), 0.5, _addr(T), _addr(ptl)) for i in sel])
    direct = np.array([-np.sum(m[np.arange(len(p)) != i] / np.sqrt(((p[np.arange(len(p)) != i] - p[i]) ** 2).sum(1)))
                       for i in sel])
    e_gf = np.abs(phi[sel] - direct) / np.abs(direct)
    e_ref = np.abs(rphi - direct) / np.abs(direct)
    print(f"treeplumpotential vs FP64 direct: libgf mean {e_gf.mean():.2e} max {e_gf.max():.2e}; "
          f"reference on the same tree mean {e_ref.mean():.2e} max {e_ref.max():.2e}")
    assert np.abs(rphi - phi[sel]).max() < 3e-3 * np.abs(phi[sel]).max()
    assert e_gf.mean() <= e_ref.mean()
    # a point that is not a particle of the tree: one-point launch
    q = _points(p[:1] + 1e-3)
    v = L.treeplumpotential(_addr(q), 0.5, _addr(T), _addr(ptl))
    d = np.sqrt(((p - (p[0] + 1e-3)) ** 2).sum(1))
    assert abs(v - (-np.sum(m / d))) < 1e-2 * abs(v)
    ctx.close()
