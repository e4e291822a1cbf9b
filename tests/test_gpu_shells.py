"""The boundedness loop's shell step batched over its cores (gf_shell_bound)
against the reference's order, core by core through the CheckExternalTE
drop-in (tests/shell_loop.py restates subhaloden.mod6.c:3033-3101)."""
import numpy as np
import pytest

from galaxyfinder_b200 import _lib, dropin
from shell_loop import NOT_MEMBER, WP_CORE, WP_SHELL, shell_loop

pytestmark = pytest.mark.gpu


def _halo(seed=31):
    """A host and two subhaloes: particles, cores (40 most central particles of
    each clump), and four shells of the rest by a density proxy."""
    rng = np.random.default_rng(seed)
    ph = dropin.physics()
    clumps = [  # (n, sigma, centre, velocity, Rtidal)
        (6000, 0.15, (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), 0.6),
        (1500, 0.03, (1.2, 1.0, 1.0), (150.0, 0.0, 0.0), 0.09),
        (800, 0.025, (0.85, 1.1, 1.0), (0.0, -120.0, 0.0), 0.075),
    ]
    pos, vel, lab = [], [], []
    for j, (n, s, c, v, _) in enumerate(clumps):
        pe = ph["potentfact"] * n * 1e8 / s
        sv = 0.8 * np.sqrt(pe) / ph["r2kineticfact"]
        pos.append(rng.normal(c, s, (n, 3)))
        vel.append(rng.normal(v, sv, (n, 3)))
        lab.append(np.full(n, j))
    pos, vel, lab = np.concatenate(pos), np.concatenate(vel), np.concatenate(lab)
    np_ = len(pos)
    bp = np.zeros(np_, _lib.BP_DTYPE)
    bp["x"], bp["y"], bp["z"] = pos.T
    bp["vx"], bp["vy"], bp["vz"] = vel.T
    bp["mass"] = 1e8
    bp["type"] = _lib.TYPE_DM
    bp["indx"] = np.arange(np_)
    flag = np.zeros(np_, np.uint8)
    haloid = np.full(np_, NOT_MEMBER, np.int32)
    cores = np.zeros(len(clumps), _lib.CORE_DTYPE)
    for j, (n, s, c, v, rt) in enumerate(clumps):
        d = np.linalg.norm(pos - np.array(c), axis=1) + np.where(flag & WP_CORE, 1e9, 0.0)
        mem = np.argsort(d)[:40]
        flag[mem] |= WP_CORE
        haloid[mem] = j
        cores[j]["cx"], cores[j]["cy"], cores[j]["cz"] = c
        cores[j]["cvx"], cores[j]["cvy"], cores[j]["cvz"] = v
        cores[j]["Rtidal"] = rt
    dens = np.max([n * np.exp(-np.sum((pos - np.array(c)) ** 2, 1) / (2 * s * s)) / s ** 3
                   for n, s, c, _, _ in clumps], axis=0)
    rest = np.nonzero((flag & WP_CORE) == 0)[0]
    rest = rest[np.argsort(-dens[rest], kind="stable")]
    shellp = [np.sort(q).astype(np.int32) for q in np.array_split(rest, 4)]
    for q in shellp:
        flag[q] |= WP_SHELL
    shellc = [[1, 2], [1, 2, 0], [0, 1], [0]]
    return bp, flag, haloid, cores, shellp, shellc


def _order(haloid, cores_of_shell):
    nmem = {j: int(np.sum(haloid == j)) for j in cores_of_shell}
    return sorted(cores_of_shell, key=lambda j: nmem[j])


def _compare(fa, ha, fb, hb_, n):
    diff = (fa != fb) | (ha != hb_)
    # the same energy tests on octrees whose float atomics ran in another
    # order: a particle on the edge of binding may flip
    assert diff.sum() <= max(2, 2e-3 * n), diff.sum()
    return int(diff.sum())


def test_shell_bound_matches_the_core_by_core_loop(cuda_device):
    bp, flag, haloid, cores, shellp, shellc = _halo()
    n = len(bp)
    fa, ha = flag.copy(), haloid.copy()
    total_bound = 0
    for s in range(len(shellp)):
        order = _order(ha, shellc[s])
        fb, hb_ = fa.copy(), ha.copy()
        nmem_a = shell_loop(bp, fa, ha, shellp, shellc, s, cores, order)
        nmem_b, nretest = dropin.shell_bound(bp, fb, hb_, shellp, shellc, s, cores, order)
        _compare(fa, ha, fb, hb_, n)
        assert all(abs(a - b) <= max(2, 2e-3 * n) for a, b in zip(nmem_a, nmem_b)), (nmem_a, nmem_b)
        total_bound += sum(nmem_a)
    # the test is not vacuous: particles were bound and others left REMAINING
    assert total_bound > n // 10
    assert np.sum(ha == NOT_MEMBER) > n // 20


def test_shell_bound_retests_a_core_whose_count_crosses_the_direct_bound(cuda_device):
    """Core 1 (first) binds most of a shell of 1200 particles, so core 0's
    1200 candidates (the batch's count: Barnes-Hut) shrink to the few hundred
    core 1 could not reach (a direct sum when the cores run one by one):
    core 0 is retested alone with its exact targets."""
    bp, flag, haloid, cores, shellp, shellc = _halo(seed=7)
    rng = np.random.default_rng(3)
    n = len(bp)
    # one shell of 1200 particles around clump 1, inside both tidal radii
    shell = np.sort(rng.choice(np.nonzero(flag & WP_SHELL)[0], 1200, replace=False)).astype(np.int32)
    flag &= ~WP_SHELL & 0xFF
    flag[shell] |= WP_SHELL
    c1 = np.array([cores[1]["cx"], cores[1]["cy"], cores[1]["cz"]], np.float64)
    for f, ax in (("x", 0), ("y", 1), ("z", 2)):
        bp[f][shell] = c1[ax] + rng.normal(0.0, 0.02, len(shell))
    bp["vx"][shell] = cores[1]["cvx"] + rng.normal(0.0, 30.0, len(shell))
    bp["vy"][shell] = cores[1]["cvy"] + rng.normal(0.0, 30.0, len(shell))
    bp["vz"][shell] = cores[1]["cvz"] + rng.normal(0.0, 30.0, len(shell))
    core1 = np.nonzero(haloid == 1)[0]
    bp["mass"][core1] = 2e11  # a deep well: core 1 binds what its tidal radius holds
    cores[1]["Rtidal"] = 0.041  # about three quarters of the shell (2.05 sigma)
    cores[0]["Rtidal"] = 2.0
    order = [1, 0]
    fa, ha = flag.copy(), haloid.copy()
    fb, hb_ = flag.copy(), haloid.copy()
    nmem_a = shell_loop(bp, fa, ha, [shell], [[1, 0]], 0, cores, order)
    nmem_b, nretest = dropin.shell_bound(bp, fb, hb_, [shell], [[1, 0]], 0, cores, order)
    assert nmem_a[0] > 300  # core 1 bound enough of the shell to move core 0 below 1000 targets
    assert nretest >= 1
    _compare(fa, ha, fb, hb_, n)


def test_bound_pass_matches_the_core_by_core_loop(cuda_device):
    """The shells first (to give the cores members), then BOUNDITER passes,
    batched against core by core."""
    from shell_loop import bound_pass
    bp, flag, haloid, cores, shellp, shellc = _halo(seed=11)
    n = len(bp)
    bp["type"][::5] = _lib.TYPE_STAR  # CheckSelfTE centres on the list's stars
    for s in range(len(shellp)):
        shell_loop(bp, flag, haloid, shellp, shellc, s, cores, _order(haloid, shellc[s]))
    fa, ha = flag.copy(), haloid.copy()
    nbatch_total = 0
    for it in range(4):  # BOUNDITER
        counts = {j: int(np.sum(ha == j)) for j in range(len(cores))}
        order = sorted(range(len(cores)), key=lambda j: counts[j])
        nmem = [counts[j] for j in order]
        fb, hb_ = fa.copy(), ha.copy()
        nb_a = bound_pass(bp, fa, ha, cores, order, nmem)
        nb_b, nbatch = dropin.bound_pass(bp, fb, hb_, cores, order, nmem)
        _compare(fa, ha, fb, hb_, n)
        assert all(abs(a - b) <= max(2, 2e-3 * n) for a, b in zip(nb_a, nb_b)), (nb_a, nb_b)
        assert 1 <= nbatch <= len(order)
        nbatch_total += nbatch
        fa, ha = fb, hb_  # continue from the batched state
    assert np.sum(ha >= 0) > n // 10
