"""Boundedness test (CheckSelfTE / CheckExternalTE), tidal radius
(AdGetTidalRCenterCore) and tidal cut on the GPU, against the reference's own
outputs in tests/golden/bound.npz and against numpy restatements of the
reference's float/double arithmetic (subhaloden.mod6.c)."""
import numpy as np
import pytest

from galaxyfinder_b200 import _lib, dropin
from oracle import bound
from oracle.bound import kinetic, star_centre

pytestmark = pytest.mark.gpu


def to_bp(pos, mass=None, typ=None):
    bp = np.zeros(len(pos), _lib.BP_DTYPE)
    bp["x"], bp["y"], bp["z"] = pos[:, 0], pos[:, 1], pos[:, 2]
    bp["mass"] = 1.0 if mass is None else mass
    bp["type"] = _lib.TYPE_DM if typ is None else typ
    return bp


def self_te(pos, vel, mass, typ):
    bp = to_bp(pos, mass, typ)
    kp = dropin.make_kp(pos[:, 0], pos[:, 1], pos[:, 2], vel[:, 0], vel[:, 1], vel[:, 2], mass, bp)
    flags, nb = dropin.CheckSelfTE(kp, bp)
    return flags, nb


def check_against(flags, ref_flags, ke, pe_ours, pe_ref, max_frac=0.02):
    """Flags equal the reference's wherever the two potentials put the
    particle on the same side; a flip needs ke between -pe_ours and -pe_ref."""
    diff = flags != ref_flags
    lo = np.minimum(-pe_ours, -pe_ref).astype(np.float64)
    hi = np.maximum(-pe_ours, -pe_ref).astype(np.float64)
    k = ke.astype(np.float64)
    assert np.all((k[diff] >= lo[diff]) & (k[diff] <= hi[diff]))
    assert diff.mean() <= max_frac, diff.mean()


def test_check_self_te(cuda_device, golden):
    g = golden("bound")
    ph = dropin.physics()
    pos, vel, mass, typ = g["pos"], g["vel"], g["mass"], g["type"]
    flags, nb = self_te(pos, vel, mass, typ)
    pe = dropin.Self_Halo_Potent(pos, mass)
    ke = kinetic(pos, vel, star_centre(pos, vel, mass, typ), ph["r1kineticfact"], ph["r2kineticfact"])
    # the rule itself, bit for bit, on this library's own potential
    expect = np.where(ke > -pe, _lib.GF_UNBOUND, _lib.GF_BOUND)
    np.testing.assert_array_equal(flags, expect)
    assert nb == int(np.sum(flags == _lib.GF_BOUND))
    check_against(flags, g["self_flag"], ke, pe, g["self_pe"])
    assert abs(nb - int(g["self_nb"])) <= 0.02 * len(pos)


def test_check_self_te_direct_and_no_stars(cuda_device, golden):
    g = golden("bound")
    ph = dropin.physics()
    pos, mass, typ = g["pos"][:70], g["mass"][:70], g["type"][:70]
    vel = g["small_vel"]
    flags, nb = self_te(pos, vel, mass, typ)
    pe = dropin.Self_Halo_Potent(pos, mass)
    ke = kinetic(pos, vel, star_centre(pos, vel, mass, typ), ph["r1kineticfact"], ph["r2kineticfact"])
    np.testing.assert_array_equal(flags, np.where(ke > -pe, _lib.GF_UNBOUND, _lib.GF_BOUND))
    check_against(flags, g["small_flag"], ke, pe, g["small_pe"], max_frac=0.05)
    # no stars: the reference's centre is 0/0, every comparison is false, all bound
    flags, nb = self_te(pos, vel, mass, np.full(70, _lib.TYPE_DM, np.int32))
    np.testing.assert_array_equal(flags, g["nostar_flag"])
    assert nb == int(g["nostar_nb"]) == 70


def test_check_external_te(cuda_device, golden):
    g = golden("bound")
    ph = dropin.physics()
    tpos, tvel, tmass = g["ext_pos"], g["ext_vel"], g["ext_mass"]
    spos, smass, c6 = g["pos"], g["mass"], g["ext_core"]
    tkp = dropin.make_kp(tpos[:, 0], tpos[:, 1], tpos[:, 2], tvel[:, 0], tvel[:, 1], tvel[:, 2], tmass)
    z = np.zeros(len(spos), np.float32)
    skp = dropin.make_kp(spos[:, 0], spos[:, 1], spos[:, 2], z, z, z, smass)
    core = np.zeros(1, _lib.CORE_DTYPE)
    for f, v in zip(("cx", "cy", "cz", "cvx", "cvy", "cvz"), c6):
        core[f] = v
    flags, nb = dropin.CheckExternalTE(tkp, skp, core)
    pe = dropin.External_Halo_Potent(tpos, tmass, spos, smass)
    ke = kinetic(tpos, tvel, c6.astype(np.float64), ph["r1kineticfact"], ph["r2kineticfact"])
    np.testing.assert_array_equal(flags, np.where(ke > -pe, _lib.GF_UNBOUND, _lib.GF_BOUND))
    assert nb == int(np.sum(flags == _lib.GF_BOUND))
    check_against(flags, g["ext_flag"], ke, pe, g["ext_pe"])


def test_tidal_radius_bit_exact(cuda_device, golden):
    g = golden("bound")
    c6 = g["tid_core"]
    core = np.zeros(len(c6), _lib.CORE_DTYPE)
    for k, f in enumerate(("cx", "cy", "cz", "cvx", "cvy", "cvz")):
        core[f] = c6[:, k]
    bp = to_bp(g["tid_pos"], g["tid_mass"])
    dropin.tidal_radius(core, g["tid_score"], bp, g["tid_haloid"])
    np.testing.assert_array_equal(core["Rtidal"], g["tid_rtidal"])
    np.testing.assert_array_equal(core["nummem"], g["tid_nummem"])
    # every branch of :1956-2029 is reached by this scene
    rt = g["tid_rtidal"]
    assert np.any(rt == np.float32(2e5)) and np.any(rt == 0) and np.all(np.isfinite(rt))


def test_tidal_radius_many_cores(cuda_device):
    """Two hundred cores (about 20k pairs, more than resident warps), against
    the restatement bit for bit on every branch."""
    rng = np.random.default_rng(7)
    ncore = 200
    sizes = rng.integers(0, 400, ncore)
    sizes[:3] = 0
    ctr = rng.random((ncore, 3)) * 0.6
    pos = np.concatenate([c + 0.03 * rng.standard_normal((n, 3)) for c, n in zip(ctr, sizes)])
    hid = np.repeat(np.arange(ncore, dtype=np.int32), sizes)
    perm = rng.permutation(len(pos))
    pos, hid = pos[perm], hid[perm]
    hid[rng.random(len(hid)) < 0.05] = -1
    mass = 10 ** rng.uniform(7, 8.5, len(pos))
    c6 = np.zeros((ncore, 6), np.float32)
    c6[:, :3] = ctr
    c6[:, 3:] = 40 * rng.standard_normal((ncore, 3))
    core = np.zeros(ncore, _lib.CORE_DTYPE)
    for k, f in enumerate(("cx", "cy", "cz", "cvx", "cvy", "cvz")):
        core[f] = c6[:, k]
    score = np.argsort(sizes, kind="stable").astype(np.int32)
    dropin.tidal_radius(core, score, to_bp(pos, mass), hid)
    ph = dropin.physics()
    rt, nm = bound.tidal_radius(c6, score, pos, mass, hid, ph["r2kineticfact"], ph["potentfact"])
    np.testing.assert_array_equal(core["nummem"], nm)
    np.testing.assert_array_equal(core["Rtidal"], rt)
    assert np.any(rt == 0) and np.any(rt == np.float32(2e5)) and len(np.unique(rt)) > ncore // 2


def test_tidal_select(cuda_device):
    rng = np.random.default_rng(9)
    pos = rng.random((50000, 3)) * 0.4
    bp = to_bp(pos)
    c = np.array([0.21, 0.19, 0.2], np.float32)
    rt = np.float32(0.07)

    got = dropin.tidal_select(bp, *c, rt)
    np.testing.assert_array_equal(got, bound.tidal_select(pos, c, rt))
    plist = rng.permutation(len(pos))[:20011].astype(np.int32)
    got = dropin.tidal_select(bp, *c, rt, plist=plist)
    np.testing.assert_array_equal(got, bound.tidal_select(pos, c, rt, plist))
    assert len(dropin.tidal_select(bp, *c, np.float32(0.0))) == 0
    assert len(dropin.tidal_select(bp, *c, rt, plist=np.zeros(0, np.int32))) == 0
