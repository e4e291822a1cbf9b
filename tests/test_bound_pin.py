"""CPU: the boundedness / tidal-radius restatement (oracle/bound.py) pinned to
the reference's own outputs (tests/golden/bound.npz), libgf's host-side NFW
arithmetic (GetBGpotent) bit for bit, and the argument checks of the new
entry points (no device work)."""
import ctypes

import numpy as np
import pytest

from galaxyfinder_b200 import _lib, dropin
from oracle import bound


@pytest.fixture(scope="module")
def g(golden):
    return golden("bound")


@pytest.fixture(scope="module")
def phys(golden):
    p = golden("potential")
    return float(p["potentfact"]), float(p["r1kineticfact"]), float(p["r2kineticfact"])


def test_self_flags_restated(g, phys):
    _, r1k, r2k = phys
    c = bound.star_centre(g["pos"], g["vel"], g["mass"], g["type"])
    ke = bound.kinetic(g["pos"], g["vel"], c, r1k, r2k)
    flags = bound.bound_flags(ke, g["self_pe"])
    np.testing.assert_array_equal(flags, g["self_flag"])
    assert int(flags.sum()) == int(g["self_nb"])
    s = slice(0, 70)
    c = bound.star_centre(g["pos"][s], g["small_vel"], g["mass"][s], g["type"][s])
    ke = bound.kinetic(g["pos"][s], g["small_vel"], c, r1k, r2k)
    np.testing.assert_array_equal(bound.bound_flags(ke, g["small_pe"]), g["small_flag"])
    c = bound.star_centre(g["pos"][s], g["small_vel"], g["mass"][s], np.full(70, 2))
    ke = bound.kinetic(g["pos"][s], g["small_vel"], c, r1k, r2k)
    np.testing.assert_array_equal(bound.bound_flags(ke, g["small_pe"]), g["nostar_flag"])


def test_external_flags_restated(g, phys):
    _, r1k, r2k = phys
    ke = bound.kinetic(g["ext_pos"], g["ext_vel"], g["ext_core"].astype(np.float64), r1k, r2k)
    flags = bound.bound_flags(ke, g["ext_pe"])
    np.testing.assert_array_equal(flags, g["ext_flag"])
    assert int(flags.sum()) == int(g["ext_nb"])


def test_tidal_radius_restated(g, phys):
    potentfact, _, r2k = phys
    rt, nm = bound.tidal_radius(g["tid_core"], g["tid_score"], g["tid_pos"], g["tid_mass"],
                                g["tid_haloid"], r2k, potentfact)
    np.testing.assert_array_equal(rt, g["tid_rtidal"])
    np.testing.assert_array_equal(nm, g["tid_nummem"])


def test_bg_potent_bit_exact(g):
    for m, ref in zip(g["bg_mass"], g["bg"]):
        assert dropin.bg_potent(float(m)) == float(ref), m


def test_tidal_radius_without_pairs_runs_on_host(g, phys):
    """One ranked core with members and one empty: no core pair, so no device
    work; MAX_TIDAL_R and 0 as in the reference."""
    potentfact, _, r2k = phys
    score = np.array([0, 4], np.int32)
    c6 = g["tid_core"]
    core = np.zeros(len(c6), _lib.CORE_DTYPE)
    for k, f in enumerate(("cx", "cy", "cz", "cvx", "cvy", "cvz")):
        core[f] = c6[:, k]
    bp = np.zeros(len(g["tid_pos"]), _lib.BP_DTYPE)
    bp["x"], bp["y"], bp["z"] = g["tid_pos"].T
    bp["mass"] = g["tid_mass"]
    dropin.tidal_radius(core, score, bp, g["tid_haloid"])
    rt, nm = bound.tidal_radius(c6, score, g["tid_pos"], g["tid_mass"], g["tid_haloid"], r2k,
                                potentfact)
    np.testing.assert_array_equal(core["Rtidal"], rt)
    np.testing.assert_array_equal(core["nummem"], nm)
    assert core["Rtidal"][4] == np.float32(2e5) and core["Rtidal"][0] == 0


def test_argument_errors():
    L = _lib.lib()
    bp = np.zeros(4, _lib.BP_DTYPE)
    out = np.zeros(4, np.int32)
    n = ctypes.c_int(-1)
    bad = np.array([0, 7], np.int32)
    assert L.gf_tidal_select(_lib.ptr(bp), 4, _lib.ptr(bad), 2, 0.0, 0.0, 0.0, 1.0, _lib.ptr(out),
                             ctypes.byref(n)) == _lib.GF_EINVAL
    assert L.gf_tidal_select(_lib.ptr(bp), -1, None, 0, 0.0, 0.0, 0.0, 1.0, _lib.ptr(out),
                             ctypes.byref(n)) == _lib.GF_EINVAL
    core = np.zeros(2, _lib.CORE_DTYPE)
    hid = np.zeros(4, np.int32)
    assert L.gf_tidal_radius(_lib.ptr(core), 2, _lib.ptr(np.array([0, 5], np.int32)), 2,
                             _lib.ptr(bp), _lib.ptr(hid), 4) == _lib.GF_EINVAL
    hid[1] = 9
    assert L.gf_tidal_radius(_lib.ptr(core), 2, _lib.ptr(np.array([0, 1], np.int32)), 2,
                             _lib.ptr(bp), _lib.ptr(hid), 4) == _lib.GF_EINVAL
    flags = np.zeros(4, np.uint8)
    assert L.CheckExternalTE(None, 4, _lib.ptr(flags), None, 0, None) == 0
    assert L.gf_last_status() == _lib.GF_EINVAL
