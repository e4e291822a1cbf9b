"""Python mirror of the reference entry points that libgf replaces.

Each function takes the reference's arguments (numpy arrays in place of the C
pointers, with the reference's struct layouts from ``_lib``) and calls the
drop-in symbol of the same name in libgf.so.  Where the reference prints a
message and calls exit(), these raise ``GFError``.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._lib import BP_DTYPE, VEC3_DTYPE, check_last, lib, ptr


def mesh_floats(nx: int, ny: int, nz: int) -> int:
    """Length of a padded r2c mesh, mx*ny*nz with mx = 2(nx/2+1) (tsc_omp2.c:16,198)."""
    return 2 * (nx // 2 + 1) * ny * nz


def _bp(bp: np.ndarray) -> np.ndarray:
    if bp.dtype != BP_DTYPE or not bp.flags.c_contiguous:
        raise TypeError("bp must be a contiguous SimpleBasicParticleType array (BP_DTYPE)")
    return bp


def assign_density_TSC(bp, nx, ny, nz, Xmin, Ymin, Zmin, cellsize, ptype, den=None):
    """tsc_omp2.c:166 — TSC deposit of bp into a zeroed mesh (returned)."""
    bp = _bp(bp)
    if den is None:
        den = np.zeros(mesh_floats(nx, ny, nz), np.float32)
    lib().assign_density_TSC(ptr(bp), len(bp), ptr(den), nx, ny, nz, Xmin, Ymin, Zmin, cellsize,
                             ptype)
    check_last()
    return den


def findDen(bp, den, nx, ny, nz, xmin, ymin, zmin, cellsize):
    """tsc_omp2.c:40 — TSC-weighted mesh value at every particle."""
    bp = _bp(bp)
    den = np.ascontiguousarray(den, np.float32)
    out = np.zeros(len(bp), np.float32)
    lib().findDen(ptr(bp), len(bp), ptr(out), xmin, ymin, zmin, cellsize, ptr(den), nx, ny, nz)
    check_last()
    return out


def gaussian_Smoothing(den, nx, ny, nz, cellsize, RG):
    """gsmooth.c:14 — in-place Gaussian smoothing of a padded mesh."""
    if den.dtype != np.float32 or not den.flags.c_contiguous:
        raise TypeError("den must be a contiguous float32 array")
    lib().gaussian_Smoothing(ptr(den), nx, ny, nz, cellsize, RG)
    check_last()
    return den


def findsphdensity(bp, numnear):
    """nnost.c:560 — k nearest neighbours (self included) and the W4 density."""
    bp = _bp(bp)
    n = len(bp)
    near = np.zeros((n, numnear), np.int64)
    dens = np.zeros(n, np.float32)
    lib().findsphdensity(ptr(bp), n, ptr(near), numnear, ptr(dens))
    check_last()
    return near, dens


def starfindsphdensity(bp, numnear):
    """nnost.c:632 — stellar density (10 nearest stars, W4 times mass) at every
    particle and every particle's k nearest neighbours (self included)."""
    bp = _bp(bp)
    n = len(bp)
    near = np.zeros((n, numnear), np.int64)
    dens = np.zeros(n, np.float32)
    lib().starfindsphdensity(ptr(bp), n, ptr(near), numnear, ptr(dens))
    check_last()
    return near, dens


def _vec3(r) -> np.ndarray:
    r = np.asarray(r)
    if r.dtype == VEC3_DTYPE:
        return np.ascontiguousarray(r)
    r = np.ascontiguousarray(r, np.float64).reshape(-1, 3)
    return r.view(VEC3_DTYPE).reshape(-1)


def Self_Halo_Potent(r, mass):
    """subhaloden.mod6.c:1477 — self-potential energy of a member set."""
    r = _vec3(r)
    mass = np.ascontiguousarray(mass, np.float32)
    pe = np.zeros(len(r), np.float32)
    lib().Self_Halo_Potent(len(r), ptr(r), ptr(mass), ptr(pe))
    check_last()
    return pe


def External_Halo_Potent(r, mass, sr, smass):
    """subhaloden.mod6.c:1537 — potential of the sources (sr, smass) at r."""
    r, sr = _vec3(r), _vec3(sr)
    mass = np.ascontiguousarray(mass, np.float32)
    smass = np.ascontiguousarray(smass, np.float32)
    pe = np.zeros(len(r), np.float32)
    lib().External_Halo_Potent(len(r), ptr(r), ptr(mass), ptr(pe), len(sr), ptr(sr), ptr(smass))
    check_last()
    return pe


def make_kp(x, y, z, vx, vy, vz, mass, bp=None) -> np.ndarray:
    """Kptype array (subhaloden.mod6.c:73-77); bp is the SimpleBasicParticleType
    array whose entries the members point to (for their types)."""
    kp = np.zeros(len(x), _lib.KP_DTYPE)
    kp["x"], kp["y"], kp["z"] = x, y, z
    kp["vx"], kp["vy"], kp["vz"] = vx, vy, vz
    kp["mass"] = mass
    if bp is not None:
        kp["bp"] = bp.ctypes.data + np.arange(len(x), dtype=np.uint64) * np.uint64(_lib.BP_DTYPE.itemsize)
    return kp


def CheckSelfTE(kp, bp_owner=None):
    """subhaloden.mod6.c:1730 — returns (bound flags, number bound).  bp_owner
    keeps alive the particle array the kp entries point to."""
    kp = np.ascontiguousarray(kp)
    flags = np.zeros(len(kp), np.uint8)
    nb = lib().CheckSelfTE(ptr(kp), len(kp), ptr(flags), None)
    check_last()
    return flags, nb


def CheckExternalTE(tkp, skp, core):
    """subhaloden.mod6.c:1622 — core: one CORE_DTYPE record (centre, velocity)."""
    tkp, skp = np.ascontiguousarray(tkp), np.ascontiguousarray(skp)
    core = np.ascontiguousarray(core, _lib.CORE_DTYPE).reshape(-1)
    flags = np.zeros(len(tkp), np.uint8)
    nb = lib().CheckExternalTE(ptr(tkp), len(tkp), ptr(flags), ptr(skp), len(skp), ptr(core))
    check_last()
    return flags, nb


def shell_bound(bp, flag, haloid, shellp, shellc, ishell, cores, order):
    """gf_shell_bound: shell `ishell` of the boundedness loop
    (subhaloden.mod6.c:3033-3101) batched over its cores.  flag (uint8) and
    haloid (int32) are updated in place; shellp / shellc are the SHELL2P /
    SHELL2C lists.  Returns (bound count per core of `order`, cores retested
    alone)."""
    bp = np.ascontiguousarray(bp, _lib.BP_DTYPE)
    assert flag.dtype == np.uint8 and flag.flags.c_contiguous
    assert haloid.dtype == np.int32 and haloid.flags.c_contiguous
    sp = np.concatenate([np.asarray(q, np.int32) for q in shellp]) if len(shellp) else np.zeros(0, np.int32)
    sps = np.concatenate([[0], np.cumsum([len(q) for q in shellp])]).astype(np.int32)
    sc = np.concatenate([np.asarray(q, np.int32) for q in shellc]) if len(shellc) else np.zeros(0, np.int32)
    scs = np.concatenate([[0], np.cumsum([len(q) for q in shellc])]).astype(np.int32)
    cores = np.ascontiguousarray(cores, _lib.CORE_DTYPE)
    order = np.ascontiguousarray(order, np.int32)
    nmem = np.zeros(max(len(order), 1), np.int32)
    nret = np.zeros(1, np.int32)
    _lib.check(lib().gf_shell_bound(ptr(bp), len(bp), ptr(flag), ptr(haloid), ptr(sp), ptr(sps), ptr(sc), ptr(scs),
                               len(shellp), ishell, ptr(cores), len(cores), ptr(order), len(order), ptr(nmem),
                               ptr(nret)))
    return [int(v) for v in nmem[:len(order)]], int(nret[0])


def bound_pass(bp, flag, haloid, cores, order, nmem):
    """gf_bound_pass: one BOUNDITER pass (subhaloden.mod6.c:3118-3172) over the
    cores of `order` (nmem: their member counts at the start of the pass),
    batched.  flag (uint8) and haloid (int32) are updated in place.  Returns
    (bound count per core of `order`, GPU passes used)."""
    bp = np.ascontiguousarray(bp, _lib.BP_DTYPE)
    assert flag.dtype == np.uint8 and flag.flags.c_contiguous
    assert haloid.dtype == np.int32 and haloid.flags.c_contiguous
    cores = np.ascontiguousarray(cores, _lib.CORE_DTYPE)
    order = np.ascontiguousarray(order, np.int32)
    nmem = np.ascontiguousarray(nmem, np.int32)
    nb = np.zeros(max(len(order), 1), np.int32)
    nbatch = np.zeros(1, np.int32)
    _lib.check(lib().gf_bound_pass(ptr(bp), len(bp), ptr(flag), ptr(haloid), ptr(cores), len(cores), ptr(order),
                                   ptr(nmem), len(order), ptr(nb), ptr(nbatch)))
    return [int(v) for v in nb[:len(order)]], int(nbatch[0])


def tidal_radius(core, score_core, bp, haloid):
    """AdGetTidalRCenterCore (subhaloden.mod6.c:1910): fills core['Rtidal'] and
    core['nummem'] in place."""
    score_core = np.ascontiguousarray(score_core, np.int32)
    haloid = np.ascontiguousarray(haloid, np.int32)
    _lib.check(lib().gf_tidal_radius(ptr(core), len(core), ptr(score_core), len(score_core),
                                     ptr(bp), ptr(haloid), len(bp)))
    return core


def tidal_select(bp, cx, cy, cz, rtidal, plist=None):
    """Tidal cut (subhaloden.mod6.c:2734-2745): indices within rtidal, in order."""
    n = len(bp) if plist is None else len(plist)
    pl = None if plist is None else np.ascontiguousarray(plist, np.int32)
    out = np.zeros(max(n, 1), np.int32)
    cnt = _lib.ctypes.c_int(0)
    _lib.check(lib().gf_tidal_select(ptr(bp), len(bp), ptr(pl), n, cx, cy, cz, rtidal, ptr(out),
                                     _lib.ctypes.byref(cnt)))
    return out[:cnt.value]


def lagFindStellarCore(bp, numnear, ptype=_lib.TYPE_ALL, maxnumcore=100000):
    """nnost.c:991 — (densph, cores (CORE_DTYPE), nearindex (np, numnear) int64).
    Loaded on its own, libgf has no MergingPeak: more than 10 cores raise."""
    bp = _bp(bp)
    n = len(bp)
    dens = np.zeros(n, np.float32)
    near = np.zeros((n, numnear), np.int64)
    cores = np.zeros(max(maxnumcore, 1), _lib.CORE_DTYPE)
    cptr = _lib.ctypes.c_void_p(cores.ctypes.data)
    ncore = _lib.ctypes.c_int(0)
    lib().lagFindStellarCore(ptr(bp), n, numnear, ptr(dens), _lib.ctypes.byref(cptr),
                             _lib.ctypes.byref(ncore), maxnumcore, ptr(near), ptype)
    check_last()
    return dens, cores[:ncore.value].copy(), near


def finddenpeak(den, neighbor, bp, jflag=0, maxnumcore=1000000):
    """subhaloden.mod6.c:416 — density peaks on the kNN graph as cores
    (CORE_DTYPE: peak, cx, cy, cz, density filled), in particle order.  jflag 1
    keeps stellar peaks only."""
    bp = _bp(bp)
    den = np.ascontiguousarray(den, np.float32)
    nb = np.ascontiguousarray(neighbor, np.int64)
    n, k = nb.shape
    cores = np.zeros(max(maxnumcore, 1), _lib.CORE_DTYPE)
    cptr = _lib.ctypes.c_void_p(cores.ctypes.data)
    nc = lib().finddenpeak(ptr(den), k, ptr(nb), n, _lib.ctypes.byref(cptr), jflag, ptr(bp))
    check_last()
    return cores[:nc].copy()


def i_potent_spline():
    """force_spline.mod3.c:81 — no table is needed by the GPU kernel."""
    lib().i_potent_spline()
    check_last()


def physics() -> dict:
    ph = _lib.Physics()
    _lib.check(lib().gf_get_physics(ph))
    return {f: getattr(ph, f) for f, _ in _lib.Physics._fields_}


def set_cosmology(amax=1.0, a=1.0, omep=0.3, omeplam=0.7, hubble=70.0):
    _lib.check(lib().gf_set_cosmology(amax, a, omep, omeplam, hubble))


def bg_potent(mvir: float) -> float:
    """GetBGpotent, subhaloden.mod6.c:1093."""
    return lib().gf_bg_potent(mvir)
