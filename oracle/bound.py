"""CPU restatement of NewGalFinder's boundedness test, tidal radius and tidal
cut (test infrastructure only; tests/ check results against it).

The reference mixes float, double and long double in these routines; the
restatement keeps each operand type:

* float steps use numpy float32 scalars/arrays,
* double steps use Python floats / float64 (IEEE, no contraction),
* the long double steps (every constant written with an L suffix in the
  reference) use numpy.longdouble, which is the x87 80-bit type on x86-64
  like the reference's compiled code,
* pow and log are the C library's (math.pow / math.log), called with the
  long double values rounded to double as the C calls receive them.

Reference: NewGalFinder/subhaloden.mod6.c
  kinetic energy         :1787-1795 (CheckSelfTE), :1667-1675 (CheckExternalTE)
  stellar centre         :1770-1784
  NFW helpers            :1059-1092
  get_tidal_ellipse      :1102-1165
  AdGetTidalRCenterCore  :1910-2035
  tidal cut              :2732-2741, :528-541
"""
from __future__ import annotations

import math

import numpy as np

L = np.longdouble
F32 = np.float32
MAX_TIDAL_R = 2.e5   # subhaloden.mod6.c:34
NUM_MASS = 10000     # header.h:97
TYPE_STAR = 1        # TYPE_STAR, the first ParticleType enumerator
RHOC = L("2.7755E11")                          # subhaloden.mod6.c:1081
THIRD_13 = float(L("0.3333333333333"))        # GetRvir's exponent as pow receives it
THIRD_14 = float(L("0.33333333333333"))       # get_tidal_ellipse's exponent


def kinetic(pos, vel, c, r1k, r2k):
    """kenergy[i] = 0.5*(tmpv.tmpv): float offsets of the FP64 positions from
    the double centre scaled in double, float velocities offset and scaled in
    double, a float sum of float squares, 0.5* in double, stored as float."""
    dist = ((np.asarray(pos, np.float64) - np.asarray(c[:3], np.float64)) * r1k).astype(F32)
    tv = (dist.astype(np.float64) + (np.asarray(vel, F32).astype(np.float64) - np.asarray(c[3:], np.float64))
          * r2k).astype(F32)
    s = (tv[:, 0] * tv[:, 0] + tv[:, 1] * tv[:, 1]) + tv[:, 2] * tv[:, 2]
    return (0.5 * s.astype(np.float64)).astype(F32)


def star_centre(pos, vel, mass, typ):
    """CheckSelfTE's centre: FP64 sums over the stars in member order of
    position*mass and velocity*mass over the FP64 sum of the float masses
    (0/0 without stars, as in the reference)."""
    st = np.asarray(typ) == TYPE_STAR
    m = np.asarray(mass, F32)[st].astype(np.float64)
    if not st.any():
        return np.full(6, np.nan)
    acc = [np.cumsum(np.asarray(pos, np.float64)[st, a] * m)[-1] for a in range(3)]
    acc += [np.cumsum(np.asarray(vel, F32)[st, a].astype(np.float64) * m)[-1] for a in range(3)]
    return np.array(acc) / np.cumsum(m)[-1]


def bound_flags(ke, pe):
    """BOUND (1) unless kenergy > -penergy (UNBOUND, 0), both float."""
    return np.where(np.asarray(ke, F32) > -np.asarray(pe, F32), 0, 1).astype(np.uint8)


class Nfw:
    """get_concentration / get_alpha / gnfw / GetRvir with the reference's
    float globals (amax, a, omep) and long double constants."""

    def __init__(self, amax=1.0, a=1.0, omep=0.3):
        self.amax, self.a, self.omep = F32(amax), F32(a), F32(omep)
        om1 = L(self.omep) - L(1)
        self.vv = L(18) * L(math.pi) * L(math.pi) + L(82) * om1 - L(39) * L(math.pow(float(om1), 2.0))

    def concentration(self, mass):
        redshift = float(L(self.amax / self.a) - L(1))
        return float(L(14.5 * math.pow(mass / float(L("1.3E13")), -0.15)) / (L(1) + L(redshift)))

    @staticmethod
    def alpha(c, s):
        cs = c * s
        t = L(cs) / (L(1) + L(cs))
        res = float(L(2) - t * t)
        return float(L(res) / (L(math.log(float(L(1) + L(cs)))) - L(cs) / (L(1) + L(cs))))

    @staticmethod
    def gnfw(c):
        return float(L(1.0) / (L(math.log(float(L(1) + L(c)))) - L(c) / (L(1) + L(c))))

    def rvir(self, mvir):
        return math.pow(float(L(3.0 * float(mvir)) / (L(4) * L(math.pi) * self.vv * RHOC)), THIRD_13)


def tidal_ellipse(nfw, my, other, mvir, mratio, bmass, r2k, potentfact):
    """get_tidal_ellipse; my/other are (cx, cy, cz, cvx, cvy, cvz) float32."""
    my, other = np.asarray(my, F32), np.asarray(other, F32)
    d = [float(my[k] - other[k]) for k in range(3)]        # float differences
    dv = [float(my[3 + k] - other[3 + k]) for k in range(3)]
    dist = math.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
    v2 = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]
    wx = d[1] * dv[2] - d[2] * dv[1]
    wy = d[2] * dv[0] - d[0] * dv[2]
    wz = d[0] * dv[1] - d[1] * dv[0]
    w2 = (wx * wx + wy * wy + wz * wz) / (dist * dist)
    pot = float(mvir) / dist
    kpdratio = r2k * r2k / potentfact
    ellipse = w2 / pot * kpdratio
    rv = nfw.rvir(mvir)
    s = dist / rv
    c = nfw.concentration(bmass)
    if s > 1:
        fact = v2 / (bmass / rv) * kpdratio
    else:
        fact = v2 * s / (nfw.gnfw(c) * math.log(float(L(1) + L(c * s))) * bmass / rv) * kpdratio
    if fact > 2.0:
        ellipse = 0.0
    return math.pow(mratio / (ellipse + nfw.alpha(c, s)), THIRD_14)


def tidal_radius(core6, score, pos, mass, haloid, r2k, potentfact, nfw=None):
    """AdGetTidalRCenterCore -> (Rtidal, nummem) for the ranked cores (others 0)."""
    nfw = nfw or Nfw()
    core6 = np.asarray(core6, F32).reshape(-1, 6)
    ncore_all = len(core6)
    pos = np.asarray(pos, np.float64)
    mass = np.asarray(mass, np.float64)
    hid = np.asarray(haloid)
    order = np.argsort(hid, kind="stable")
    sh = hid[order]
    members = [order[np.searchsorted(sh, c):np.searchsorted(sh, c, "right")] for c in range(ncore_all)]
    tmass = np.zeros(ncore_all, F32)
    for c in range(ncore_all):              # core2member[].tmass += bp[i].mass (float)
        acc = F32(0)
        for w in mass[members[c]]:
            acc = F32(float(acc) + float(w))
        tmass[c] = acc
    rt_out = np.zeros(ncore_all, F32)
    nm_out = np.zeros(ncore_all, np.int32)
    for a, ci in enumerate(score):
        n_i = len(members[ci])
        nm_out[ci] = n_i
        if n_i == 0:
            rt_out[ci] = 0
            continue
        rt = F32(MAX_TIDAL_R)
        ci_c = core6[ci, :3].astype(np.float64)
        for cj in score[a + 1:]:
            mj = members[cj]
            if len(mj) == 0:
                continue
            cj_c = core6[cj, :3].astype(np.float64)
            dc = cj_c - ci_c
            r2 = (dc[0] * dc[0] + dc[1] * dc[1]) + dc[2] * dc[2]
            t = pos[mj] - cj_c
            sel = (t[:, 0] * t[:, 0] + t[:, 1] * t[:, 1]) + t[:, 2] * t[:, 2] < r2
            if not sel.any():
                rt = rt if float(rt) < MAX_TIDAL_R else F32(MAX_TIDAL_R)
                continue
            mvir = np.cumsum(mass[mj][sel].astype(F32), dtype=F32)[-1]   # float Mvir += mass
            q = F32(tmass[ci] / mvir) * F32(NUM_MASS)
            if NUM_MASS <= q < 2147483648.0:      # int conversion out of range -> INT_MIN
                rt = F32(math.sqrt(r2) * 0.5)
            else:
                mratio = float(F32(tmass[ci] / mvir))
                tr = tidal_ellipse(nfw, core6[ci], core6[cj], mvir, mratio, float(tmass[cj]), r2k,
                                   potentfact)
                tr = tr if tr < 0.5 else 0.5
                cand = math.sqrt(r2) * tr
                rt = rt if float(rt) < cand else F32(cand)
        rt_out[ci] = rt
    return rt_out, nm_out


def tidal_select(pos, c, rtidal, plist=None):
    """Entries whose float offset from the float centre has float |d|^2 < Rt^2."""
    pos = np.asarray(pos, np.float64)
    idx = np.arange(len(pos), dtype=np.int32) if plist is None else np.asarray(plist, np.int32)
    c = np.asarray(c, F32).astype(np.float64)
    t = (pos[idx] - c).astype(F32)
    d2 = (t[:, 0] * t[:, 0] + t[:, 1] * t[:, 1]) + t[:, 2] * t[:, 2]
    rt = F32(rtidal)
    return idx[d2 < rt * rt]
