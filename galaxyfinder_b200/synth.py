"""Seeded synthetic FoF halos standing in for RAMSES/opFoF catalogues.

The reference runs on private simulation snapshots; these generators produce
inputs with the same shapes, units and statistics as the benchmark
configurations: FP64 comoving positions (cMpc/h) in a 100 cMpc/h periodic
box, masses in Msun/h, NFW profiles sampled by the inverse CDF of
mu(x) = ln(1 + x) - x/(1 + x) (the normalisation of gnfw,
NewGalFinder/subhaloden.mod6.c:1083-1087), r200 from
M = 200 rho_c 4/3 pi r200^3 with rho_c = 2.7755e11 h^2 Msun/Mpc^3
(subhaloden.mod6.c:1081), isotropic Gaussian velocities (300 km/s) and
sequential int64 IDs.  Every generator takes a numpy PCG64 seed.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

RHO_C = 2.7755e11
BOX = 100.0
DM_MASS = 1.0e8
SEED_BASE = 20261203
TYPE_STAR, TYPE_DM = 1, 2


@dataclass
class HaloBatch:
    """Concatenated particles of many halos; halo h is [pstart[h], pstart[h+1])."""
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    mass: np.ndarray
    type: np.ndarray
    ids: np.ndarray
    pstart: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def nhalo(self) -> int:
        return len(self.pstart) - 1

    @property
    def n(self) -> int:
        return int(self.pstart[-1])

    def halo(self, h: int) -> "HaloBatch":
        a, b = int(self.pstart[h]), int(self.pstart[h + 1])
        return HaloBatch(self.x[a:b], self.y[a:b], self.z[a:b], self.vx[a:b], self.vy[a:b],
                         self.vz[a:b], self.mass[a:b], self.type[a:b], self.ids[a:b],
                         np.array([0, b - a], np.int64), dict(self.meta))


def r200_of_mass(m: float) -> float:
    return (3.0 * m / (4.0 * np.pi * 200.0 * RHO_C)) ** (1.0 / 3.0)


def _mu(x):
    return np.log1p(x) - x / (1.0 + x)


def nfw_radii(rng: np.random.Generator, n: int, c: float, r200: float) -> np.ndarray:
    """Radii in (0, r200] with the NFW enclosed-mass profile of concentration c."""
    s = np.linspace(0.0, 1.0, 8193)[1:]
    cdf = _mu(c * s) / _mu(c)
    u = rng.random(n)
    s_of_u = np.interp(u, np.concatenate([[0.0], cdf]), np.concatenate([[0.0], s]))
    return np.maximum(s_of_u, 1e-6) * r200


def _directions(rng: np.random.Generator, n: int) -> np.ndarray:
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def nfw_blob(rng, n, c, r200, centre):
    r = nfw_radii(rng, n, c, r200)
    return centre[None, :] + r[:, None] * _directions(rng, n)


def _wrap(p):
    return np.mod(p, BOX)


def _finish(pos_list, mass_list, type_list, rng, meta) -> HaloBatch:
    counts = [len(p) for p in pos_list]
    pstart = np.zeros(len(counts) + 1, np.int64)
    pstart[1:] = np.cumsum(counts)
    pos = np.concatenate(pos_list) if pos_list else np.zeros((0, 3))
    n = len(pos)
    vel = rng.standard_normal((n, 3)) * 300.0
    return HaloBatch(
        x=np.ascontiguousarray(pos[:, 0]), y=np.ascontiguousarray(pos[:, 1]),
        z=np.ascontiguousarray(pos[:, 2]), vx=vel[:, 0].copy(), vy=vel[:, 1].copy(),
        vz=vel[:, 2].copy(), mass=np.concatenate(mass_list).astype(np.float64),
        type=np.concatenate(type_list).astype(np.int32), ids=np.arange(n, dtype=np.int64),
        pstart=pstart, meta=meta)


def config1(seed: int = SEED_BASE + 1, n: int = 131072) -> HaloBatch:
    """One halo: N equal-mass (1e8) DM particles, NFW r200 = 0.5, c = 8, with two
    embedded NFW subhalos of 10% and 3% of the mass (c = 8,
    r200_sub = r200 (m/M)^(1/3)) offset by 0.1-0.3 r200 in random directions."""
    rng = np.random.default_rng(seed)
    r200, c = 0.5, 8.0
    centre = rng.random(3) * BOX
    fr = [0.10, 0.03]
    nsub = [int(round(f * n)) for f in fr]
    nhost = n - sum(nsub)
    parts = [nfw_blob(rng, nhost, c, r200, centre)]
    for f, ns in zip(fr, nsub):
        off = _directions(rng, 1)[0] * rng.uniform(0.1, 0.3) * r200
        parts.append(nfw_blob(rng, ns, c, r200 * f ** (1.0 / 3.0), centre + off))
    pos = _wrap(np.concatenate(parts))
    perm = rng.permutation(n)
    pos = pos[perm]
    return _finish([pos], [np.full(n, DM_MASS)], [np.full(n, TYPE_DM, np.int32)], rng,
                   {"config": 1, "seed": seed, "r200": r200, "c": c})


def config3(seed: int = SEED_BASE + 3, n: int = 50_000_000, nsub: int = 300,
            star_frac: float = 0.1) -> HaloBatch:
    """Single massive cluster: n particles, NFW c = 4, r200 = 2 Mpc/h, nsub
    subhalos with masses from dN/dm ~ m^-1.9 on [1e-5, 1e-2] of the host
    (NFW, c = 8, r200 scaled as m^(1/3), centred within r200), stars at
    star_frac by number (masses 1e6-1e7, concentrated x3 in radius); the
    remaining particles share the host mass."""
    rng = np.random.default_rng(seed)
    r200, c = 2.0, 4.0
    mhost = 200.0 * RHO_C * 4.0 / 3.0 * np.pi * r200 ** 3
    centre = 10.0 + rng.random(3) * (BOX - 20.0)
    fr = powerlaw_counts(rng, nsub, 1.0, 1e3).astype(float) * 1e-5
    nsubp = np.maximum((fr * n).astype(np.int64), 10)
    nhostp = n - int(nsubp.sum())
    parts = [nfw_blob(rng, nhostp, c, r200, centre)]
    rs = r200 * rng.random(nsub) ** (1.0 / 3.0)
    ctrs = centre + _directions(rng, nsub) * rs[:, None]
    for k, f in enumerate(fr):
        parts.append(nfw_blob(rng, int(nsubp[k]), 8.0, r200 * f ** (1.0 / 3.0), ctrs[k]))
    pos = np.concatenate(parts)
    typ = np.where(rng.random(n) < star_frac, TYPE_STAR, TYPE_DM).astype(np.int32)
    st = typ == TYPE_STAR
    # stars three times more concentrated about their component's centre
    owner = np.repeat(np.arange(nsub + 1), [nhostp] + nsubp.tolist())
    cen = np.concatenate([centre[None, :], ctrs])[owner]
    pos[st] = cen[st] + (pos[st] - cen[st]) / 3.0
    mass = np.where(st, 10 ** rng.uniform(6, 7, n), mhost / n)
    perm = rng.permutation(n)
    return _finish([_wrap(pos[perm])], [mass[perm]], [typ[perm]], rng,
                   {"config": 3, "seed": seed, "r200": r200, "c": c, "nsub": nsub})


def config4(seed: int = SEED_BASE + 4, n: int = 10_000_000, nclump: int = 64) -> HaloBatch:
    """Differentiable-density workload: one Gaussian-mixture halo of n
    equal-mass (1e8) DM particles in nclump clumps with sigma log-uniform in
    5-50 kpc/h, log-uniform weights (normalised) and centres uniform in a
    sphere of radius 0.5 Mpc/h."""
    rng = np.random.default_rng(seed)
    centre = 10.0 + rng.random(3) * (BOX - 20.0)
    sig = np.exp(rng.uniform(np.log(0.005), np.log(0.05), nclump))
    w = np.exp(rng.uniform(0.0, np.log(100.0), nclump))
    w /= w.sum()
    counts = rng.multinomial(n, w)
    rad = 0.5 * rng.random(nclump) ** (1.0 / 3.0)
    ctr = centre + _directions(rng, nclump) * rad[:, None]
    pos = np.concatenate([c + s * rng.standard_normal((k, 3)) for c, s, k in zip(ctr, sig, counts)])
    pos = pos[rng.permutation(n)]
    return _finish([pos], [np.full(n, DM_MASS)], [np.full(n, TYPE_DM, np.int32)], rng,
                   {"config": 4, "seed": seed, "nclump": nclump})


G_KMS = 4.30091e-9  # G in Mpc (km/s)^2 / Msun


def galaxy_group(seed: int = SEED_BASE + 6, ndm: int = 20000, nsat: int = 4,
                 star_frac: float = 0.25) -> HaloBatch:
    """One FoF halo with galaxies for the whole per-halo pipeline: an NFW host
    (c = 8) and nsat satellites, each with a compact stellar core (stars at a
    third of the component's scale radius, masses 1e6-1e7) inside its own NFW
    dark halo, and isotropic velocities about each component's bulk velocity
    with the dispersion sqrt(G M / (2 r_half)) of that component, so that the
    galaxies are bound.  meta["component"] is each particle's component
    (0 = host)."""
    rng = np.random.default_rng(seed)
    centre = 20.0 + rng.random(3) * (BOX - 40.0)
    comps = [(1.0, np.zeros(3), np.zeros(3))]
    for _ in range(nsat):
        f = 10 ** rng.uniform(-1.3, -0.7)
        off = _directions(rng, 1)[0] * rng.uniform(0.25, 0.6)
        comps.append((f, off, 120.0 * rng.standard_normal(3)))
    ftot = sum(c[0] for c in comps)
    pos, vel, mass, typ, comp = [], [], [], [], []
    mhost = None
    for ic, (f, off, vbulk) in enumerate(comps):
        nd = max(200, int(ndm * f / ftot))
        ns = max(60, int(star_frac * nd))
        mcomp = nd * DM_MASS + ns * 5e6
        r200 = r200_of_mass(mcomp) * (1.0 if mhost is None else 0.6)
        mhost = mhost or mcomp
        sig = np.sqrt(G_KMS * mcomp / (2.0 * 0.4 * r200))
        p = np.concatenate([nfw_blob(rng, nd, 8.0, r200, centre + off),
                            nfw_blob(rng, ns, 8.0, r200 / 3.0, centre + off)])
        pos.append(p)
        vel.append(vbulk + sig * rng.standard_normal((nd + ns, 3)) / np.sqrt(3.0) * 1.2)
        mass.append(np.concatenate([np.full(nd, DM_MASS), 10 ** rng.uniform(6, 7, ns)]))
        typ.append(np.concatenate([np.full(nd, TYPE_DM), np.full(ns, TYPE_STAR)]).astype(np.int32))
        comp.append(np.full(nd + ns, ic, np.int32))
    pos, vel, mass, typ, comp = map(np.concatenate, (pos, vel, mass, typ, comp))
    perm = rng.permutation(len(pos))
    pos, vel, mass, typ, comp = _wrap(pos[perm]), vel[perm], mass[perm], typ[perm], comp[perm]
    n = len(pos)
    return HaloBatch(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(), vx=vel[:, 0].copy(),
                     vy=vel[:, 1].copy(), vz=vel[:, 2].copy(), mass=mass, type=typ,
                     ids=np.arange(n, dtype=np.int64), pstart=np.array([0, n], np.int64),
                     meta={"seed": seed, "nsat": nsat, "component": comp})


def powerlaw_counts(rng, nhalo, nmin, nmax, slope=-1.9):
    """N_p drawn from dN/dN_p ~ N_p^slope on [nmin, nmax] by inverse CDF."""
    a = slope + 1.0
    u = rng.random(nhalo)
    lo, hi = nmin ** a, nmax ** a
    return np.floor((lo + u * (hi - lo)) ** (1.0 / a)).astype(np.int64)


def _catalogue_halo(rng, npart, star_frac=0.2, straddle=False):
    c = 10 ** (np.log10(6.0) + 0.15 * rng.standard_normal())
    nstar = int(round(star_frac * npart))
    ndm = npart - nstar
    mtot = ndm * DM_MASS + nstar * 10 ** rng.uniform(6, 7)
    r200 = r200_of_mass(mtot)
    centre = rng.random(3) * BOX
    if straddle:  # put the centre on a box face so the halo wraps
        ax = rng.integers(3)
        centre[ax] = rng.uniform(-0.3, 0.3) * r200 % BOX
    nsub_halo = rng.poisson(mtot / 1e11)
    # subhalo masses from dN/dm ~ m^-1.9 on [1e-5, 1e-2] M, as particle fractions
    fr = powerlaw_counts(rng, nsub_halo, 1.0, 1e3).astype(float) * 1e-5 if nsub_halo else np.zeros(0)
    fr = fr[np.cumsum(fr) < 0.5]
    pos_dm = [nfw_blob(rng, ndm - int(fr.sum() * ndm), c, r200, centre)]
    for f in fr:
        ns = int(f * ndm)
        if ns < 1:
            continue
        off = _directions(rng, 1)[0] * rng.uniform(0.1, 0.8) * r200
        pos_dm.append(nfw_blob(rng, ns, c, r200 * f ** (1.0 / 3.0), centre + off))
    pos_dm = np.concatenate(pos_dm)[:ndm]
    if len(pos_dm) < ndm:
        pos_dm = np.concatenate([pos_dm, nfw_blob(rng, ndm - len(pos_dm), c, r200, centre)])
    pos_st = nfw_blob(rng, nstar, 3.0 * c, r200, centre)
    pos = _wrap(np.concatenate([pos_dm, pos_st]))
    mass = np.concatenate([np.full(ndm, DM_MASS), 10 ** rng.uniform(6, 7, nstar)])
    typ = np.concatenate([np.full(ndm, TYPE_DM, np.int32), np.full(nstar, TYPE_STAR, np.int32)])
    perm = rng.permutation(npart)
    return pos[perm], mass[perm], typ[perm]


def catalogue(seed: int = SEED_BASE + 2, nhalo: int = 4096, nmin: int = 100,
              nmax: int = 2_000_000, star_frac: float = 0.2,
              straddle_frac: float = 0.05) -> HaloBatch:
    """Batched catalogue: N_p ~ N^-1.9 on [nmin, nmax]; NFW with log-normal c
    (median 6, 0.15 dex); Poisson(M/1e11) subhalos with a m^-1.9 mass function
    on [1e-5, 1e-2] M; stars at `star_frac` by number (1e6-1e7 Msun/h,
    concentration x3); `straddle_frac` of the halos wrap the periodic box."""
    rng = np.random.default_rng(seed)
    counts = powerlaw_counts(rng, nhalo, nmin, nmax)
    P, M, T = [], [], []
    for npart in counts:
        p, m, t = _catalogue_halo(rng, int(npart), star_frac, rng.random() < straddle_frac)
        P.append(p); M.append(m); T.append(t)
    return _finish(P, M, T, rng, {"config": 2, "seed": seed, "nhalo": nhalo})


def postprocessing_catalogue(seed: int = SEED_BASE + 5, nhalo: int = 100_000, nmin: int = 50,
                             nmax: int = 10_000_000, background_frac: float = 0.1,
                             star_frac: float = 0.2) -> HaloBatch:
    """The full post-processing workload: nhalo halos from the catalogue law
    (N_p ~ N^-1.9 on [nmin, nmax], NFW with subhalos and stars, as
    `catalogue`), each FoF group also holding background_frac x N_p unbound
    DM particles spread uniformly over its r200 sphere (the unbound
    background of the groups).  The expected total is about 1.1e8 group
    particles for the default law; the realised count is in pstart[-1]."""
    rng = np.random.default_rng(seed)
    counts = powerlaw_counts(rng, nhalo, nmin, nmax)
    P, M, T = [], [], []
    for npart in counts:
        p, m, t = _catalogue_halo(rng, int(npart), star_frac, rng.random() < 0.05)
        nb = int(round(background_frac * npart))
        if nb:
            # uniform in the r200 sphere about the group's centre of mass
            r200 = r200_of_mass(float(m.sum()))
            ctr = p[np.argmin(np.abs(p - np.median(p, 0)).sum(1))]
            rb = r200 * rng.random(nb) ** (1.0 / 3.0)
            pb = _wrap(ctr[None, :] + rb[:, None] * _directions(rng, nb))
            p = np.concatenate([p, pb])
            m = np.concatenate([m, np.full(nb, DM_MASS)])
            t = np.concatenate([t, np.full(nb, TYPE_DM, np.int32)])
        P.append(p); M.append(m); T.append(t)
    return _finish(P, M, T, rng, {"config": 5, "seed": seed, "nhalo": nhalo,
                                  "background_frac": background_frac})


def gaussian_blob(seed: int, n: int, sigma: float = 0.05, centre=(50.0, 50.0, 50.0),
                  mass: float = DM_MASS) -> HaloBatch:
    """Small isotropic Gaussian halo used by unit tests."""
    rng = np.random.default_rng(seed)
    pos = np.asarray(centre)[None, :] + sigma * rng.standard_normal((n, 3))
    return _finish([pos], [np.full(n, mass)], [np.full(n, TYPE_DM, np.int32)], rng,
                   {"config": "blob", "seed": seed})


def to_bp(hb: HaloBatch, recentre: bool = True) -> np.ndarray:
    """SimpleBasicParticleType array of one halo; recentred as Dump2BP does
    (x - min(x) per axis, subhaloden.mod6.c:2810-2837) when `recentre`."""
    from ._lib import BP_DTYPE
    n = hb.n
    bp = np.zeros(n, BP_DTYPE)
    bp["type"] = hb.type
    bp["mass"] = hb.mass
    x, y, z = hb.x, hb.y, hb.z
    if recentre:
        x, y, z = x - x.min(), y - y.min(), z - z.min()
    bp["x"], bp["y"], bp["z"] = x, y, z
    bp["vx"], bp["vy"], bp["vz"] = hb.vx, hb.vy, hb.vz
    bp["indx"] = np.arange(n, dtype=np.int32)
    return bp
