"""Generates the golden fixtures in tests/golden/ by running the reference's
own NewGalFinder C code (compiled from /root/reference by oracle/Makefile,
with the one-token INSERT fix for the "fixed" variant and the FP64 fftw3f
shim standing in for FFTW) on small seeded inputs.

    python tests/golden/make_golden.py

The reference runs single-threaded (OMP_NUM_THREADS=1) so that its float
accumulations happen in particle order and the fixtures are reproducible.
Fixtures hold the inputs as well as the outputs, so tests never need the
reference tree.  Test infrastructure only.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

os.environ["OMP_NUM_THREADS"] = "1"
ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

from oracle.oracle import Reference  # noqa: E402

OUT = Path(__file__).resolve().parent
CELL, NBUFF, RG = 0.004, 10, 0.008


def blob(seed, n, sigma, nsub=2):
    """Clustered test halo: a Gaussian core plus two compact clumps, positions
    recentred as Dump2BP does (x - min)."""
    rng = np.random.default_rng(seed)
    parts = [sigma * rng.standard_normal((n - 2 * (n // 8), 3))]
    for _ in range(nsub):
        c = sigma * 1.5 * rng.standard_normal(3)
        parts.append(c + 0.2 * sigma * rng.standard_normal((n // 8, 3)))
    p = np.concatenate(parts)[:n]
    p -= p.min(axis=0)
    return p


def ref_mesh(p):
    """lagFindStellarCore's mesh for recentred positions (nnost.c:1040-1059)."""
    xmax = p.max(axis=0)
    xmax = xmax + xmax * 0.0001
    n = (xmax / CELL + NBUFF).astype(int)
    origin = 0.0 - CELL * NBUFF / 2.0
    return int(n[0]), int(n[1]), int(n[2]), origin


def main():
    ref = Reference("fixed")
    ref_asbuilt = Reference("asbuilt")

    # ---- mesh chain: TSC (all / stars) -> smoothing -> findDen
    p = blob(11, 2000, 0.012)
    rng = np.random.default_rng(12)
    mass = 10 ** rng.uniform(6, 8, len(p))
    typ = np.where(rng.random(len(p)) < 0.3, 1, 2).astype(np.int32)
    nx, ny, nz, o = ref_mesh(p)
    out = dict(pos=p, mass=mass, type=typ, dims=np.array([nx, ny, nz]), origin=o, cell=CELL, rg=RG)
    for tag, ptype in (("all", 5), ("star", 1)):
        den = ref.assign_density_TSC(p[:, 0], p[:, 1], p[:, 2], mass, typ, nx, ny, nz, o, o, o,
                                     CELL, ptype)
        sm = ref.gaussian_Smoothing(den, nx, ny, nz, CELL, RG)
        dens = ref.findDen(p[:, 0], p[:, 1], p[:, 2], sm, nx, ny, nz, o, o, o, CELL)
        out[f"tsc_{tag}"] = den
        out[f"smooth_{tag}"] = sm
        out[f"findden_{tag}"] = dens
    ldens, lidx, lpeak, lcore = ref.lagFindStellarCore(p[:, 0], p[:, 1], p[:, 2], mass, typ, 32, 5)
    out["lag_dens_all"] = ldens
    np.savez_compressed(OUT / "mesh_chain.npz", **out)

    # ---- smoothing on odd / prime mesh sizes with random content
    rng = np.random.default_rng(13)
    sm_out = {}
    for (a, b, c) in ((23, 29, 31), (16, 12, 20)):
        mx = 2 * (a // 2 + 1)
        den = np.zeros((c, b, mx), np.float32)
        den[:, :, :a] = rng.random((c, b, a)).astype(np.float32) ** 8 * 1e4
        den = den.ravel()
        sm_out[f"in_{a}_{b}_{c}"] = den
        sm_out[f"out_{a}_{b}_{c}"] = ref.gaussian_Smoothing(den, a, b, c, CELL, 0.006)
    np.savez_compressed(OUT / "smooth_sizes.npz", **sm_out)

    # ---- kNN + SPH density (findsphdensity): fixed and as-built
    q = blob(21, 2000, 0.05).astype(np.float32).astype(np.float64)  # FP32-rounded positions
    m = np.full(len(q), 1e8)
    idx_f, dens_f = ref.findsphdensity(q[:, 0], q[:, 1], q[:, 2], m, 32)
    idx_a, dens_a = ref_asbuilt.findsphdensity(q[:, 0], q[:, 1], q[:, 2], m, 32)
    fidx, fd2, fmaxr = ref.find_near_all(q[:, 0], q[:, 1], q[:, 2], m, 32)
    np.savez_compressed(OUT / "knn.npz", pos=q, idx_fixed=idx_f.astype(np.int32), dens_fixed=dens_f,
                        idx_asbuilt=idx_a.astype(np.int32), dens_asbuilt=dens_a,
                        maxr_fixed=fmaxr)

    # ---- tree potential, Self_Halo_Potent, External_Halo_Potent
    r = blob(31, 3000, 0.05)
    rng = np.random.default_rng(32)
    mf = (10 ** rng.uniform(7, 8.5, len(r))).astype(np.float32)
    phi = ref.tree_potential(r[:, 0], r[:, 1], r[:, 2], mf, 0.5)
    self_pe = ref.Self_Halo_Potent(r[:, 0], r[:, 1], r[:, 2], mf)
    small = r[:80]
    self_small = ref.Self_Halo_Potent(small[:, 0], small[:, 1], small[:, 2], mf[:80])
    tgt = r[::3][:1500]
    ext_pe = ref.External_Halo_Potent(tgt[:, 0], tgt[:, 1], tgt[:, 2], mf[::3][:1500], r[:, 0],
                                      r[:, 1], r[:, 2], mf)
    potentfact, r1k, r2k = ref.physics()
    np.savez_compressed(OUT / "potential.npz", pos=r, mass=mf, phi_tree=phi, self_pe=self_pe,
                        self_small=self_small, ext_pe=ext_pe, potentfact=potentfact,
                        r1kineticfact=r1k, r2kineticfact=r2k,
                        bg_1e12=ref.bg_potent(1e12), bg_mass=ref.bg_potent(float(np.sum(mf, dtype=np.float64))))
    bound_fixture(ref)
    cores_fixture(ref)
    starden_fixture(ref)
    for f in sorted(OUT.glob("*.npz")):
        print(f.name, f.stat().st_size)


def starden_fixture(ref):
    """starfindsphdensity (nnost.c:632-744): the stellar density of every
    particle over its 10 nearest stars and every particle's 32-neighbour
    list, for a halo with 20 % stars and one with 6 stars (fewer than 10)."""
    out = {}
    for tag, seed, n, frac in (("a", 41, 1500, 0.2), ("b", 42, 300, 0.02)):
        p = blob(seed, n, 0.03).astype(np.float32).astype(np.float64)  # float-representable
        rng = np.random.default_rng(seed + 100)
        typ = np.full(n, 2, np.int32)
        typ[rng.choice(n, max(1, int(round(frac * n))), replace=False)] = 1
        mass = np.where(typ == 1, 10.0 ** rng.uniform(6, 7, n), 1e8)
        idx, dens = ref.starfindsphdensity(p[:, 0], p[:, 1], p[:, 2], mass, typ, 32)
        out.update({f"pos_{tag}": p, f"mass_{tag}": mass, f"type_{tag}": typ,
                    f"idx_{tag}": idx.astype(np.int32), f"dens_{tag}": dens})
    np.savez_compressed(OUT / "starden.npz", **out)


def cores_fixture(ref):
    """finddenpeak (subhaloden.mod6.c:416; all particles and stars only) and
    FindCoreDensity (:1167) on the reference's own kNN lists and SPH
    densities (findsphdensity) of a clustered halo with four clumps."""
    n = 3000
    p = blob(21, n, 0.02, nsub=4)
    rng = np.random.default_rng(21)
    mass = 10 ** rng.uniform(6, 8, n)
    typ = np.where(rng.random(n) < 0.3, 1, 2).astype(np.int32)
    idx, dens = ref.findsphdensity(p[:, 0], p[:, 1], p[:, 2], mass, 32)
    peak, xyzd = ref.finddenpeak(dens, idx, typ, p[:, 0], p[:, 1], p[:, 2], 0)
    speak, sxyzd = ref.finddenpeak(dens, idx, typ, p[:, 0], p[:, 1], p[:, 2], 1)
    cd = ref.FindCoreDensity(dens, idx, typ, mass, peak)
    out = dict(pos=p, mass=mass, type=typ, neighbor=idx.astype(np.int16), den=dens, peak=peak,
               peak_xyzd=xyzd, star_peak=speak, star_peak_xyzd=sxyzd)
    out.update({f"core_{k}": v for k, v in cd.items()})
    np.savez_compressed(OUT / "cores.npz", **out)


def clumps(rng, sizes, centres, sigmas):
    """Gaussian clumps (one per core) in shuffled particle order, plus 400
    unassigned background particles (haloid -1)."""
    pos, hid = [], []
    for c, (n, ctr, sg) in enumerate(zip(sizes, centres, sigmas)):
        pos.append(np.asarray(ctr) + sg * rng.standard_normal((n, 3)))
        hid.append(np.full(n, c, np.int32))
    pos.append(0.25 + 0.2 * rng.standard_normal((400, 3)))
    hid.append(np.full(400, -1, np.int32))
    pos, hid = np.concatenate(pos), np.concatenate(hid)
    perm = rng.permutation(len(pos))
    return pos[perm], hid[perm]


def bound_fixture(ref):
    """CheckSelfTE / CheckExternalTE (subhaloden.mod6.c:1730, 1622), the
    tidal radius (AdGetTidalRCenterCore, :1910) and GetBGpotent (:1093)."""
    potentfact, r1k, r2k = ref.physics()
    rng = np.random.default_rng(41)
    r = blob(41, 3000, 0.03)
    mf = (10 ** rng.uniform(7, 8.5, len(r))).astype(np.float32)
    typ = np.where(rng.random(len(r)) < 0.3, 1, 2).astype(np.int32)
    pe = ref.Self_Halo_Potent(r[:, 0], r[:, 1], r[:, 2], mf)
    vs = np.sqrt(np.median(-pe.astype(np.float64))) / r2k  # about half bound
    v = (vs * rng.standard_normal((len(r), 3))).astype(np.float32)
    out = dict(pos=r, vel=v, mass=mf, type=typ, self_pe=pe)
    out["self_flag"], out["self_nb"] = ref.CheckSelfTE(r[:, 0], r[:, 1], r[:, 2], v[:, 0], v[:, 1],
                                                       v[:, 2], mf, typ)
    # fewer than 100 members (direct sum) and a member set without stars
    s = slice(0, 70)
    vsm = v[s] * np.float32(0.15)
    out["small_vel"] = vsm
    out["small_flag"], out["small_nb"] = ref.CheckSelfTE(r[s, 0], r[s, 1], r[s, 2], vsm[:, 0],
                                                         vsm[:, 1], vsm[:, 2], mf[s], typ[s])
    out["small_pe"] = ref.Self_Halo_Potent(r[s, 0], r[s, 1], r[s, 2], mf[s])
    dm = np.full(70, 2, np.int32)
    out["nostar_flag"], out["nostar_nb"] = ref.CheckSelfTE(r[s, 0], r[s, 1], r[s, 2], vsm[:, 0],
                                                           vsm[:, 1], vsm[:, 2], mf[s], dm)
    # a satellite's particles against the host's potential
    sat = r[1::2][:1200] + np.array([0.02, -0.01, 0.015])
    vsat = v[1::2][:1200] * np.float32(0.7)
    msat = mf[1::2][:1200]
    core6 = np.array([*r.mean(0), *v.mean(0)], np.float32)
    out.update(ext_pos=sat, ext_vel=vsat, ext_mass=msat, ext_core=core6,
               ext_pe=ref.External_Halo_Potent(sat[:, 0], sat[:, 1], sat[:, 2], msat, r[:, 0],
                                               r[:, 1], r[:, 2], mf))
    out["ext_flag"], out["ext_nb"] = ref.CheckExternalTE(sat[:, 0], sat[:, 1], sat[:, 2],
                                                         vsat[:, 0], vsat[:, 1], vsat[:, 2], msat,
                                                         r[:, 0], r[:, 1], r[:, 2], mf, core6)
    # tidal radius: cores of 0..2500 members, overlapping and far pairs
    rng = np.random.default_rng(43)
    sizes = [0, 40, 90, 150, 400, 900, 2000, 2500, 60, 300]
    centres = [(0.2, 0.2, 0.2), (0.30, 0.30, 0.30), (0.301, 0.302, 0.299), (0.5, 0.2, 0.3),
               (0.32, 0.28, 0.31), (0.8, 0.8, 0.8), (0.3, 0.3, 0.3), (0.55, 0.25, 0.3),
               (0.9, 0.1, 0.5), (0.82, 0.78, 0.81)]
    sigmas = [0.01, 0.004, 0.003, 0.006, 0.008, 0.012, 0.02, 0.025, 0.003, 0.006]
    tpos, thid = clumps(rng, sizes, centres, sigmas)
    tmass = 10 ** rng.uniform(7, 8.5, len(tpos))
    tcore = np.zeros((len(sizes), 6), np.float32)
    for c in range(len(sizes)):
        sel = thid == c
        tcore[c, :3] = tpos[sel].mean(0) if sel.any() else centres[c]
        tcore[c, 3:] = 30.0 * rng.standard_normal(3)
    counts = np.array(sizes)
    score = np.array([c for c in np.argsort(counts, kind="stable") if c != 3], np.int32)  # core 3 unranked
    rt, nm = ref.AdGetTidalRCenterCore(tpos[:, 0], tpos[:, 1], tpos[:, 2], tmass, thid, tcore, score)
    out.update(tid_pos=tpos, tid_mass=tmass, tid_haloid=thid, tid_core=tcore, tid_score=score,
               tid_rtidal=rt, tid_nummem=nm)
    masses = np.array([1e8, 3.3e9, 1e11, 2.7e12, 1e14, 4.4e15])
    out.update(bg_mass=masses, bg=np.array([ref.bg_potent(float(m)) for m in masses]))
    np.savez_compressed(OUT / "bound.npz", **out)


if __name__ == "__main__":
    if len(sys.argv) > 1:  # named fixtures only, e.g. `make_golden.py cores`
        for name in sys.argv[1:]:
            globals()[f"{name}_fixture"](Reference("fixed"))
    else:
        main()
