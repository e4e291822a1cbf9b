"""CPU restatement of the reference's core finding on the kNN graph (test
infrastructure only: the reference results for libgf's gf_density_peaks / gf_core_density
and of the finddenpeak / FindCoreDensity drop-ins).

* density_peaks follows NewGalFinder/subhaloden.mod6.c:416-494 (finddenpeak):
  den[i] > PEAKTHRESHOLD (2000, params.h:19; stars only for the stellar path)
  and no kNN neighbour denser; peaks in particle order.
* core_density follows :1167-1475 (FindCoreDensity) with COREDENRESOLUTION
  1e-3 (params.h:12) and DENFLOOR 1 (params.h:109): per core, bisection of the
  threshold between the peak density and max(DENFLOOR, min density) with
  breadth-first searches along kNN edges through particles denser than the
  threshold (a search fails when it reaches another peak), then the members
  reached at the core density.  The float arithmetic of the bisection is the
  reference's: t = float(up + down) * 0.5, |float(up - down) / t| > 1e-3 in
  double.  The searches here run level by level with numpy (the reached set
  and the failure do not depend on the visiting order); starmass is summed in
  FP64 in particle order and rounded once, while the reference adds in float
  in its search order (the two agree to float rounding).
"""
from __future__ import annotations

import numpy as np

PEAKTHRESHOLD = 2000.0
COREDENRESOLUTION = 1e-3
DENFLOOR = 1.0
NOT_HALO_MEMBER = -9999
WP_PEAK, WP_CORE, WP_BOUND = 0x01, 0x04, 0x10
TYPE_STAR = 1


def density_peaks(den, neighbor, type_=None, threshold=PEAKTHRESHOLD):
    den = np.asarray(den, np.float32)
    nb = np.asarray(neighbor, np.int64)
    cand = den.astype(np.float64) > threshold
    if type_ is not None:
        cand &= np.asarray(type_) == TYPE_STAR
    denser = (den[nb] > den[:, None]).any(axis=1)
    return np.nonzero(cand & ~denser)[0].astype(np.int32)


def _search(start, thr, den, nb, ispeak):
    """Particles reached from start through den > thr; (set, reached another peak)."""
    visited = np.zeros(len(den), bool)
    visited[start] = True
    frontier = np.array([start], np.int64)
    reached = [frontier]
    while len(frontier):
        v = nb[frontier].ravel()
        v = v[den[v] > thr]
        if np.any(ispeak[v] & (v != start)):
            return None, True
        v = np.unique(v[~visited[v]])
        visited[v] = True
        frontier = v
        reached.append(v)
    return np.concatenate(reached), False


def core_density(den, neighbor, type_, mass, peaks):
    den = np.asarray(den, np.float32)
    nb = np.asarray(neighbor, np.int64)
    type_ = np.asarray(type_)
    mass = np.asarray(mass, np.float64)
    peaks = np.asarray(peaks, np.int64)
    n = len(den)
    ispeak = np.zeros(n, bool)
    ispeak[peaks] = True
    minden = np.float32(max(DENFLOOR, float(den.min())))
    nc = len(peaks)
    out = dict(coredensity=np.zeros(nc, np.float32), nummem=np.zeros(nc, np.int32),
               numstar=np.zeros(nc, np.int32), starmass=np.zeros(nc, np.float32),
               haloid=np.full(n, NOT_HALO_MEMBER, np.int32), flag=np.zeros(n, np.uint8))
    for c, p in enumerate(peaks):
        up, down = np.float32(den[p]), minden
        while True:
            thr = np.float32(np.float32(up + down) * np.float32(0.5))
            _, fail = _search(p, thr, den, nb, ispeak)
            if fail:
                down = thr
            else:
                up = thr
            if not abs(float(np.float32(np.float32(up - down) / thr))) > COREDENRESOLUTION:
                break
        members, fail = _search(p, up, den, nb, ispeak)
        if fail:
            members = np.zeros(0, np.int64)
        stars = members[type_[members] == TYPE_STAR]
        out["coredensity"][c] = up
        out["nummem"][c] = len(members)
        out["numstar"][c] = len(stars)
        out["starmass"][c] = np.float32(mass[np.sort(stars)].sum())
        out["haloid"][members] = c  # later cores overwrite, as the reference's serial loop
    out["flag"] = (np.where(ispeak, WP_PEAK, 0) |
                   np.where(out["haloid"] != NOT_HALO_MEMBER, WP_CORE | WP_BOUND, 0)).astype(np.uint8)
    return out
