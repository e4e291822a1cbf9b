"""The shell loop of subhalo_den (NewGalFinder/subhaloden.mod6.c:3033-3101),
restated core by core for the tests: the targets of
GetShellParticleFromRestParticleLIST (:516-543), the sources of
GetMemCandidateList (:544-560), MULTIHALOSHELL's marking (:1706-1721, the
energy test through libgf's CheckExternalTE drop-in, one call per core) and
UnboundShellP2Rest (:2111-2121).  This is the one-call-per-core path that
gf_shell_bound batches."""
import numpy as np

from galaxyfinder_b200 import _lib, dropin

WP_CORE, WP_SHELL, WP_BOUND, WP_REMAINING = 0x04, 0x08, 0x10, 0x20  # :181-186
NOT_MEMBER = -9999  # NOT_HALO_MEMBER, defs.h:29


def within(bp, idx, core):
    """The tidal cut (:532-541): float offsets from the float centre, float
    squared distance, float Rtidal squared."""
    idx = np.asarray(idx, np.int64)
    t = [(bp[f][idx] - np.float64(np.float32(core[c]))).astype(np.float32)
         for f, c in (("x", "cx"), ("y", "cy"), ("z", "cz"))]
    dist2 = (t[0] * t[0] + t[1] * t[1]) + t[2] * t[2]
    rt = np.float32(core["Rtidal"])
    return dist2 < rt * rt


def _kp(bp, idx):
    idx = np.asarray(idx, np.int64)
    kp = dropin.make_kp(bp["x"][idx], bp["y"][idx], bp["z"][idx], bp["vx"][idx].astype(np.float32),
                        bp["vy"][idx].astype(np.float32), bp["vz"][idx].astype(np.float32),
                        bp["mass"][idx].astype(np.float32))
    kp["bp"] = bp.ctypes.data + idx.astype(np.uint64) * np.uint64(_lib.BP_DTYPE.itemsize)
    return kp


def shell_loop(bp, flag, haloid, shellp, shellc, ishell, cores, order):
    """One shell, in place on flag and haloid; returns each core's bound count."""
    np_ = len(bp)
    sp = np.asarray(shellp[ishell], np.int64)
    nmem = []
    for j in order:
        c = cores[j]
        plist = np.concatenate([sp[(flag[sp] & WP_BOUND) == 0],
                                np.nonzero(flag & WP_REMAINING)[0]]).astype(np.int64)
        tl = plist[within(bp, plist, c)] if len(plist) else plist
        if len(tl) == 0:
            nmem.append(0)
            continue
        sl = [np.nonzero(haloid == j)[0]]
        for s in range(ishell + 1, len(shellp)):
            if j in shellc[s]:
                sl.append(np.asarray(shellp[s], np.int64))
        sl = np.concatenate(sl).astype(np.int64)
        flags, nb = dropin.CheckExternalTE(_kp(bp, tl), _kp(bp, sl), c)
        for t, f in zip(tl, flags):  # MULTIHALOSHELL
            if f == _lib.GF_BOUND:
                flag[t] |= WP_BOUND
            else:
                flag[t] |= WP_REMAINING
                flag[t] &= ~WP_BOUND & 0xFF
                haloid[t] = NOT_MEMBER
        for t, f in zip(tl, flags):  # the caller's marking, :3090-3095
            if f == _lib.GF_BOUND:
                flag[t] |= WP_BOUND
                flag[t] &= ~WP_REMAINING & 0xFF
                haloid[t] = j
        nmem.append(int(nb))
    unb = sp[(flag[sp] & WP_BOUND) == 0]  # UnboundShellP2Rest
    haloid[unb] = NOT_MEMBER
    flag[unb] |= WP_REMAINING
    return nmem


def member_rest_list(bp, flag, haloid, core, hid, rank, now, release):
    """GetMemberRestParticleList (:2722-2768): particles within Rtidal that are
    free, hid's own, or non-core members of a core later in the order (rank);
    with `release`, hid's own members beyond Rtidal become free REMAINING."""
    inside = within(bp, np.arange(len(bp)), core)
    if release:
        out = np.nonzero(~inside & (haloid == hid))[0]
        haloid[out] = NOT_MEMBER
        flag[out] |= WP_REMAINING
    lst = np.nonzero(inside)[0]
    ids = haloid[lst]
    later = np.array([rank.get(int(i), -1) > now for i in ids], bool) if len(lst) else np.zeros(0, bool)
    keep = (ids == NOT_MEMBER) | (ids == hid) | (((flag[lst] & WP_CORE) == 0) & later)
    return lst[keep]


def bound_pass(bp, flag, haloid, cores, order, nmem):
    """One BOUNDITER pass (:3118-3172) core by core, in place; returns the
    bound count per core of `order` (SINGLEHALO through CheckSelfTE)."""
    rank = {int(c): j for j, c in enumerate(order)}
    nb_out = []
    for j, hid in enumerate(order):
        if nmem[j] == 0:
            nb_out.append(0)
            continue
        lst = member_rest_list(bp, flag, haloid, cores[hid], hid, rank, j, True)
        if len(lst) == 0:
            nb_out.append(0)
            continue
        flags, nb = dropin.CheckSelfTE(_kp(bp, lst), bp)
        for i, f in zip(lst, flags):  # SINGLEHALO (:1868-1877)
            if f == _lib.GF_BOUND:
                haloid[i] = hid
                flag[i] &= ~WP_REMAINING & 0xFF
            elif haloid[i] == hid:
                haloid[i] = NOT_MEMBER
                flag[i] |= WP_REMAINING
        nb_out.append(int(nb))
    return nb_out
