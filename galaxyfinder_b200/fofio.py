"""The data formats on either side of the stage: the FoF halo catalogue and
member-particle files the galaxy finder reads, and the GALFIND records it
writes (NewGalFinder/gfind.c).  Host code (numpy), no device work.

Input.  A catalogue file is a sequence of HaloQ records (tree.h:55-60); the
member file holds, for each halo in catalogue order, its DM, gas, sink and
star particles as raw DmType / GasType / SinkType / StarType records
(ramses.h), in that order (FREAD, gfind.c:23-91).  FREAD turns them into the
finder's particles: type, FP64 position, velocity and mass, and the linking
length link02 = 0.2 (m / 2.7755e11 / omep)^(1/3), evaluated in long double
and stored as a float.  read_halos returns the selected halos as a HaloBatch
(the batch the GPU stage consumes) plus the raw records; halos are located by
the cumulative record sizes, so any subset is read directly.

Output.  write_data (gfind.c:690-732) writes, per halo with sub-halos, a
HaloInfo (defs.h:3-7; GetHaloInfo, gfind.c:557-617) to the data and list
files, then per sub-halo a SubInfo (defs.h:21-25; GetSubHaloInfo,
gfind.c:618-689) to both and the sub-halo's raw records (DM, gas, sink, star)
to the data file, and the background's (id NOT_HALO_MEMBER) SubInfo and
records to the background file.  The sums are sequential FP64 sums in
particle order, as the reference's loops.

The record layouts are those of the reference's build flags
(NewGalFinder/Makefile: -DXYZDBL -DNCHEM=3 -DREAD_SINK, int ids, no NBODY or
FBK): sizes 96 (HaloQ), 136 (DmType = StarType), 112 (GasType), 168
(SinkType), 112 (HaloInfo, SubInfo).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .synth import HaloBatch

TYPE_STAR, TYPE_DM, TYPE_GAS, TYPE_SINK = 1, 2, 3, 4  # tree.h:47-48
NOT_HALO_MEMBER = -9999                               # defs.h:29


def _rec(fields, itemsize):
    names, formats, offsets = zip(*fields)
    return np.dtype({"names": list(names), "formats": list(formats), "offsets": list(offsets),
                     "itemsize": itemsize})


HALOQ_DTYPE = _rec([("np", "<u8", 0), ("npstar", "<u8", 8), ("npgas", "<u8", 16), ("npdm", "<u8", 24),
                    ("npsink", "<u8", 32), ("x", "<f8", 40), ("y", "<f8", 48), ("z", "<f8", 56),
                    ("mass", "<f4", 64), ("mstar", "<f4", 68), ("mgas", "<f4", 72), ("mdm", "<f4", 76),
                    ("msink", "<f4", 80), ("vx", "<f4", 84), ("vy", "<f4", 88), ("vz", "<f4", 92)], 96)

# PmType (ramses.h:70-90): DmType and StarType
PM_DTYPE = _rec([("x", "<f8", 0), ("y", "<f8", 8), ("z", "<f8", 16), ("vx", "<f8", 24), ("vy", "<f8", 32),
                 ("vz", "<f8", 40), ("mass", "<f8", 48), ("id", "<i4", 56), ("levelp", "<i4", 60),
                 ("family", "i1", 64), ("tag", "i1", 65), ("tp", "<f8", 72), ("zp", "<f8", 80),
                 ("chem", ("<f8", (3,)), 88), ("mass0", "<f8", 112),
                 ("birth_d", "<f8", 120), ("partp", "<i4", 128)], 136)

# GasType (ramses.h:137-159)
GAS_DTYPE = _rec([("x", "<f8", 0), ("y", "<f8", 8), ("z", "<f8", 16), ("cellsize", "<f8", 24),
                  ("vx", "<f4", 32), ("vy", "<f4", 36), ("vz", "<f4", 40), ("den", "<f8", 48),
                  ("temp", "<f4", 56), ("metallicity", "<f4", 60), ("chem", ("<f4", (3,)), 64),
                  ("mass", "<f4", 76), ("potent", "<f8", 80), ("fx", "<f8", 88), ("fy", "<f8", 96),
                  ("fz", "<f8", 104)], 112)

# SinkType (ramses.h:94-104)
SINK_DTYPE = _rec([("x", "<f8", 0), ("y", "<f8", 8), ("z", "<f8", 16), ("vx", "<f8", 24), ("vy", "<f8", 32),
                   ("vz", "<f8", 40), ("mass", "<f8", 48), ("tbirth", "<f8", 56), ("Jx", "<f8", 64),
                   ("Jy", "<f8", 72), ("Jz", "<f8", 80), ("Sx", "<f8", 88), ("Sy", "<f8", 96), ("Sz", "<f8", 104),
                   ("dMsmbh", "<f8", 112), ("dMBH_coarse", "<f8", 120), ("dMEd_coarse", "<f8", 128),
                   ("Esave", "<f8", 136), ("Smag", "<f8", 144), ("eps", "<f8", 152), ("id", "<i4", 160)], 168)

# HaloInfo (defs.h:3-7) and SubInfo (defs.h:21-25)
HALOINFO_DTYPE = _rec([("nsub", "<i4", 0), ("ndm", "<i4", 4), ("nstar", "<i4", 8), ("nsink", "<i4", 12),
                       ("ngas", "<i4", 16), ("npall", "<i4", 20), ("totm", "<f8", 24), ("mdm", "<f8", 32),
                       ("mgas", "<f8", 40), ("msink", "<f8", 48), ("mstar", "<f8", 56), ("x", "<f8", 64),
                       ("y", "<f8", 72), ("z", "<f8", 80), ("vx", "<f8", 88), ("vy", "<f8", 96),
                       ("vz", "<f8", 104)], 112)
SUBINFO_DTYPE = _rec([("npdm", "<i4", 0), ("npgas", "<i4", 4), ("npsink", "<i4", 8), ("npstar", "<i4", 12),
                      ("npall", "<i4", 16), ("totm", "<f8", 24), ("mdm", "<f8", 32), ("mgas", "<f8", 40),
                      ("msink", "<f8", 48), ("mstar", "<f8", 56), ("x", "<f8", 64), ("y", "<f8", 72),
                      ("z", "<f8", 80), ("vx", "<f8", 88), ("vy", "<f8", 96), ("vz", "<f8", 104)], 112)

# member-file order of the particle kinds in FREAD (gfind.c:33-90)
KINDS = (("dm", "npdm", PM_DTYPE, TYPE_DM), ("gas", "npgas", GAS_DTYPE, TYPE_GAS),
         ("sink", "npsink", SINK_DTYPE, TYPE_SINK), ("star", "npstar", PM_DTYPE, TYPE_STAR))


def link02(mass, omep: float) -> np.ndarray:
    """0.2*pow(mass/2.7755e11L/omep, 0.33333333333333333333L) in long double,
    stored as float (gfind.c:49, FoFTPtlStruct.link02)."""
    ld = np.longdouble
    r = np.power(np.asarray(mass, np.float64).astype(ld) / ld("2.7755e11") / ld(np.float32(omep)),
                 ld("0.33333333333333333333"))
    return (ld(0.2) * r).astype(np.float32)


def read_catalogue(path) -> np.ndarray:
    """All HaloQ records of a catalogue file."""
    return np.fromfile(path, dtype=HALOQ_DTYPE)


def halo_offsets(cat: np.ndarray) -> np.ndarray:
    """Byte offset of every halo's records in the member file (+ the total)."""
    size = sum(cat[cnt].astype(np.int64) * dt.itemsize for _, cnt, dt, _ in KINDS)
    return np.concatenate([[0], np.cumsum(size)]).astype(np.int64)


@dataclass
class HaloRecords:
    """The raw records of one halo, by kind (member-file order)."""
    dm: np.ndarray
    gas: np.ndarray
    sink: np.ndarray
    star: np.ndarray

    def particles(self):
        """FREAD's particle fields in its order: type, x, y, z, vx, vy, vz, mass."""
        parts = [(self.dm, TYPE_DM), (self.gas, TYPE_GAS), (self.sink, TYPE_SINK), (self.star, TYPE_STAR)]
        out = {k: np.concatenate([np.asarray(r[k], np.float64) for r, _ in parts])
               for k in ("x", "y", "z", "vx", "vy", "vz", "mass")}
        out["type"] = np.concatenate([np.full(len(r), t, np.int32) for r, t in parts])
        return out


def read_halo_records(member_path, cat: np.ndarray, offsets: np.ndarray, h: int) -> HaloRecords:
    with open(member_path, "rb") as f:
        f.seek(int(offsets[h]))
        recs = {}
        for name, cnt, dt, _ in KINDS:
            n = int(cat[cnt][h])
            recs[name] = np.fromfile(f, dtype=dt, count=n)
            if len(recs[name]) != n:
                raise EOFError(f"member file ends inside halo {h}")
    return HaloRecords(**recs)


def read_halos(cat_path, member_path, omep: float, halos=None, min_np: int = 0):
    """The selected halos (default: every halo with at least min_np
    particles; the reference runs those with np >= 30, gfind.c:388) as a
    HaloBatch in catalogue order, plus their raw records and link02."""
    cat = read_catalogue(cat_path)
    off = halo_offsets(cat)
    if halos is None:
        halos = np.nonzero(cat["np"] >= min_np)[0]
    cols = {k: [] for k in ("x", "y", "z", "vx", "vy", "vz", "mass", "type")}
    records, counts = [], []
    for h in halos:
        r = read_halo_records(member_path, cat, off, int(h))
        p = r.particles()
        for k in cols:
            cols[k].append(p[k])
        records.append(r)
        counts.append(len(p["x"]))
    cat_n = {k: (np.concatenate(v) if v else np.zeros(0, np.int32 if k == "type" else np.float64))
             for k, v in cols.items()}
    pstart = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    hb = HaloBatch(x=cat_n["x"], y=cat_n["y"], z=cat_n["z"], vx=cat_n["vx"], vy=cat_n["vy"], vz=cat_n["vz"],
                   mass=cat_n["mass"], type=cat_n["type"], ids=np.arange(int(pstart[-1]), dtype=np.int64),
                   pstart=pstart, meta={"halos": np.asarray(halos, np.int64), "source": str(cat_path)})
    return hb, records, link02(hb.mass, omep)


def write_catalogue(cat_path, member_path, halos: list[HaloRecords]) -> None:
    """Writes halos (raw records by kind) as a catalogue / member-file pair
    (the HaloQ sums are float sums of the records, for tests and tools)."""
    cat = np.zeros(len(halos), HALOQ_DTYPE)
    with open(member_path, "wb") as f:
        for h, r in enumerate(halos):
            for name, cnt, _, _ in KINDS:
                rec = getattr(r, name)
                cat[cnt][h] = len(rec)
                rec.tofile(f)
            p = r.particles()
            cat["np"][h] = len(p["x"])
            m = p["mass"]
            tot = m.sum() if len(m) else 1.0
            cat["mass"][h] = m.sum()
            for k in ("x", "y", "z"):
                cat[k][h] = (m * p[k]).sum() / tot
            for k in ("vx", "vy", "vz"):
                cat[k][h] = (m * p[k]).sum() / tot
    cat.tofile(cat_path)


def _seqsum(a) -> float:
    """Left-to-right FP64 sum (the reference's += loops)."""
    a = np.asarray(a, np.float64)
    return float(np.cumsum(a)[-1]) if len(a) else 0.0


def halo_info(records: HaloRecords, nsub: int) -> np.ndarray:
    """GetHaloInfo (gfind.c:557-617) with nsub = mpeak."""
    p = records.particles()
    t, m = p["type"], p["mass"]
    out = np.zeros(1, HALOINFO_DTYPE)
    out["nsub"] = nsub
    for name, tcode in (("dm", TYPE_DM), ("sink", TYPE_SINK), ("star", TYPE_STAR), ("gas", TYPE_GAS)):
        sel = t == tcode
        out[{"dm": "ndm", "sink": "nsink", "star": "nstar", "gas": "ngas"}[name]] = int(sel.sum())
        out[{"dm": "mdm", "sink": "msink", "star": "mstar", "gas": "mgas"}[name]] = _seqsum(m[sel])
    totm = _seqsum(m)
    out["totm"] = totm
    out["npall"] = len(m)
    with np.errstate(invalid="ignore", divide="ignore"):
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            out[k] = np.float64(_seqsum(m * p[k])) / np.float64(totm)
    return out


def sub_info(records: HaloRecords, membership, sid: int):
    """GetSubHaloInfo (gfind.c:618-689): the SubInfo of the particles with
    membership == sid and their raw records packed DM, gas, sink, star."""
    p = records.particles()
    sel = np.asarray(membership) == sid
    t, m = p["type"][sel], p["mass"][sel]
    out = np.zeros(1, SUBINFO_DTYPE)
    for cnt, mk, tcode in (("npdm", "mdm", TYPE_DM), ("npsink", "msink", TYPE_SINK),
                           ("npstar", "mstar", TYPE_STAR), ("npgas", "mgas", TYPE_GAS)):
        out[cnt] = int((t == tcode).sum())
        out[mk] = _seqsum(m[t == tcode])
    totm = _seqsum(m)
    out["totm"] = totm
    out["npall"] = int(sel.sum())
    with np.errstate(invalid="ignore", divide="ignore"):
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            out[k] = np.float64(_seqsum(m * p[k][sel])) / np.float64(totm)
    # the records of each kind, in particle order (FREAD's order is by kind)
    n = {name: len(getattr(records, name)) for name, _, _, _ in KINDS}
    a = 0
    packed = []
    for name in ("dm", "gas", "sink", "star"):
        rec = getattr(records, name)
        packed.append(rec[sel[a:a + n[name]]].tobytes())
        a += n[name]
    return out, b"".join(packed)


def write_halo(records: HaloRecords, membership, nsub: int, data, listf=None, background=None) -> None:
    """write_data (gfind.c:690-732) for one halo with nsub > 0 sub-halos:
    file objects data (GALFIND data), listf (catalogue list) and background
    (the unassigned particles)."""
    if nsub <= 0:
        return
    hinfo = halo_info(records, nsub).tobytes()
    data.write(hinfo)
    if listf is not None:
        listf.write(hinfo)
    for i in range(nsub):
        si, recs = sub_info(records, membership, i)
        data.write(si.tobytes())
        if listf is not None:
            listf.write(si.tobytes())
        data.write(recs)
    if background is not None:
        si, recs = sub_info(records, membership, NOT_HALO_MEMBER)
        background.write(si.tobytes())
        background.write(recs)
