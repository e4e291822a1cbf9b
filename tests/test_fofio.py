"""CPU: the FoF catalogue reader and GALFIND writer (galaxyfinder_b200/fofio.py)
against the reference's own gfind.c (FREAD, GetHaloInfo, GetSubHaloInfo)
compiled into the oracle: record layouts (sizes and field offsets of the
reference build), every particle field FREAD produces including the long
double linking length, and the HaloInfo / SubInfo records and packed
particle records write_data emits."""
import numpy as np
import pytest

from galaxyfinder_b200 import fofio as F
from oracle.oracle import ReferenceIO

OMEP = 0.3


@pytest.fixture(scope="module")
def rio():
    return ReferenceIO()


def _halo(rng, ndm, ngas, nsink, nstar):
    def fill(dt, n, mlog):
        r = np.zeros(n, dt)
        for name in dt.names:
            f = r[name]
            if np.issubdtype(f.dtype, np.floating):
                r[name] = rng.uniform(-1, 1, f.shape)
        for k in ("x", "y", "z"):
            r[k] = 30.0 + rng.random(n)
        for k in ("vx", "vy", "vz"):
            r[k] = rng.normal(0, 300, n)
        r["mass"] = 10 ** rng.uniform(*mlog, n)
        if "id" in dt.names:
            r["id"] = rng.integers(0, 2 ** 31 - 1, n)
        return r
    return F.HaloRecords(dm=fill(F.PM_DTYPE, ndm, (8, 9)), gas=fill(F.GAS_DTYPE, ngas, (6, 7.5)),
                         sink=fill(F.SINK_DTYPE, nsink, (5, 6)), star=fill(F.PM_DTYPE, nstar, (6, 7)))


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    rng = np.random.default_rng(17)
    halos = [_halo(rng, 200, 50, 2, 80), _halo(rng, 25, 0, 0, 3), _halo(rng, 0, 10, 1, 40),
             _halo(rng, 1000, 300, 0, 500)]
    d = tmp_path_factory.mktemp("fof")
    cat, mem = d / "FoF_halo_cat", d / "FoF_member_particle"
    F.write_catalogue(cat, mem, halos)
    return cat, mem, halos


def test_layouts_match_the_reference_build(rio):
    lay = rio.layout()
    want = [F.HALOQ_DTYPE.itemsize] + [F.HALOQ_DTYPE.fields[f][1] for f in
                                       ("np", "npstar", "npgas", "npdm", "npsink", "x", "mass", "vx")]
    want += [F.PM_DTYPE.itemsize] + [F.PM_DTYPE.fields[f][1] for f in
                                     ("x", "mass", "id", "levelp", "family", "tag", "tp", "zp", "chem",
                                      "mass0", "birth_d", "partp")]
    want += [F.GAS_DTYPE.itemsize] + [F.GAS_DTYPE.fields[f][1] for f in
                                      ("x", "cellsize", "vx", "den", "temp", "metallicity", "chem", "mass",
                                       "potent")]
    want += [F.SINK_DTYPE.itemsize] + [F.SINK_DTYPE.fields[f][1] for f in
                                       ("x", "mass", "tbirth", "Jx", "Sx", "dMsmbh", "Esave", "id")]
    want += [F.PM_DTYPE.itemsize]  # StarType
    want += [F.HALOINFO_DTYPE.itemsize] + [F.HALOINFO_DTYPE.fields[f][1] for f in ("nsub", "totm", "x")]
    want += [F.SUBINFO_DTYPE.itemsize] + [F.SUBINFO_DTYPE.fields[f][1] for f in ("npdm", "totm", "x")]
    np.testing.assert_array_equal(lay, want)


def test_reader_matches_fread(rio, files):
    cat, mem, halos = files
    hb, recs, l02 = F.read_halos(cat, mem, OMEP)
    assert hb.nhalo == len(halos)
    for h in range(hb.nhalo):
        a, b = int(hb.pstart[h]), int(hb.pstart[h + 1])
        ref = rio.fread(cat, mem, h, np.float32(OMEP), 4096)
        np.testing.assert_array_equal(hb.type[a:b], ref["type"])
        for k in ("x", "y", "z", "vx", "vy", "vz", "mass"):
            np.testing.assert_array_equal(getattr(hb, k)[a:b], ref[k], err_msg=k)
        np.testing.assert_array_equal(l02[a:b], ref["link02"])


def test_reader_subsets(files):
    cat, mem, halos = files
    hb, _, _ = F.read_halos(cat, mem, OMEP, min_np=30)  # the halos the reference runs
    np.testing.assert_array_equal(hb.meta["halos"], [0, 2, 3])
    sub, _, _ = F.read_halos(cat, mem, OMEP, halos=[3, 0])
    full, _, _ = F.read_halos(cat, mem, OMEP)
    np.testing.assert_array_equal(sub.x[: int(sub.pstart[1])], full.x[int(full.pstart[3]):int(full.pstart[4])])


def _parse(buf, nsub):
    """HaloInfo, then per sub-halo and the background: SubInfo + records."""
    off = 0
    hinfo = np.frombuffer(buf, F.HALOINFO_DTYPE, 1, off)
    off += F.HALOINFO_DTYPE.itemsize
    subs = []
    for _ in range(nsub + 1):
        si = np.frombuffer(buf, F.SUBINFO_DTYPE, 1, off)
        off += F.SUBINFO_DTYPE.itemsize
        recs = {}
        for name, cnt, dt, _ in F.KINDS:
            n = int(si[cnt][0])
            recs[name] = np.frombuffer(buf, dt, n, off)
            off += n * dt.itemsize
        subs.append((si, recs))
    assert off == len(buf)
    return hinfo, subs


def _same_records(a, b):
    assert a.dtype == b.dtype and len(a) == len(b)
    for f in a.dtype.names:  # field by field: padding bytes are not data
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)


def test_writer_matches_reference(rio, files, tmp_path):
    cat, mem, halos = files
    rng = np.random.default_rng(5)
    for h, nsub in ((0, 3), (3, 5)):
        n = sum(len(getattr(halos[h], k)) for k in ("dm", "gas", "sink", "star"))
        memb = rng.integers(-1, nsub, n)
        memb[memb < 0] = F.NOT_HALO_MEMBER
        ref = rio.write_halo(cat, mem, h, np.float32(OMEP), nsub, memb)
        with open(tmp_path / "d", "wb") as d, open(tmp_path / "l", "wb") as lf, open(tmp_path / "b", "wb") as bg:
            F.write_halo(halos[h], memb, nsub, d, lf, bg)
        ours = (tmp_path / "d").read_bytes() + (tmp_path / "b").read_bytes()
        (h0, s0), (h1, s1) = _parse(ref, nsub), _parse(ours, nsub)
        assert h0.tobytes() == h1.tobytes()
        for (si0, r0), (si1, r1) in zip(s0, s1):
            _same_records(si0, si1)  # SubInfo has 4 padding bytes
            for k in r0:
                _same_records(r0[k], r1[k])
        # the list file holds the HaloInfo and the SubInfos
        lst = (tmp_path / "l").read_bytes()
        assert len(lst) == F.HALOINFO_DTYPE.itemsize + nsub * F.SUBINFO_DTYPE.itemsize
        assert lst[:F.HALOINFO_DTYPE.itemsize] == h0.tobytes()


def test_empty_subhalo_and_single_kind_halo(rio, tmp_path):
    """A halo of stars only, written with a sub-halo that has no member: the
    reference divides its zero sums by a zero mass (NaN centre); so does the
    writer."""
    rng = np.random.default_rng(9)
    halos = [_halo(rng, 0, 0, 0, 60)]
    cat, mem = tmp_path / "cat", tmp_path / "mem"
    F.write_catalogue(cat, mem, halos)
    hb, _, _ = F.read_halos(cat, mem, OMEP)
    assert hb.n == 60 and np.all(hb.type == F.TYPE_STAR)
    memb = np.zeros(60, np.int64)  # every particle in sub-halo 0; sub-halo 1 empty
    ref = rio.write_halo(cat, mem, 0, np.float32(OMEP), 2, memb)
    with open(tmp_path / "d", "wb") as d, open(tmp_path / "b", "wb") as bg:
        F.write_halo(halos[0], memb, 2, d, None, bg)
    ours = (tmp_path / "d").read_bytes() + (tmp_path / "b").read_bytes()
    (h0, s0), (h1, s1) = _parse(ref, 2), _parse(ours, 2)
    assert h0.tobytes() == h1.tobytes()
    for (si0, _), (si1, _) in zip(s0, s1):
        for f in si0.dtype.names:
            a, b = si0[f], si1[f]
            if np.issubdtype(a.dtype, np.floating):
                np.testing.assert_array_equal(np.isnan(a), np.isnan(b), err_msg=f)
                np.testing.assert_array_equal(a[~np.isnan(a)], b[~np.isnan(b)], err_msg=f)
            else:
                np.testing.assert_array_equal(a, b, err_msg=f)
    assert np.isnan(s1[1][0]["x"][0]) and s1[1][0]["npall"][0] == 0
