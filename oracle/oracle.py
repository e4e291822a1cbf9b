"""Python bindings of the oracle libraries (test infrastructure only).

* ``Restatement`` — oracle/_build/libgforacle.so, the C restatement
  (gf_oracle.c) of the reference's TSC / smoothing / findDen / kNN / W4 /
  tree-potential arithmetic.
* ``Reference`` — oracle/_ref/libgfref_{fixed,asbuilt}.so, the reference's own
  NewGalFinder C compiled from its sources by oracle/Makefile, behind the thin
  harness in oracle/ref/ref_harness.c; ``Reference("linked")`` is the same
  reference code with libgf's drop-ins linked in its place (the reference
  objects with the drop-in symbols weakened, linked with the whole libgf.a
  archive; `make -C oracle linked`), used to test the drop-in boundary inside the
  reference's own pipeline.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
RESTATEMENT = HERE / "_build" / "libgforacle.so"
REF_DIR = HERE / "_ref"
# the read-only reference tree the recipe compiles; GF_REFERENCE_SOURCE overrides
# the location this build container mounts it at
REF_SOURCE = Path(os.environ.get("GF_REFERENCE_SOURCE") or "/root/reference")

_VP, _I, _I64, _F, _D = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_float, ctypes.c_double


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def build(ref: bool = True) -> None:
    """Builds the restatement and, when the reference tree is present, the
    reference libraries (make -C oracle [ref]) and, when libgf.a exists, the
    reference linked with libgf (make -C oracle linked)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    if ref and REF_SOURCE.exists():
        subprocess.run(["make", "-s", "-C", str(HERE), f"REF={REF_SOURCE}", "ref"], check=True)
        if (HERE.parent / "galaxyfinder_b200" / "libgf.a").exists():
            subprocess.run(["make", "-s", "-C", str(HERE), f"REF={REF_SOURCE}", "linked"], check=True)


class Restatement:
    _lib = None

    def __init__(self):
        if Restatement._lib is None:
            if not RESTATEMENT.exists():
                build(ref=False)
            L = ctypes.CDLL(str(RESTATEMENT))
            L.or_tsc.argtypes = [_I64, _VP, _VP, _VP, _VP, _VP, _VP, _I, _I, _I, _D, _D, _D, _D, _I, _I, _I]
            L.or_find_den.argtypes = [_I64, _VP, _VP, _VP, _VP, _D, _D, _D, _D, _VP, _I, _I, _I]
            L.or_smooth.argtypes = [_VP, _I, _I, _I, _D, _F, _VP]
            L.or_knn_brute.argtypes = [_I64, _VP, _VP, _VP, _I, _VP, _VP]
            L.or_knn_grid.argtypes = [_I64, _VP, _VP, _VP, _I, _VP, _VP]
            L.or_sph_density.argtypes = [_I64, _I, _VP, _VP]
            L.or_star_density.argtypes = [_I64, _I, _VP, _VP, _VP, _VP, _VP]
            L.or_tree_potential.argtypes = [ctypes.c_int32, _VP, _I64, _VP, _VP, _VP, _VP, _I64,
                                            _VP, _VP, _VP, _VP, _VP, _VP, _VP]
            L.or_direct_potential.argtypes = [_I64, _VP, _VP, _VP, _VP, _I64, _VP, _VP, _VP, _VP]
            Restatement._lib = L
        self.L = Restatement._lib

    @staticmethod
    def mesh_size(nx, ny, nz):
        return 2 * (nx // 2 + 1) * ny * nz

    def tsc(self, x, y, z, mass, type_, nx, ny, nz, xmin, ymin, zmin, cellsize, ptype=5,
            acc_double=False, ref_threads=1):
        den = np.zeros(self.mesh_size(nx, ny, nz), np.float32)
        x, y, z, mass = (np.ascontiguousarray(a, np.float64) for a in (x, y, z, mass))
        t = None if type_ is None else np.ascontiguousarray(type_, np.int32)
        bad = self.L.or_tsc(len(x), _p(x), _p(y), _p(z), _p(mass), _p(t), _p(den), nx, ny, nz,
                            xmin, ymin, zmin, cellsize, ptype, int(acc_double), int(ref_threads))
        if bad:
            raise ValueError("a particle's TSC stencil falls outside the mesh")
        return den

    def find_den(self, x, y, z, den, nx, ny, nz, xmin, ymin, zmin, cellsize):
        x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
        den = np.ascontiguousarray(den, np.float32)
        out = np.zeros(len(x), np.float32)
        bad = self.L.or_find_den(len(x), _p(x), _p(y), _p(z), _p(out), xmin, ymin, zmin, cellsize,
                                 _p(den), nx, ny, nz)
        if bad:
            raise ValueError("a particle's TSC stencil falls outside the mesh")
        return out

    def smooth(self, den, nx, ny, nz, cellsize, rg):
        d = np.array(den, np.float32, copy=True)
        out64 = np.zeros(len(d), np.float64)
        self.L.or_smooth(_p(d), nx, ny, nz, cellsize, rg, _p(out64))
        return d, out64

    def knn(self, x, y, z, k, method="grid"):
        x, y, z = (np.ascontiguousarray(a, np.float32) for a in (x, y, z))
        n = len(x)
        idx = np.zeros((n, k), np.int64)
        d2 = np.zeros((n, k), np.float64)
        fn = self.L.or_knn_grid if method == "grid" else self.L.or_knn_brute
        if fn(n, _p(x), _p(y), _p(z), k, _p(idx), _p(d2)):
            raise ValueError("k larger than the number of particles")
        return idx, d2

    def sph_density(self, d2):
        d2 = np.ascontiguousarray(d2, np.float64)
        n, k = d2.shape
        out = np.zeros(n, np.float32)
        self.L.or_sph_density(n, k, _p(d2), _p(out))
        return out


    def star_density(self, d2, sidx, cnt, smass):
        """starfindsphdensity's stellar density (nnost.c:687-703) from each
        particle's k nearest stars: d2 and sidx (n, k) in distance order, cnt
        (n,) the stars found, smass the stars' masses."""
        d2 = np.ascontiguousarray(d2, np.float64)
        sidx = np.ascontiguousarray(sidx, np.int64)
        cnt = np.ascontiguousarray(cnt, np.int32)
        smass = np.ascontiguousarray(smass, np.float32)
        n, k = d2.shape
        out = np.zeros(n, np.float32)
        self.L.or_star_density(n, k, _p(d2), _p(sidx), _p(cnt), _p(smass), _p(out))
        return out

    def tree_potential(self, nodes, spos4, tpos, troot, trend, topen=None):
        """FP64 walk of an exported tree.  nodes: BH_NODE_DTYPE array;
        spos4: (n, 4) float32 tree-ordered sources; tpos: (m, 3) float32."""
        nodes = np.ascontiguousarray(nodes)
        s = np.ascontiguousarray(spos4, np.float32)
        sx, sy, sz, sm = (np.ascontiguousarray(s[:, i]) for i in range(4))
        t = np.ascontiguousarray(tpos, np.float32)
        tx, ty, tz = (np.ascontiguousarray(t[:, i]) for i in range(3))
        troot = np.ascontiguousarray(troot, np.int32)
        trend = np.ascontiguousarray(trend, np.int32)
        to = None if topen is None else np.ascontiguousarray(topen, np.int32)
        phi = np.zeros(len(t), np.float64)
        self.L.or_tree_potential(len(nodes), _p(nodes), len(s), _p(sx), _p(sy), _p(sz), _p(sm),
                                 len(t), _p(tx), _p(ty), _p(tz), _p(troot), _p(trend), _p(to),
                                 _p(phi))
        return phi

    def direct_potential(self, spos4, tpos):
        s = np.ascontiguousarray(spos4, np.float32)
        sx, sy, sz, sm = (np.ascontiguousarray(s[:, i]) for i in range(4))
        t = np.ascontiguousarray(tpos, np.float32)
        tx, ty, tz = (np.ascontiguousarray(t[:, i]) for i in range(3))
        phi = np.zeros(len(t), np.float64)
        self.L.or_direct_potential(len(s), _p(sx), _p(sy), _p(sz), _p(sm), len(t), _p(tx), _p(ty),
                                   _p(tz), _p(phi))
        return phi


class Reference:
    """The reference's own code (compiled from its sources)."""
    _libs: dict = {}

    def __init__(self, variant: str = "fixed", arena_mb: int = 4096):
        path = REF_DIR / f"libgfref_{variant}.so"
        if variant not in Reference._libs:
            if not path.exists():
                if REF_SOURCE.exists():
                    build(ref=True)
                else:
                    raise FileNotFoundError(f"{path} was not built (reference tree absent)")
            L = ctypes.CDLL(str(path))
            L.ref_init.argtypes = [ctypes.c_longlong]
            L.ref_set_cosmology.argtypes = [_F, _F, _F, _F, _F]
            for name in ("ref_get_potentfact", "ref_get_r1kineticfact", "ref_get_r2kineticfact"):
                getattr(L, name).restype = _D
            L.ref_GetBGpotent.argtypes = [_D]
            L.ref_GetBGpotent.restype = _D
            L.ref_findsphdensity.argtypes = [_I, _VP, _VP, _VP, _VP, _VP, _I, _VP]
            L.ref_starfindsphdensity.argtypes = [_I, _VP, _VP, _VP, _VP, _VP, _VP, _I, _VP]
            L.ref_lagFindStellarCore.argtypes = [_I, _VP, _VP, _VP, _VP, _VP, _I, _VP, _VP, _I, _I,
                                                 _VP, _VP, _VP]
            L.ref_assign_density_TSC.argtypes = [_I, _VP, _VP, _VP, _VP, _VP, _VP, _I, _I, _I, _D,
                                                 _D, _D, _D, _I]
            L.ref_findDen.argtypes = [_I, _VP, _VP, _VP, _VP, _D, _D, _D, _D, _VP, _I, _I, _I]
            L.ref_gaussian_Smoothing.argtypes = [_VP, _I, _I, _I, _D, _F]
            L.ref_find_near_all.argtypes = [_I, _VP, _VP, _VP, _VP, _I, _VP, _VP, _VP]
            L.ref_Self_Halo_Potent.argtypes = [_I, _VP, _VP, _VP, _VP, _VP]
            L.ref_External_Halo_Potent.argtypes = [_I, _VP, _VP, _VP, _VP, _VP, _I, _VP, _VP, _VP,
                                                   _VP]
            L.ref_tree_potential.argtypes = [_I, _VP, _VP, _VP, _VP, _F, _VP]
            L.ref_subhalo_den.argtypes = [_I, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]
            L.ref_CheckSelfTE.argtypes = [_I, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]
            L.ref_CheckExternalTE.argtypes = [_I, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _I, _VP, _VP,
                                              _VP, _VP, _VP, _VP]
            L.ref_AdGetTidalRCenterCore.argtypes = [_I, _VP, _VP, _VP, _VP, _VP, _I, _VP, _I, _VP,
                                                    _VP, _VP]
            L.ref_finddenpeak.argtypes = [_I, _VP, _VP, _I, _VP, _VP, _VP, _VP, _I, _I, _VP, _VP]
            L.ref_FindCoreDensity.argtypes = [_I, _VP, _VP, _I, _VP, _VP, _I, _VP, _VP, _VP, _VP, _VP,
                                              _VP, _VP]
            if L.ref_init(arena_mb) != 0:
                raise RuntimeError("reference arena allocation failed")
            Reference._libs[variant] = L
        self.L = Reference._libs[variant]

    @staticmethod
    def _d(a):
        return np.ascontiguousarray(a, np.float64)

    def physics(self):
        return (self.L.ref_get_potentfact(), self.L.ref_get_r1kineticfact(),
                self.L.ref_get_r2kineticfact())

    def bg_potent(self, mvir):
        return self.L.ref_GetBGpotent(mvir)

    def findsphdensity(self, x, y, z, mass, k):
        x, y, z, mass = map(self._d, (x, y, z, mass))
        n = len(x)
        idx = np.zeros(n * k, np.int64)
        dens = np.zeros(n, np.float32)
        self.L.ref_findsphdensity(n, _p(x), _p(y), _p(z), _p(mass), _p(idx), k, _p(dens))
        return idx.reshape(n, k), dens

    def starfindsphdensity(self, x, y, z, mass, type_, k):
        """nnost.c:632-744: stellar density at every particle and its k-NN list."""
        x, y, z, mass = map(self._d, (x, y, z, mass))
        t = np.ascontiguousarray(type_, np.int32)
        n = len(x)
        idx = np.zeros(n * k, np.int64)
        dens = np.zeros(n, np.float32)
        self.L.ref_starfindsphdensity(n, _p(t), _p(x), _p(y), _p(z), _p(mass), _p(idx), k, _p(dens))
        return idx.reshape(n, k), dens

    def find_near_all(self, x, y, z, mass, k):
        x, y, z = map(self._d, (x, y, z))
        m = None if mass is None else self._d(mass)
        n = len(x)
        idx = np.zeros(n * k, np.int64)
        d2 = np.zeros(n * k, np.float64)
        maxr = np.zeros(n, np.float32)
        self.L.ref_find_near_all(n, _p(x), _p(y), _p(z), _p(m), k, _p(idx), _p(d2), _p(maxr))
        return idx.reshape(n, k), d2.reshape(n, k), maxr

    def assign_density_TSC(self, x, y, z, mass, type_, nx, ny, nz, xmin, ymin, zmin, cellsize,
                           ptype=5):
        x, y, z, mass = map(self._d, (x, y, z, mass))
        t = np.ascontiguousarray(type_, np.int32)
        den = np.zeros(2 * (nx // 2 + 1) * ny * nz, np.float32)
        self.L.ref_assign_density_TSC(len(x), _p(t), _p(x), _p(y), _p(z), _p(mass), _p(den), nx,
                                      ny, nz, xmin, ymin, zmin, cellsize, ptype)
        return den

    def findDen(self, x, y, z, den, nx, ny, nz, xmin, ymin, zmin, cellsize):
        x, y, z = map(self._d, (x, y, z))
        den = np.ascontiguousarray(den, np.float32)
        out = np.zeros(len(x), np.float32)
        self.L.ref_findDen(len(x), _p(x), _p(y), _p(z), _p(out), xmin, ymin, zmin, cellsize,
                           _p(den), nx, ny, nz)
        return out

    def gaussian_Smoothing(self, den, nx, ny, nz, cellsize, rg):
        d = np.array(den, np.float32, copy=True)
        self.L.ref_gaussian_Smoothing(_p(d), nx, ny, nz, cellsize, rg)
        return d

    def lagFindStellarCore(self, x, y, z, mass, type_, k, ptype, maxcore=100000):
        x, y, z, mass = map(self._d, (x, y, z, mass))
        t = np.ascontiguousarray(type_, np.int32)
        n = len(x)
        dens = np.zeros(n, np.float32)
        idx = np.zeros(n * k, np.int64)
        ncore = np.zeros(1, np.int32)
        peak = np.zeros(maxcore, np.int32)
        xyzd = np.zeros(4 * maxcore, np.float32)
        self.L.ref_lagFindStellarCore(n, _p(t), _p(x), _p(y), _p(z), _p(mass), k, _p(dens), _p(idx),
                                      ptype, maxcore, _p(ncore), _p(peak), _p(xyzd))
        nc = int(ncore[0])
        return dens, idx.reshape(n, k), peak[:nc], xyzd[:4 * nc].reshape(nc, 4)

    def tree_potential(self, x, y, z, mass_f32, theta2=0.5):
        x, y, z = map(self._d, (x, y, z))
        m = np.ascontiguousarray(mass_f32, np.float32)
        phi = np.zeros(len(x), np.float32)
        self.L.ref_tree_potential(len(x), _p(x), _p(y), _p(z), _p(m), theta2, _p(phi))
        return phi

    def Self_Halo_Potent(self, x, y, z, mass_f32):
        x, y, z = map(self._d, (x, y, z))
        m = np.ascontiguousarray(mass_f32, np.float32)
        pe = np.zeros(len(x), np.float32)
        self.L.ref_Self_Halo_Potent(len(x), _p(x), _p(y), _p(z), _p(m), _p(pe))
        return pe

    def External_Halo_Potent(self, tx, ty, tz, tmass, sx, sy, sz, smass):
        tx, ty, tz, sx, sy, sz = map(self._d, (tx, ty, tz, sx, sy, sz))
        tm = np.ascontiguousarray(tmass, np.float32)
        sm = np.ascontiguousarray(smass, np.float32)
        pe = np.zeros(len(tx), np.float32)
        self.L.ref_External_Halo_Potent(len(tx), _p(tx), _p(ty), _p(tz), _p(tm), _p(pe), len(sx),
                                        _p(sx), _p(sy), _p(sz), _p(sm))
        return pe

    @staticmethod
    def _f(a):
        return np.ascontiguousarray(a, np.float32)

    def CheckSelfTE(self, x, y, z, vx, vy, vz, mass, type_):
        """subhaloden.mod6.c:1730 -> (bound flags, number bound)."""
        x, y, z = map(self._d, (x, y, z))
        vx, vy, vz, m = map(self._f, (vx, vy, vz, mass))
        t = np.ascontiguousarray(type_, np.int32)
        flag = np.zeros(len(x), np.uint8)
        nb = self.L.ref_CheckSelfTE(len(x), _p(x), _p(y), _p(z), _p(vx), _p(vy), _p(vz), _p(m),
                                    _p(t), _p(flag))
        return flag, nb

    def CheckExternalTE(self, x, y, z, vx, vy, vz, mass, sx, sy, sz, smass, core6):
        """subhaloden.mod6.c:1622; core6 = (cx, cy, cz, cvx, cvy, cvz)."""
        x, y, z, sx, sy, sz = map(self._d, (x, y, z, sx, sy, sz))
        vx, vy, vz, m, sm, c6 = map(self._f, (vx, vy, vz, mass, smass, core6))
        flag = np.zeros(len(x), np.uint8)
        nb = self.L.ref_CheckExternalTE(len(x), _p(x), _p(y), _p(z), _p(vx), _p(vy), _p(vz), _p(m),
                                        len(sx), _p(sx), _p(sy), _p(sz), _p(sm), _p(c6), _p(flag))
        return flag, nb

    def AdGetTidalRCenterCore(self, x, y, z, mass, haloid, core6, score_core):
        """subhaloden.mod6.c:1910 -> (Rtidal, nummem) per core; core6 is
        (numcore, 6) centres and velocities, score_core the ranked core ids."""
        x, y, z, mass = map(self._d, (x, y, z, mass))
        hid = np.ascontiguousarray(haloid, np.int32)
        c6 = np.ascontiguousarray(core6, np.float32).reshape(-1, 6)
        sc = np.ascontiguousarray(score_core, np.int32)
        nc = len(c6)
        rt = np.zeros(nc, np.float32)
        nm = np.zeros(nc, np.int32)
        self.L.ref_AdGetTidalRCenterCore(len(x), _p(x), _p(y), _p(z), _p(mass), _p(hid), nc,
                                         _p(c6), len(sc), _p(sc), _p(rt), _p(nm))
        return rt, nm

    def finddenpeak(self, den, neighbor, type_, x, y, z, jflag=0):
        """subhaloden.mod6.c:416 -> (peak particles, (npeak, 4) float cx, cy, cz, density)."""
        den = np.ascontiguousarray(den, np.float32)
        nb = np.ascontiguousarray(neighbor, np.int64)
        t = np.ascontiguousarray(type_, np.int32)
        x, y, z = map(self._d, (x, y, z))
        n, k = nb.shape
        peak = np.zeros(max(n, 1), np.int32)
        xyzd = np.zeros(4 * max(n, 1), np.float32)
        nc = self.L.ref_finddenpeak(n, _p(den), _p(nb), k, _p(t), _p(x), _p(y), _p(z), jflag, n,
                                    _p(peak), _p(xyzd))
        return peak[:nc], xyzd[:4 * nc].reshape(nc, 4)

    def FindCoreDensity(self, den, neighbor, type_, mass, peak):
        """subhaloden.mod6.c:1167, one thread -> dict of per-core coredensity,
        nummem, numstar, starmass and per-particle haloid, flag."""
        den = np.ascontiguousarray(den, np.float32)
        nb = np.ascontiguousarray(neighbor, np.int64)
        t = np.ascontiguousarray(type_, np.int32)
        m = self._d(mass)
        pk = np.ascontiguousarray(peak, np.int32)
        n, k = nb.shape
        nc = len(pk)
        out = dict(coredensity=np.zeros(nc, np.float32), nummem=np.zeros(nc, np.int32),
                   numstar=np.zeros(nc, np.int32), starmass=np.zeros(nc, np.float32),
                   haloid=np.zeros(n, np.int32), flag=np.zeros(n, np.uint8))
        self.L.ref_FindCoreDensity(n, _p(den), _p(nb), k, _p(t), _p(m), nc, _p(pk),
                                   *(_p(out[f]) for f in ("coredensity", "nummem", "numstar",
                                                          "starmass", "haloid", "flag")))
        return out

    def subhalo_den(self, x, y, z, vx, vy, vz, mass, type_):
        """subhaloden.mod6.c:2861 on one FoF halo -> (result, p2halo)."""
        x, y, z, vx, vy, vz, mass = map(self._d, (x, y, z, vx, vy, vz, mass))
        t = np.ascontiguousarray(type_, np.int32)
        p2 = np.zeros(len(x), np.int32)
        r = self.L.ref_subhalo_den(len(x), _p(t), _p(x), _p(y), _p(z), _p(vx), _p(vy), _p(vz),
                                   _p(mass), _p(p2))
        return r, p2


class ReferenceIO:
    """The reference's FoF reader (FREAD) and GALFIND writer helpers
    (GetHaloInfo, GetSubHaloInfo) from gfind.c, in oracle/_ref/libgfref_io.so
    (loaded lazily: gfind.c's MPI calls stay unresolved and are never made)."""
    _lib = None

    def __init__(self, arena_mb: int = 512):
        if ReferenceIO._lib is None:
            path = REF_DIR / "libgfref_io.so"
            if not path.exists():
                if REF_SOURCE.exists():
                    build(ref=True)
                else:
                    raise FileNotFoundError(f"{path} was not built (reference tree absent)")
            import os
            L = ctypes.CDLL(str(path), mode=os.RTLD_LAZY | os.RTLD_LOCAL)
            L.io_init.argtypes = [ctypes.c_longlong]
            L.io_layout.argtypes = [_VP]
            L.io_fread.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_longlong, _F] + [_VP] * 9 + \
                [ctypes.c_longlong]
            L.io_fread.restype = ctypes.c_longlong
            L.io_write_halo.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_longlong, _F, _I, _VP, _VP,
                                        ctypes.c_longlong]
            L.io_write_halo.restype = ctypes.c_longlong
            if L.io_init(arena_mb) != 0:
                raise RuntimeError("reference arena allocation failed")
            ReferenceIO._lib = L
        self.L = ReferenceIO._lib

    def layout(self):
        out = np.zeros(64, np.int64)
        k = self.L.io_layout(_p(out))
        return out[:k]

    def fread(self, cat, mem, index, omep, cap):
        o = {k: np.zeros(cap, np.float64) for k in ("x", "y", "z", "vx", "vy", "vz", "mass")}
        t = np.zeros(cap, np.int32)
        l02 = np.zeros(cap, np.float32)
        n = self.L.io_fread(str(cat).encode(), str(mem).encode(), index, omep, _p(t), _p(o["x"]), _p(o["y"]),
                            _p(o["z"]), _p(o["vx"]), _p(o["vy"]), _p(o["vz"]), _p(o["mass"]), _p(l02), cap)
        if n < 0:
            raise RuntimeError("io_fread failed")
        o = {k: v[:n] for k, v in o.items()}
        o["type"], o["link02"] = t[:n], l02[:n]
        return o

    def write_halo(self, cat, mem, index, omep, nsub, membership, cap=1 << 26):
        buf = np.zeros(cap, np.uint8)
        m = np.ascontiguousarray(membership, np.int64)
        n = self.L.io_write_halo(str(cat).encode(), str(mem).encode(), index, omep, nsub, _p(m), _p(buf), cap)
        if n < 0:
            raise RuntimeError("io_write_halo failed")
        return buf[:n].tobytes()


class GalCenterSearch:
    """GalCenter's own centre search (find_centers.c:25-175), from
    oracle/_ref/libgalcenter.so."""
    _lib = None

    def __init__(self, arena_mb: int = 1024):
        if GalCenterSearch._lib is None:
            path = REF_DIR / "libgalcenter.so"
            if not path.exists():
                if REF_SOURCE.exists():
                    build(ref=True)
                else:
                    raise FileNotFoundError(f"{path} was not built (reference tree absent)")
            L = ctypes.CDLL(str(path))
            L.gc_init.argtypes = [ctypes.c_longlong]
            L.gc_find_centers.argtypes = [_I, _VP, _VP, _VP, _VP, _VP, _VP]
            if L.gc_init(arena_mb) != 0:
                raise RuntimeError("GalCenter arena allocation failed")
            GalCenterSearch._lib = L
        self.L = GalCenterSearch._lib

    def find_centers(self, x, y, z, mass, type_):
        """-> (stellar centre (x, y, z, R), dark-matter centre (x, y, z, R))."""
        x, y, z, m = (np.ascontiguousarray(a, np.float64) for a in (x, y, z, mass))
        t = np.ascontiguousarray(type_, np.int32)
        out = np.zeros(8)
        self.L.gc_find_centers(len(x), _p(t), _p(x), _p(y), _p(z), _p(m), _p(out))
        return out[:4], out[4:]


def ref_available() -> bool:
    return (REF_DIR / "libgfref_fixed.so").exists() or REF_SOURCE.exists()


def cpu_threads() -> int:
    return len(os.sched_getaffinity(0))
