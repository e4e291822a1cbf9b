"""ctypes binding of libgf.so (the C ABI declared in include/gf.h).

The library is built in-tree by ``galaxyfinder_b200.build`` and loaded from
this package directory.  There is no fallback: if the library is missing or
fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

# GF_LIBGF selects another build of the library (tune.py times variants this way)
LIB_PATH = Path(os.environ.get("GF_LIBGF") or Path(__file__).resolve().parent / "libgf.so")

# status codes (gf.h)
GF_OK, GF_EINVAL, GF_ENOMEM, GF_EDEVICE, GF_ETIMEOUT, GF_ERANGE, GF_ENOTIMPL, GF_ESTALE = range(8)

# particle types (NewGalFinder/tree.h:47-48)
TYPE_STAR, TYPE_DM, TYPE_GAS, TYPE_SINK, TYPE_ALL = 1, 2, 3, 4, 5
GF_UNBOUND, GF_BOUND = 0, 1  # subhaloden.mod6.c:32-33

# SimpleBasicParticleType, NewGalFinder/tree.h:155-162 (88 bytes)
BP_DTYPE = np.dtype([
    ("type", "<u4"), ("_pad0", "<u4"), ("mass", "<f8"), ("x", "<f8"), ("y", "<f8"),
    ("z", "<f8"), ("vx", "<f8"), ("vy", "<f8"), ("vz", "<f8"), ("link02", "<f8"),
    ("indx", "<i4"), ("_pad1", "<i4"), ("bp", "<u8"),
])
assert BP_DTYPE.itemsize == 88

# Vector3d, NewGalFinder/subhaloden.mod6.c:70-72
VEC3_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8")])

# Kptype, NewGalFinder/subhaloden.mod6.c:73-77 (48 bytes)
KP_DTYPE = np.dtype([
    ("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("vx", "<f4"), ("vy", "<f4"), ("vz", "<f4"),
    ("mass", "<f4"), ("bp", "<u8"),
])
assert KP_DTYPE.itemsize == 48

# Coretype, NewGalFinder/tree.h:204-213 (56 bytes)
CORE_DTYPE = np.dtype([
    ("peak", "<i4"), ("nummem", "<i4"), ("numstar", "<i4"), ("starmass", "<f4"),
    ("coredensity", "<f4"), ("cx", "<f4"), ("cy", "<f4"), ("cz", "<f4"), ("cvx", "<f4"),
    ("cvy", "<f4"), ("cvz", "<f4"), ("Rtidal", "<f4"), ("density", "<f4"), ("flag", "u1"),
    ("_pad", "u1", (3,)),
])
assert CORE_DTYPE.itemsize == 56

# TPtlStruct, NewGalFinder/tree.h:72-77 (56 bytes): a particle of the threaded tree
TPTL_DTYPE = np.dtype([
    ("type", "<u4"), ("_pad0", "<u4"), ("sibling", "<u8"), ("x", "<f8"), ("y", "<f8"), ("z", "<f8"),
    ("mass", "<f8"), ("indx", "<i4"), ("_pad1", "<i4"),
])
assert TPTL_DTYPE.itemsize == 56

# TStruct, NewGalFinder/tree.h:79-91 (176 bytes): a node of the threaded tree
TSTRUCT_DTYPE = np.dtype([
    ("type", "<u4"), ("_pad0", "<u4"), ("sibling", "<u8"), ("daughter", "<u8"), ("L", "<f8"),
    ("dist", "<f8"), ("dist2", "<f8"), ("x0", "<f8"), ("y0", "<f8"), ("z0", "<f8"), ("mass", "<f8"),
    ("Nparticle", "<i4"), ("_pad1", "<i4"), ("monox", "<f8"), ("monoy", "<f8"), ("monoz", "<f8"),
    ("trQ", "<f8"), ("quad", "<f8", (6,)), ("dist_over_thetasq", "<f8"),
])
assert TSTRUCT_DTYPE.itemsize == 176

# particle, NewGalFinder/tree.h:145-149 (40 bytes): a query point
PARTICLE_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("link02", "<f8"),
                           ("indx", "<i4"), ("_pad", "<i4")])
assert PARTICLE_DTYPE.itemsize == 40

# gf_mesh_desc (gf.h), 64 bytes
MESH_DTYPE = np.dtype([
    ("off", "<i8"), ("nx", "<i4"), ("ny", "<i4"), ("nz", "<i4"), ("ptype", "<i4"),
    ("xmin", "<f8"), ("ymin", "<f8"), ("zmin", "<f8"), ("cellsize", "<f8"), ("rg", "<f8"),
])
assert MESH_DTYPE.itemsize == 64

MESH_REFERENCE, MESH_FIXED, MESH_POW2 = 0, 1, 2


class MeshRule(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32), ("nfixed", ctypes.c_int32), ("nmin", ctypes.c_int32),
        ("nmax", ctypes.c_int32), ("nbuff", ctypes.c_int32), ("ptype", ctypes.c_int32),
        ("rg_in_cells", ctypes.c_int32), ("reserved", ctypes.c_int32),
        ("cell", ctypes.c_double), ("rg", ctypes.c_double),
    ]


class Batch(ctypes.Structure):
    _fields_ = [
        ("nhalo", ctypes.c_int32), ("nparticle", ctypes.c_int64), ("pstart", ctypes.c_void_p),
        ("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("z", ctypes.c_void_p),
        ("mass", ctypes.c_void_p), ("type", ctypes.c_void_p),
    ]


class Physics(ctypes.Structure):
    _fields_ = [
        ("amax", ctypes.c_float), ("a", ctypes.c_float), ("omep", ctypes.c_float),
        ("omeplam", ctypes.c_float), ("hubble", ctypes.c_float),
        ("potentfact", ctypes.c_double), ("r1kineticfact", ctypes.c_double),
        ("r2kineticfact", ctypes.c_double),
    ]


class TreeInfo(ctypes.Structure):
    _fields_ = [("nparticle", ctypes.c_int64), ("nhalo", ctypes.c_int32), ("nnode", ctypes.c_int32)]


class StageConfig(ctypes.Structure):
    _fields_ = [
        ("mesh", MeshRule), ("box", ctypes.c_double), ("knn_k", ctypes.c_int32),
        ("do_mesh", ctypes.c_int32), ("do_potential", ctypes.c_int32), ("ndirect", ctypes.c_int32),
        ("theta2", ctypes.c_float), ("add_bg", ctypes.c_int32), ("q5_asbuilt", ctypes.c_int32),
        ("count_work", ctypes.c_int32), ("potentfact", ctypes.c_double),
        ("mesh_onchip", ctypes.c_int32), ("plain_fp64", ctypes.c_int32),
    ]


class StageOut(ctypes.Structure):
    _fields_ = [
        ("nearindex", ctypes.c_void_p), ("dens_sph", ctypes.c_void_p),
        ("dens_mesh", ctypes.c_void_p), ("penergy", ctypes.c_void_p), ("xr", ctypes.c_void_p),
        ("yr", ctypes.c_void_p), ("zr", ctypes.c_void_p), ("phi", ctypes.c_void_p),
    ]


class StageStats(ctypes.Structure):
    _fields_ = [
        ("nparticle", ctypes.c_int64), ("nnode", ctypes.c_int64), ("mesh_cells", ctypes.c_int64),
        ("nhalo", ctypes.c_int32), ("reserved", ctypes.c_int32),
        ("pp_interactions", ctypes.c_uint64), ("pc_interactions", ctypes.c_uint64),
        ("ms_recentre", ctypes.c_float), ("ms_tree", ctypes.c_float), ("ms_knn", ctypes.c_float),
        ("ms_tsc", ctypes.c_float), ("ms_smooth", ctypes.c_float), ("ms_findden", ctypes.c_float),
        ("ms_potential", ctypes.c_float), ("ms_pad", ctypes.c_float),
        ("knn_nodes", ctypes.c_uint64), ("knn_batches", ctypes.c_uint64),
        ("knn_candidates", ctypes.c_uint64), ("knn_single_inserts", ctypes.c_uint64),
        ("knn_bitonic_merges", ctypes.c_uint64),
        ("mesh_cells_device", ctypes.c_int64), ("onchip_meshes", ctypes.c_int64),
        ("onchip_particles", ctypes.c_int64), ("mesh_pass_cells", ctypes.c_int64),
    ]


# preorder node records exported by gf_tree_export
BH_NODE_DTYPE = np.dtype([
    ("com", "<f8", (3,)), ("open_r2", "<f8"), ("mass", "<f4"), ("trq", "<f4"), ("q", "<f4", (6,)),
    ("skip", "<i4"), ("lstart", "<i4"), ("lcount", "<i4"), ("count", "<i4"),
])
KNN_NODE_DTYPE = np.dtype([
    ("lo", "<f4", (3,)), ("hi", "<f4", (3,)), ("skip", "<i4"), ("lstart", "<i4"),
    ("lcount", "<i4"), ("count", "<i4"), ("parent", "<i4"), ("pad", "<i4"),
])
assert BH_NODE_DTYPE.itemsize == 80 and KNN_NODE_DTYPE.itemsize == 48


class GFError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"libgf status {status}: {msg}")
        self.status = status


_lib = None

_VP, _I32, _I64, _F, _D = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float, ctypes.c_double
_INT = ctypes.c_int

# name -> (restype, argtypes)
SIGNATURES = {
    "gf_status_string": (ctypes.c_char_p, [_INT]),
    "gf_last_status": (_INT, []),
    "gf_last_error": (ctypes.c_char_p, []),
    "gf_set_device": (_INT, [_INT]),
    "gf_kernel_launch_count": (ctypes.c_uint64, []),
    "gf_tuning_value": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]),
    "gf_set_cosmology": (_INT, [_F, _F, _F, _F, _F]),
    "gf_get_physics": (_INT, [ctypes.POINTER(Physics)]),
    "gf_bg_potent": (_D, [_D]),
    "assign_density_TSC": (None, [_VP, _INT, _VP, _INT, _INT, _INT, _D, _D, _D, _D, _INT]),
    "findDen": (None, [_VP, _INT, _VP, _D, _D, _D, _D, _VP, _INT, _INT, _INT]),
    "gaussian_Smoothing": (None, [_VP, _INT, _INT, _INT, _D, _F]),
    "findsphdensity": (None, [_VP, _INT, _VP, _INT, _VP]),
    "starfindsphdensity": (None, [_VP, _INT, _VP, _INT, _VP]),
    "Self_Halo_Potent": (None, [_INT, _VP, _VP, _VP]),
    "new_Make_Tree_Near": (None, [_VP, ctypes.c_size_t, _VP, ctypes.c_size_t, _INT]),
    "Make_Tree": (None, [_VP, ctypes.c_size_t, _VP, ctypes.c_size_t, _F, _INT]),
    "Find_Near": (_INT, [_VP, _INT, _VP, _VP, _VP, _VP, _VP, _VP]),
    "treeplumpotential": (_F, [_VP, _F, _VP, _VP]),
    "External_Halo_Potent": (None, [_INT, _VP, _VP, _VP, _INT, _VP, _VP]),
    "i_potent_spline": (None, []),
    "lagFindStellarCore": (None, [_VP, _INT, _INT, _VP, _VP, _VP, _INT, _VP, _INT]),
    "CheckSelfTE": (_INT, [_VP, _INT, _VP, _VP]),
    "CheckExternalTE": (_INT, [_VP, _INT, _VP, _VP, _INT, _VP]),
    "gf_tidal_radius": (_INT, [_VP, _INT, _VP, _INT, _VP, _VP, _INT]),
    "gf_tidal_select": (_INT, [_VP, _INT, _VP, _INT, _F, _F, _F, _F, _VP, ctypes.POINTER(_INT)]),
    "gf_ctx_create": (_INT, [ctypes.POINTER(_VP), _INT, _VP]),
    "gf_ctx_destroy": (_INT, [_VP]),
    "gf_ctx_set_stream": (_INT, [_VP, _VP]),
    "gf_plan_meshes": (_INT, [_I32, _VP, ctypes.POINTER(MeshRule), _VP, ctypes.POINTER(_I64)]),
    "gf_mesh_stage": (_INT, [_VP, ctypes.POINTER(Batch), _VP, _VP, _VP, _VP, _INT]),
    "gf_tsc_deposit": (_INT, [_VP, ctypes.POINTER(Batch), _VP, _VP, _VP]),
    "gf_gaussian_smooth": (_INT, [_VP, _I32, _VP, _VP, _VP]),
    "gf_gaussian_smooth_noalloc": (_INT, [_VP, _INT, _INT, _INT, _D, _F, _VP]),
    "gf_find_den": (_INT, [_VP, ctypes.POINTER(Batch), _VP, _VP, _VP]),
    "gf_tree_build": (_INT, [_VP, _I32, _I64, _VP, _VP, _F, _INT, ctypes.POINTER(TreeInfo)]),
    "gf_tree_export": (_INT, [_VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "gf_knn_density": (_INT, [_VP, _I32, _I64, _VP, _VP, _INT, _VP, _VP]),
    "gf_knn_query": (_INT, [_VP, _I32, _I64, _VP, _VP, _INT, _I64, _VP, _VP, _VP]),
    "gf_knn_density_adjoint": (_INT, [_VP, _I32, _I64, _VP, _VP, _VP, _VP, _INT, _I64, _VP, _VP,
                                      _VP, _VP, _VP, _VP]),
    "gf_tsc_adjoint": (_INT, [_VP, ctypes.POINTER(Batch), _VP, _VP, _VP, _VP, _VP, _VP]),
    "gf_find_den_adjoint": (_INT, [_VP, ctypes.POINTER(Batch), _VP, _VP, _VP, _VP, _VP, _VP,
                                   _VP]),
    "gf_refine_centres": (_INT, [_VP, _I32, _VP, _VP, _I32, _VP, _VP, _VP, _VP, _INT, _D, _VP, _VP]),
    "gf_density_peaks": (_INT, [_VP, _I32, _INT, _VP, _VP, _VP, _D, _I32, _VP, _VP]),
    "gf_core_density": (_INT, [_VP, _I32, _INT, _VP, _VP, _VP, _VP, _I32, _VP, _VP, _VP, _VP, _VP, _VP,
                               _VP]),
    "finddenpeak": (_INT, [_VP, _INT, _VP, _INT, _VP, _INT, _VP]),
    "FindCoreDensity": (_INT, [_VP, _INT, _VP, _INT, _VP, _INT]),
    "gf_mesh_peaks": (_INT, [_VP, _I32, _VP, _VP, _VP, _INT, _F, _I64, _VP, _VP, _VP,
                             ctypes.POINTER(_I64)]),
    "gf_self_potential": (_INT, [_VP, _I32, _I64, _VP, _VP, _F, _I32, _D, _INT, _VP, _VP]),
    "gf_bg_potent_device": (_INT, [_VP, _I32, _VP, _VP]),
    "mkRtidal": (None, []),
    "nfw_rtidal": (_F, [_F, _F, _F]),
    "gf_nfw_rtidal_cells": (_INT, []),
    "gf_nfw_rtidal_table": (_INT, [_VP, _VP]),
    "gf_nfw_rtidal_lookup": (_INT, [_VP, _I64, _VP, _VP, _VP, _VP, _VP]),
    "gf_stage_run": (_INT, [_VP, ctypes.POINTER(Batch), ctypes.POINTER(StageConfig),
                            ctypes.POINTER(StageOut), ctypes.POINTER(StageStats)]),
    "gf_stage_graph_create": (_INT, [_VP, ctypes.POINTER(Batch), ctypes.POINTER(StageConfig),
                                     ctypes.POINTER(StageOut), ctypes.POINTER(_VP)]),
    "gf_stage_graph_launch": (_INT, [_VP]),
    "gf_bound_pass": (_INT, [_VP, _INT, _VP, _VP, _VP, _INT, _VP, _VP, _INT, _VP, _VP]),
    "gf_shell_bound": (_INT, [_VP, _INT, _VP, _VP, _VP, _VP, _VP, _VP, _INT, _INT, _VP, _INT, _VP, _INT, _VP,
                              _VP]),
    "gf_stage_graph_sync": (_INT, [_VP]),
    "gf_stage_graph_run": (_INT, [_VP, ctypes.POINTER(_I32)]),
    "gf_stage_graph_replans": (_INT, [_VP]),
    "gf_stage_graph_nodes": (_INT, [_VP, ctypes.POINTER(_I32), ctypes.POINTER(_I32)]),
    "gf_stage_graph_destroy": (None, [_VP]),
}


def lib() -> ctypes.CDLL:
    """Loads libgf.so (once).  Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(
                f"{LIB_PATH} is not built; run `python -m galaxyfinder_b200.build`")
        # the void drop-ins exit(99) on error like the reference unless
        # GF_NOEXIT is set; from Python, errors are raised instead
        os.environ.setdefault("GF_NOEXIT", "1")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != GF_OK:
        msg = lib().gf_last_error().decode(errors="replace")
        raise GFError(status, msg or lib().gf_status_string(status).decode())


def check_last() -> None:
    """Raises if the last drop-in (void) call on this thread failed."""
    check(lib().gf_last_status())


def ptr(a) -> int:
    """Address of a numpy array or a torch tensor (host or device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def tuning_value(name: str) -> int:
    """A compile-time launch parameter of the loaded libgf (gf_tuning.cuh)."""
    v = ctypes.c_int64()
    check(lib().gf_tuning_value(name.encode(), ctypes.byref(v)))
    return int(v.value)


def exported_symbols() -> list[str]:
    return list(SIGNATURES)


def default_device() -> int:
    return int(os.environ.get("GF_DEVICE", "0"))
