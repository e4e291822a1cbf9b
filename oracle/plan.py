"""Per-halo TSC mesh plan, restated in numpy (test and baseline infrastructure).

The stage sizes one padded r2c mesh per halo from its recentred extent.  The
reference does this inside lagFindStellarCore (NewGalFinder/nnost.c:1050-1056:
upper bound padded by 1e-4 of the extent, n = extent/cellsize + nbuff per
axis, origin nbuff/2 cells below the halo minimum); the stage adds two
cubic-mesh rules (a fixed n, or the smallest power of two that holds the
extent, clamped).  This restatement lets the CPU legs of the benchmark (the
reference's own functions timed on the host) plan their meshes without
loading libgf; tests/test_plan_pin.py pins it to libgf's gf_plan_meshes.
"""
from __future__ import annotations

import numpy as np

# gf_mesh_rule.mode values (include/gf.h)
MESH_REFERENCE, MESH_FIXED, MESH_POW2 = 0, 1, 2


def plan_one(ext, mode=MESH_POW2, nfixed=128, nmin=64, nmax=256, nbuff=10, cell=0.004, rg=0.008,
             rg_in_cells=False) -> dict:
    """Mesh of one halo whose recentred particles span [0, ext] per axis.
    Returns nx, ny, nz, cellsize, origin (the same on every axis) and rg."""
    e = [float(v) + float(v) * 0.0001 for v in ext]  # nnost.c:1050-1052
    cs = float(cell)
    if mode == MESH_REFERENCE:
        n = [int(v / cs + nbuff) for v in e]  # nnost.c:1053-1055 (C truncation)
    else:
        w = max(e)
        if mode == MESH_FIXED:
            nc = int(nfixed)
            cs = w / float(nc - nbuff)
            if not cs > 0:
                cs = float(cell)
        else:  # smallest power of two holding extent/cell + nbuff, clamped
            need = w / float(cell) + nbuff
            nc = 1
            while nc < need and nc < (1 << 20):
                nc <<= 1
            nc = min(max(nc, int(nmin)), int(nmax))
            cs = max(float(cell), w / float(nc - nbuff))
        n = [nc, nc, nc]
    origin = 0.0 - cs * nbuff / 2.0  # nnost.c:1056
    return {"nx": n[0], "ny": n[1], "nz": n[2], "cellsize": cs, "xmin": origin,
            "rg": rg * cs if rg_in_cells else float(rg)}


def mesh_floats(nx: int, ny: int, nz: int) -> int:
    """Padded r2c mesh size, den[i + mx*(j + ny*k)] with mx = 2(nx/2+1) (tsc_omp2.c:16)."""
    return 2 * (nx // 2 + 1) * ny * nz


def plan(extents, **rule) -> tuple[list[dict], int]:
    """Meshes of many halos and their total float count, each mesh starting
    on a 64-float (256-byte) boundary as the stage lays them out."""
    out, off = [], 0
    for ext in np.asarray(extents, np.float64).reshape(-1, 3):
        m = plan_one(ext, **rule)
        m["off"] = off
        off += mesh_floats(m["nx"], m["ny"], m["nz"])
        off = (off + 63) & ~63
        out.append(m)
    return out, off
