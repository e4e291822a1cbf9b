"""Galaxy-centre refinement on the GPU: gradient ascent of each centre on its
halo's smoothed (stellar, by default) TSC density, the refinement compared
with GalCenter's search-based centres (GalCenter/find_centers.c:25-104).

All galaxies of all halos are refined by one kernel launch
(gf_refine_centres); the meshes come from the batched TSC + smoothing
(gf_tsc_deposit + gf_gaussian_smooth) of the same halos.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr
from .batch import Context, DeviceBatch, mesh_rule, plan_meshes


def recentre(x, y, z, pstart, box=100.0):
    """Per halo: periodic unwrap (a halo spanning more than half the box is
    shifted by the box on the side that makes it compact) and x - min(x),
    as the stage's Dump2BP/mklocalize do.  Returns (positions (n, 3), the
    per-halo offsets (nhalo, 3) to add back)."""
    p = np.stack([x, y, z], 1).astype(np.float64)
    off = np.zeros((len(pstart) - 1, 3))
    for h in range(len(pstart) - 1):
        a, b = int(pstart[h]), int(pstart[h + 1])
        q = p[a:b]
        for ax in range(3):
            c = q[:, ax]
            cs = np.where(c < 0.5 * box, c + box, c)
            if c.max() - c.min() > 0.5 * box and cs.max() - cs.min() < c.max() - c.min():
                q[:, ax] = cs
        off[h] = q.min(0)
        p[a:b] = q - off[h]
    return p, off


def refine_centres(ctx: Context, x, y, z, mass, type_, pstart, starts, halo_of, ptype=_lib.TYPE_STAR,
                   max_steps=20, step_frac=0.1, rule=None, box=100.0):
    """Refined centres (ncentre, 3) in box coordinates, their densities and
    the moves taken.  starts: (ncentre, 3) box coordinates; halo_of: the halo
    of each centre."""
    pstart = np.asarray(pstart, np.int64)
    p, off = recentre(x, y, z, pstart, box)
    if rule is None:
        rule = mesh_rule(mode=_lib.MESH_REFERENCE, ptype=ptype)
    ext = np.array([p[pstart[h]:pstart[h + 1]].max(0) for h in range(len(pstart) - 1)])
    mesh, total = plan_meshes(ext, rule)
    dev = torch.device("cuda", ctx.device)
    db = DeviceBatch.from_arrays(p[:, 0], p[:, 1], p[:, 2], mass, type_, pstart, device=dev)
    mesh_dev = torch.from_numpy(mesh.view(np.uint8).copy()).to(dev)
    den = torch.empty(total, dtype=torch.float32, device=dev)
    b = db.c()
    L = lib()
    check(L.gf_tsc_deposit(ctx.handle, ctypes.byref(b), ptr(mesh_dev), ptr(mesh), ptr(den)))
    check(L.gf_gaussian_smooth(ctx.handle, db.nhalo, ptr(mesh), ptr(mesh_dev), ptr(den)))
    halo_of = np.asarray(halo_of, np.int32)
    s = np.asarray(starts, np.float64) - off[halo_of]
    # the same periodic image as the halo's particles
    s = np.where(s > 0.5 * box, s - box, np.where(s < -0.5 * box, s + box, s))
    cx, cy, cz = (torch.tensor(s[:, a].copy(), dtype=torch.float64, device=dev) for a in range(3))
    hd = torch.as_tensor(halo_of, device=dev)
    rho = torch.empty(len(s), dtype=torch.float64, device=dev)
    moves = torch.empty(len(s), dtype=torch.int32, device=dev)
    check(L.gf_refine_centres(ctx.handle, db.nhalo, ptr(mesh_dev), ptr(den), len(s), ptr(hd), ptr(cx), ptr(cy),
                              ptr(cz), max_steps, step_frac, ptr(rho), ptr(moves)))
    local = torch.stack([cx, cy, cz], 1).cpu().numpy()
    c = np.mod(local + off[halo_of], box)
    return c, rho.cpu().numpy(), moves.cpu().numpy(), dict(mesh=mesh, den=den, offset=off, start=s,
                                                           local=local)
