"""Device-side batched API: many halos per call, torch tensors as device
buffers, libgf kernels through the C ABI (gf.h, native layer)."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import MESH_DTYPE, Batch, MeshRule, check, lib, ptr


class Context:
    """Owns a gf_ctx bound to a CUDA device and stream (default: torch's
    current stream, so libgf kernels order with torch work)."""

    def __init__(self, device: int = 0, stream: torch.cuda.Stream | None = None):
        self.device = device
        with torch.cuda.device(device):
            s = stream if stream is not None else torch.cuda.current_stream(device)
        self.stream = s
        h = ctypes.c_void_p()
        check(lib().gf_ctx_create(ctypes.byref(h), device, ctypes.c_void_p(s.cuda_stream)))
        self.handle = h

    def close(self):
        if self.handle:
            lib().gf_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceBatch:
    """Concatenated halos in device memory (FP64 positions and masses)."""

    def __init__(self, x, y, z, mass, type_, pstart):
        self.x, self.y, self.z, self.mass = x, y, z, mass
        self.type = type_
        self.pstart = pstart
        self.nhalo = int(pstart.numel() - 1)
        self.n = int(x.numel())

    @classmethod
    def from_arrays(cls, x, y, z, mass, type_, pstart, device="cuda:0"):
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=device)
        return cls(t(x, torch.float64), t(y, torch.float64), t(z, torch.float64),
                   t(mass, torch.float64), t(type_, torch.int32), t(pstart, torch.int64))

    @classmethod
    def from_halobatch(cls, hb, device="cuda:0"):
        return cls.from_arrays(hb.x, hb.y, hb.z, hb.mass, hb.type, hb.pstart, device)

    def c(self) -> Batch:
        return Batch(self.nhalo, self.n, ptr(self.pstart), ptr(self.x), ptr(self.y), ptr(self.z),
                     ptr(self.mass), ptr(self.type))


def mesh_rule(mode=_lib.MESH_REFERENCE, nfixed=128, nmin=64, nmax=256, nbuff=10,
              ptype=_lib.TYPE_ALL, cell=0.004, rg=0.008, rg_in_cells=False) -> MeshRule:
    return MeshRule(mode, nfixed, nmin, nmax, nbuff, ptype, int(rg_in_cells), 0, cell, rg)


def plan_meshes(extent: np.ndarray, rule: MeshRule):
    """One mesh per halo from recentred extents (nhalo, 3); returns the
    gf_mesh_desc array and the total float count of all meshes."""
    extent = np.ascontiguousarray(extent, np.float64).reshape(-1, 3)
    nh = len(extent)
    out = np.zeros(nh, MESH_DTYPE)
    total = ctypes.c_int64()
    check(lib().gf_plan_meshes(nh, ptr(extent), ctypes.byref(rule), ptr(out), ctypes.byref(total)))
    return out, int(total.value)


def mesh_stage(ctx: Context, batch: DeviceBatch, mesh: np.ndarray, total: int, smooth=True):
    """TSC deposit -> Gaussian smoothing -> findDen for every halo of the batch
    (positions must be in each mesh's frame).  Returns (den, densph)."""
    dev = batch.x.device
    mesh_dev = torch.from_numpy(mesh.view(np.uint8)).to(dev)
    den = torch.empty(total, dtype=torch.float32, device=dev)
    densph = torch.empty(batch.n, dtype=torch.float32, device=dev)
    b = batch.c()
    check(lib().gf_mesh_stage(ctx.handle, ctypes.byref(b), ptr(mesh_dev), ptr(mesh), ptr(den),
                              ptr(densph), int(smooth)))
    return den, densph
