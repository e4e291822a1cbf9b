"""Differentiable density: torch.autograd.Functions over libgf's forward and
hand-written adjoint kernels (gf.h: gf_tsc_adjoint, gf_find_den_adjoint,
gf_knn_density_adjoint; the Gaussian smoothing is its own adjoint).

* ``MeshDensity``   S = smooth(TSC(x, m))            (mesh; gradients in x, m)
* ``MeshDensityAt`` rho_p = findDen(S)(x_p)          (backward recomputes S)
* ``KnnDensity``    rho_i = sum_j W4(d_ij, r_k/2)    at query particles (gradients in x)

Positions are FP64 CUDA tensors in each mesh's frame (recentred, as the
stage's Dump2BP), masses FP64; everything runs on libgf's CUDA kernels.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import Batch, check, lib, ptr
from .batch import Context, plan_meshes


def _pos4_unit_mass(x, y, z):
    """FP32 (x, y, z, 1) rows: the kNN octree is built with unit masses, as
    lagFindStellarCore's all-particle kNN (nnost.c:1361-1536)."""
    return torch.stack([x.float(), y.float(), z.float(), torch.ones_like(x, dtype=torch.float32)],
                       1).contiguous()


class MeshPlan:
    """Meshes of a batch (gf_mesh_desc per halo) plus the context they run on."""

    def __init__(self, ctx: Context, pstart, mesh: np.ndarray, total: int, type_=None):
        self.ctx = ctx
        dev = torch.device("cuda", ctx.device)
        self.pstart = torch.as_tensor(np.asarray(pstart, np.int64), device=dev)
        self.nhalo = int(self.pstart.numel() - 1)
        self.mesh = np.ascontiguousarray(mesh)
        self.mesh_dev = torch.from_numpy(self.mesh.view(np.uint8).copy()).to(dev)
        self.total = int(total)
        self.type = None if type_ is None else torch.as_tensor(np.asarray(type_, np.int32), device=dev)

    @classmethod
    def for_positions(cls, ctx: Context, pstart, pos: np.ndarray, rule, type_=None):
        ps = np.asarray(pstart, np.int64)
        ext = np.array([pos[ps[h]:ps[h + 1]].max(0) for h in range(len(ps) - 1)])
        mesh, total = plan_meshes(ext, rule)
        return cls(ctx, ps, mesh, total, type_)

    def batch(self, x, y, z, m) -> Batch:
        return Batch(self.nhalo, int(x.numel()), ptr(self.pstart), ptr(x), ptr(y), ptr(z), ptr(m),
                     ptr(self.type))

    def density_mesh(self, x, y, z, m) -> torch.Tensor:
        den = torch.empty(self.total, dtype=torch.float32, device=x.device)
        b = self.batch(x, y, z, m)
        L = lib()
        check(L.gf_tsc_deposit(self.ctx.handle, ctypes.byref(b), ptr(self.mesh_dev), ptr(self.mesh), ptr(den)))
        check(L.gf_gaussian_smooth(self.ctx.handle, self.nhalo, ptr(self.mesh), ptr(self.mesh_dev), ptr(den)))
        return den

    def smooth_(self, g: torch.Tensor) -> torch.Tensor:
        check(lib().gf_gaussian_smooth(self.ctx.handle, self.nhalo, ptr(self.mesh), ptr(self.mesh_dev), ptr(g)))
        return g

    def tsc_adjoint(self, x, y, z, m, G, gx, gy, gz, gm):
        b = self.batch(x, y, z, m)
        check(lib().gf_tsc_adjoint(self.ctx.handle, ctypes.byref(b), ptr(self.mesh_dev), ptr(G), ptr(gx),
                                   ptr(gy), ptr(gz), ptr(gm)))

    def peaks(self, S: torch.Tensor, margin=1, threshold=0.0, cap=1 << 20):
        """Strict 26-neighbour maxima: (halo, cell offset within its mesh, value),
        sorted by decreasing value."""
        dev = S.device
        while True:
            oh = torch.empty(cap, dtype=torch.int32, device=dev)
            oc = torch.empty(cap, dtype=torch.int64, device=dev)
            ov = torch.empty(cap, dtype=torch.float32, device=dev)
            n = ctypes.c_int64()
            check(lib().gf_mesh_peaks(self.ctx.handle, self.nhalo, ptr(self.mesh), ptr(self.mesh_dev), ptr(S),
                                      margin, threshold, cap, ptr(oh), ptr(oc), ptr(ov), ctypes.byref(n)))
            if n.value <= cap:
                break
            cap = int(n.value)
        k = int(n.value)
        h, c, v = oh[:k].cpu().numpy(), oc[:k].cpu().numpy(), ov[:k].cpu().numpy()
        order = np.lexsort((c, h, -v))
        return h[order], c[order], v[order]


class MeshDensity(torch.autograd.Function):
    """S = smooth(TSC deposit of (x, m)) on the plan's meshes."""

    @staticmethod
    def forward(ctx, x, y, z, m, plan: MeshPlan):
        ctx.plan = plan
        ctx.save_for_backward(x, y, z, m)
        return plan.density_mesh(x, y, z, m)

    @staticmethod
    def backward(ctx, gS):
        x, y, z, m = ctx.saved_tensors
        plan = ctx.plan
        G = plan.smooth_(gS.detach().to(torch.float32).contiguous().clone())
        gx, gy, gz, gm = (torch.zeros_like(x) for _ in range(4))
        plan.tsc_adjoint(x, y, z, m, G, gx, gy, gz, gm)
        return gx, gy, gz, gm, None


class MeshDensityAt(torch.autograd.Function):
    """rho_p = findDen of the smoothed TSC mesh at every particle.  The mesh is
    recomputed in backward instead of being kept."""

    @staticmethod
    def forward(ctx, x, y, z, m, plan: MeshPlan):
        ctx.plan = plan
        ctx.save_for_backward(x, y, z, m)
        S = plan.density_mesh(x, y, z, m)
        rho = torch.empty(x.numel(), dtype=torch.float32, device=x.device)
        b = plan.batch(x, y, z, m)
        check(lib().gf_find_den(plan.ctx.handle, ctypes.byref(b), ptr(plan.mesh_dev), ptr(S), ptr(rho)))
        return rho

    @staticmethod
    def backward(ctx, grho):
        x, y, z, m = ctx.saved_tensors
        plan = ctx.plan
        S = plan.density_mesh(x, y, z, m)  # recomputed
        gd = grho.detach().to(torch.float64).contiguous()
        gx, gy, gz, gm = (torch.zeros_like(x) for _ in range(4))
        gS = torch.zeros(plan.total, dtype=torch.float32, device=x.device)
        b = plan.batch(x, y, z, m)
        check(lib().gf_find_den_adjoint(plan.ctx.handle, ctypes.byref(b), ptr(plan.mesh_dev), ptr(S), ptr(gd),
                                        ptr(gS), ptr(gx), ptr(gy), ptr(gz)))
        plan.smooth_(gS)
        plan.tsc_adjoint(x, y, z, m, gS, gx, gy, gz, gm)
        return gx, gy, gz, gm, None


def knn_query(ctx: Context, pstart, x, y, z, qidx, k=32):
    """k nearest neighbours (halo-local indices) and W4 density of the
    particles qidx, on the FP32-rounded positions."""
    dev = x.device
    ps = torch.as_tensor(np.asarray(pstart, np.int64), device=dev)
    pos4 = _pos4_unit_mass(x, y, z)
    q = torch.as_tensor(qidx, device=dev, dtype=torch.int64).contiguous()
    near = torch.empty((q.numel(), k), dtype=torch.int32, device=dev)
    dens = torch.empty(q.numel(), dtype=torch.float32, device=dev)
    check(lib().gf_knn_query(ctx.handle, ps.numel() - 1, x.numel(), ptr(ps), ptr(pos4), k, q.numel(), ptr(q),
                             ptr(near), ptr(dens)))
    return near, dens


class KnnDensity(torch.autograd.Function):
    """W4 density (k neighbours, self included) at the query particles qidx.
    The neighbour lists come from the FP32 search; the backward differentiates
    at the FP64 positions."""

    @staticmethod
    def forward(ctx, x, y, z, qidx, k: int, gctx: Context, pstart):
        ps = torch.as_tensor(np.asarray(pstart, np.int64), device=x.device)
        near, dens = knn_query(gctx, ps.cpu().numpy(), x, y, z, qidx, k)
        q = torch.as_tensor(qidx, device=x.device, dtype=torch.int64).contiguous()
        ctx.gctx, ctx.k = gctx, k
        ctx.save_for_backward(x, y, z, ps, q, near)
        return dens

    @staticmethod
    def backward(ctx, gd):
        x, y, z, ps, q, near = ctx.saved_tensors
        g = gd.detach().to(torch.float64).contiguous()
        gx, gy, gz = (torch.zeros_like(x) for _ in range(3))
        check(lib().gf_knn_density_adjoint(ctx.gctx.handle, ps.numel() - 1, x.numel(), ptr(ps), ptr(x), ptr(y),
                                           ptr(z), ctx.k, q.numel(), ptr(q), ptr(near), ptr(g), ptr(gx), ptr(gy),
                                           ptr(gz)))
        return gx, gy, gz, None, None, None, None


def peak_and_probe_loss(x, y, z, m, plan: MeshPlan, probes, k=32, npeak=64, margin=1):
    """Sum of the smoothed mesh density at its npeak highest peaks plus the
    kNN density at the probe particles.  Returns (loss, the peak cells as
    offsets into the mesh buffer).  The peak cells are chosen on the forward
    mesh and held fixed (a selection, not differentiated)."""
    S = MeshDensity.apply(x, y, z, m, plan)
    h, c, _ = plan.peaks(S.detach(), margin=margin)
    cells = torch.as_tensor(plan.mesh["off"][h[:npeak]] + c[:npeak], device=S.device)
    rho = KnnDensity.apply(x, y, z, probes, k, plan.ctx, plan.pstart.cpu().numpy())
    return S.double()[cells].sum() + rho.double().sum(), cells
