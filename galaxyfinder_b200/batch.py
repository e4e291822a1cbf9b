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


def _pos4(x, y, z, m, device):
    p = np.stack([np.asarray(x, np.float32), np.asarray(y, np.float32),
                  np.asarray(z, np.float32), np.asarray(m, np.float32)], 1)
    return torch.as_tensor(np.ascontiguousarray(p), device=device)


def tree_build_export(ctx: Context, pstart, pos4, theta2=0.5, q5_asbuilt=False) -> dict:
    """Builds the octree of FP32 recentred positions (pos4: (n, 4) x, y, z, mass;
    torch tensor on the device or numpy) and returns it in host memory."""
    dev = torch.device("cuda", ctx.device)
    pos4 = torch.as_tensor(pos4, dtype=torch.float32, device=dev).contiguous()
    ps = torch.as_tensor(np.asarray(pstart, np.int64), device=dev)
    info = _lib.TreeInfo()
    n, nh = pos4.shape[0], ps.numel() - 1
    check(lib().gf_tree_build(ctx.handle, nh, n, ptr(ps), ptr(pos4), theta2, int(q5_asbuilt),
                              ctypes.byref(info)))
    nn = info.nnode
    bh = np.zeros(nn, _lib.BH_NODE_DTYPE)
    kn = np.zeros(nn, _lib.KNN_NODE_DTYPE)
    tpos = np.zeros((n, 4), np.float32)
    perm = np.zeros(n, np.int32)
    root = np.zeros(nh, np.int32)
    rend = np.zeros(nh, np.int32)
    check(lib().gf_tree_export(ctx.handle, ptr(bh), ptr(kn), ptr(tpos), ptr(perm), ptr(root),
                               ptr(rend)))
    return dict(bh=bh, knn=kn, pos=tpos, perm=perm, root=root, rend=rend, nnode=nn)


def knn_density(ctx: Context, pstart, pos4, k=32):
    """k nearest neighbours (halo-local indices) and W4 density per particle."""
    dev = torch.device("cuda", ctx.device)
    pos4 = torch.as_tensor(pos4, dtype=torch.float32, device=dev).contiguous()
    ps = torch.as_tensor(np.asarray(pstart, np.int64), device=dev)
    n = pos4.shape[0]
    near = torch.empty((n, k), dtype=torch.int32, device=dev)
    dens = torch.empty(n, dtype=torch.float32, device=dev)
    check(lib().gf_knn_density(ctx.handle, ps.numel() - 1, n, ptr(ps), ptr(pos4), k, ptr(near),
                               ptr(dens)))
    return near, dens


def self_potential(ctx: Context, pstart, pos4, theta2=0.5, ndirect=0, potentfact=0.0,
                   add_bg=False):
    """Returns (penergy, raw potential) for every particle of every halo."""
    dev = torch.device("cuda", ctx.device)
    pos4 = torch.as_tensor(pos4, dtype=torch.float32, device=dev).contiguous()
    ps = torch.as_tensor(np.asarray(pstart, np.int64), device=dev)
    n = pos4.shape[0]
    pe = torch.empty(n, dtype=torch.float32, device=dev)
    raw = torch.empty(n, dtype=torch.float32, device=dev)
    check(lib().gf_self_potential(ctx.handle, ps.numel() - 1, n, ptr(ps), ptr(pos4), theta2,
                                  ndirect, potentfact, int(add_bg), ptr(pe), ptr(raw)))
    return pe, raw


def stage_config(mesh: MeshRule | None = None, box=100.0, knn_k=32, do_mesh=True,
                 do_potential=True, ndirect=100, theta2=0.5, add_bg=True, q5_asbuilt=False,
                 potentfact=0.0, count_work=False, mesh_onchip=False,
                 plain_fp64=False) -> _lib.StageConfig:
    """mesh_onchip: keep 64^3 meshes on chip (one thread-block cluster per
    mesh) instead of in device memory.
    plain_fp64: the plain FP64 stage (every phase in FP64)."""
    if mesh is None:
        mesh = mesh_rule(mode=_lib.MESH_POW2, rg=2.0, rg_in_cells=True)
    return _lib.StageConfig(mesh, box, knn_k, int(do_mesh), int(do_potential), ndirect, theta2,
                            int(add_bg), int(q5_asbuilt), int(count_work), potentfact,
                            int(mesh_onchip), int(plain_fp64))


class StageBuffers:
    """Device outputs of gf_stage_run for a batch of n particles."""

    def __init__(self, n: int, k: int, device, keep_positions=False, keep_phi=False):
        self.nearindex = torch.empty((n, max(k, 1)), dtype=torch.int32, device=device)
        self.dens_sph = torch.empty(n, dtype=torch.float32, device=device)
        self.dens_mesh = torch.empty(n, dtype=torch.float32, device=device)
        self.penergy = torch.empty(n, dtype=torch.float32, device=device)
        # raw tree potential phi (penergy = phi * potentfact + bg, rounded to float)
        self.phi = torch.empty(n, dtype=torch.float32, device=device) if keep_phi else None
        self.xr = self.yr = self.zr = None
        if keep_positions:
            self.xr = torch.empty(n, dtype=torch.float64, device=device)
            self.yr = torch.empty(n, dtype=torch.float64, device=device)
            self.zr = torch.empty(n, dtype=torch.float64, device=device)

    def c(self) -> _lib.StageOut:
        return _lib.StageOut(ptr(self.nearindex), ptr(self.dens_sph), ptr(self.dens_mesh),
                             ptr(self.penergy), ptr(self.xr), ptr(self.yr), ptr(self.zr), ptr(self.phi))


class HaloViews:
    """Each halo of a batch as a batch of one (device pointers offset into the
    batch and its outputs): the plain path, one halo per gf_stage_run call."""

    def __init__(self, batch: DeviceBatch, out: StageBuffers, k: int, pstart_host: np.ndarray):
        ps = np.asarray(pstart_host, np.int64)
        counts = np.diff(ps)
        self.one = torch.zeros((batch.nhalo, 2), dtype=torch.int64, device=batch.x.device)
        self.one[:, 1] = torch.as_tensor(counts, device=batch.x.device)
        self.views = []
        kk = max(k, 1)
        for h in range(batch.nhalo):
            a, n = int(ps[h]), int(counts[h])
            b = Batch(1, n, self.one.data_ptr() + 16 * h, batch.x.data_ptr() + 8 * a,
                      batch.y.data_ptr() + 8 * a, batch.z.data_ptr() + 8 * a,
                      batch.mass.data_ptr() + 8 * a, batch.type.data_ptr() + 4 * a)
            o = _lib.StageOut(out.nearindex.data_ptr() + 4 * kk * a, out.dens_sph.data_ptr() + 4 * a,
                              out.dens_mesh.data_ptr() + 4 * a, out.penergy.data_ptr() + 4 * a,
                              None, None, None, None)
            self.views.append((b, o))

    def run(self, ctx: Context, cfg: _lib.StageConfig, halos=None):
        L = lib()
        for h in (range(len(self.views)) if halos is None else halos):
            b, o = self.views[h]
            check(L.gf_stage_run(ctx.handle, ctypes.byref(b), ctypes.byref(cfg), ctypes.byref(o), None))


def stage_run(ctx: Context, batch: DeviceBatch, cfg: _lib.StageConfig,
              out: StageBuffers | None = None, stats=False):
    """Runs the whole density-and-potential stage on the batch."""
    if out is None:
        out = StageBuffers(batch.n, cfg.knn_k, batch.x.device, keep_positions=True, keep_phi=True)
    st = _lib.StageStats() if stats else None
    b = batch.c()
    oc = out.c()
    check(lib().gf_stage_run(ctx.handle, ctypes.byref(b), ctypes.byref(cfg), ctypes.byref(oc),
                             ctypes.byref(st) if st is not None else None))
    if stats:
        return out, {f: getattr(st, f) for f, _ in _lib.StageStats._fields_}
    return out


class StageGraph:
    """The stage of one batch captured as a CUDA graph (gf_stage_graph_*).

    Creating it runs the stage once eagerly (its outputs are the batch's
    results) and captures a pass with every launch shape fixed by that run's
    plan.  launch() replays it on the batch's current contents, asynchronously
    on the context's stream; sync() waits and raises GFError(GF_ESTALE) if a
    replay no longer fitted the plan.  run() replays, waits and re-plans when
    needed (returns True then).  The batch and output tensors must stay alive
    and in place while the graph exists."""

    def __init__(self, ctx: Context, batch: DeviceBatch, cfg: _lib.StageConfig, out: StageBuffers):
        self.ctx, self.batch, self.cfg, self.out = ctx, batch, cfg, out
        self._b = batch.c()
        self._o = out.c()
        h = ctypes.c_void_p()
        check(lib().gf_stage_graph_create(ctx.handle, ctypes.byref(self._b), ctypes.byref(cfg),
                                          ctypes.byref(self._o), ctypes.byref(h)))
        self.handle = h

    def launch(self):
        check(lib().gf_stage_graph_launch(self.handle))

    def sync(self):
        check(lib().gf_stage_graph_sync(self.handle))

    def run(self) -> bool:
        replanned = ctypes.c_int32()
        check(lib().gf_stage_graph_run(self.handle, ctypes.byref(replanned)))
        return bool(replanned.value)

    @property
    def replans(self) -> int:
        return int(lib().gf_stage_graph_replans(self.handle))

    def nodes(self):
        """(kernel nodes, all nodes) of the captured graph."""
        k, n = ctypes.c_int32(), ctypes.c_int32()
        check(lib().gf_stage_graph_nodes(self.handle, ctypes.byref(k), ctypes.byref(n)))
        return k.value, n.value

    def close(self):
        if self.handle:
            lib().gf_stage_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def density_peaks(ctx: Context, den, neighbor, type_=None, threshold=2000.0):
    """finddenpeak's peaks (subhaloden.mod6.c:416-494) of one halo on the
    device: den (np,) float32, neighbor (np, k) int32 halo-local kNN lists,
    type_ (np,) int32 to keep stars only.  Returns the peak indices (int32
    device tensor, particle order)."""
    np_, k = neighbor.shape
    peak = torch.empty(max(np_, 1), dtype=torch.int32, device=den.device)
    npeak = ctypes.c_int32()
    check(lib().gf_density_peaks(ctx.handle, np_, k, ptr(den), ptr(neighbor), ptr(type_), threshold,
                                 np_, ptr(peak), ctypes.byref(npeak)))
    return peak[:npeak.value]


def core_density(ctx: Context, den, neighbor, type_, mass, peak):
    """FindCoreDensity (subhaloden.mod6.c:1167-1475) of one halo on the device:
    per core its core density, member and star counts and star mass, per
    particle its core id (-9999 for none) and working-particle flag."""
    np_, k = neighbor.shape
    nc = int(peak.numel())
    dev = den.device
    out = dict(coredensity=torch.empty(nc, dtype=torch.float32, device=dev),
               nummem=torch.empty(nc, dtype=torch.int32, device=dev),
               numstar=torch.empty(nc, dtype=torch.int32, device=dev),
               starmass=torch.empty(nc, dtype=torch.float32, device=dev),
               haloid=torch.empty(np_, dtype=torch.int32, device=dev),
               flag=torch.empty(np_, dtype=torch.uint8, device=dev))
    check(lib().gf_core_density(ctx.handle, np_, k, ptr(den), ptr(neighbor), ptr(type_), ptr(mass), nc,
                                ptr(peak), *(ptr(out[f]) for f in ("coredensity", "nummem", "numstar",
                                                                  "starmass", "haloid", "flag"))))
    return out


def chunk_cuts(pstart, nchunk: int) -> list[int]:
    """Halo indices that split a batch into at most nchunk contiguous chunks
    of similar particle counts: the first halo starting at or after each
    multiple of n/nchunk particles (a halo larger than a chunk stays whole,
    so there may be fewer chunks); ascending, from 0 to nhalo."""
    ps = np.asarray(pstart, np.int64)
    n = int(ps[-1])
    cuts = [0] + [int(np.searchsorted(ps, c * n / nchunk)) for c in range(1, nchunk)] + [len(ps) - 1]
    return sorted(set(cuts))


class PipelinedStage:
    """The stage over a catalogue split into halo chunks of similar particle
    counts, each with its own context, CUDA stream, device buffers and host
    thread, so that one chunk's host<->device copies and host-side syncs
    (halo frames, tree levels) overlap other chunks' kernels.

    With `prioritise`, earlier chunks get higher stream priorities (CUDA
    offers four levels through torch), so the GPU works through the chunks
    roughly in order and fills the gaps of one chunk's host syncs with the
    next chunk's kernels; the first chunks finish early and their outputs
    travel back while the later ones compute.

    run_resident(steps) runs every chunk `steps` times on inputs already on
    the device; run_e2e(steps) also copies each chunk's inputs from pinned
    host memory and its outputs back every time, inside the same overlapped
    schedule.  Both return the (start, end) CUDA events that bracket all
    chunks' passes."""

    def __init__(self, hb, cfg: _lib.StageConfig, nchunk: int = 3, device: int = 0, k: int = 32,
                 prioritise: bool = True, graph: bool = False):
        import concurrent.futures as cf
        self.cfg = cfg
        self.k = k
        dev = torch.device("cuda", device)
        ps = np.asarray(hb.pstart, np.int64)
        cuts = chunk_cuts(ps, nchunk)
        self.chunks = []
        _, top = torch.cuda.Stream.priority_range()  # (least, greatest): (0, -3)
        for a, b in zip(cuts[:-1], cuts[1:]):
            if b <= a:
                continue
            p0, p1 = int(ps[a]), int(ps[b])
            prio = min(0, top + len(self.chunks)) if prioritise else 0
            stream = torch.cuda.Stream(device=dev, priority=prio)
            ctx = Context(device, stream)
            host = {f: torch.from_numpy(np.ascontiguousarray(getattr(hb, f)[p0:p1], dt)).pin_memory()
                    for f, dt in (("x", np.float64), ("y", np.float64), ("z", np.float64),
                                  ("mass", np.float64), ("type", np.int32))}
            host["pstart"] = torch.from_numpy(ps[a:b + 1] - p0).pin_memory()
            db = DeviceBatch(*(torch.empty_like(host[f], device=dev) for f in ("x", "y", "z", "mass", "type")),
                             torch.empty_like(host["pstart"], device=dev))
            for f in ("x", "y", "z", "mass", "type", "pstart"):
                getattr(db, f).copy_(host[f])
            out = StageBuffers(p1 - p0, k, dev)
            hout = {f: torch.empty(getattr(out, f).shape, dtype=getattr(out, f).dtype).pin_memory()
                    for f in ("nearindex", "dens_sph", "dens_mesh", "penergy")}
            self.chunks.append(dict(ctx=ctx, stream=stream, host=host, db=db, out=out, hout=hout, n=p1 - p0))
        torch.cuda.synchronize(dev)
        # with `graph`, each chunk's stage is captured once and replayed
        self.graph = graph
        for c in self.chunks:
            c["graph"] = StageGraph(c["ctx"], c["db"], cfg, c["out"]) if graph else None
        torch.cuda.synchronize(dev)
        self.pool = cf.ThreadPoolExecutor(max_workers=len(self.chunks))
        self.h2d_bytes = sum(t.numel() * t.element_size() for c in self.chunks for t in c["host"].values())
        self.d2h_bytes = sum(t.numel() * t.element_size() for c in self.chunks for t in c["hout"].values())

    def _chunk(self, c, e2e: bool, start, steps: int):
        s = c["stream"]
        s.wait_event(start)
        for _ in range(steps):  # this chunk's steps back to back on its stream
            if e2e:
                with torch.cuda.stream(s):
                    for f in ("x", "y", "z", "mass", "type", "pstart"):
                        getattr(c["db"], f).copy_(c["host"][f], non_blocking=True)
            if c["graph"] is not None:
                c["graph"].launch()
            else:
                stage_run(c["ctx"], c["db"], self.cfg, c["out"])
            if e2e:
                with torch.cuda.stream(s):
                    for f, t in c["hout"].items():
                        t.copy_(getattr(c["out"], f), non_blocking=True)
        done = torch.cuda.Event()
        done.record(s)
        return done

    def _run(self, e2e: bool, steps: int):
        cur = torch.cuda.current_stream()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(cur)
        dones = list(self.pool.map(lambda c: self._chunk(c, e2e, start, steps), self.chunks))
        for d in dones:
            cur.wait_event(d)
        end.record(cur)
        return start, end

    def run_resident(self, steps: int = 1):
        """`steps` passes over the catalogue; each chunk runs its passes back
        to back, so one chunk's next pass overlaps another's current one."""
        return self._run(False, steps)

    def run_e2e(self, steps: int = 1):
        return self._run(True, steps)

    def check(self):
        """With graphs: waits for every chunk and raises GFError(GF_ESTALE) if
        a replay no longer fitted its chunk's plan."""
        for c in self.chunks:
            if c["graph"] is not None:
                c["graph"].sync()

    def close(self):
        self.pool.shutdown()
        for c in self.chunks:
            if c.get("graph") is not None:
                c["graph"].close()
            c["ctx"].close()
