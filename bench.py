#!/usr/bin/env python
"""Benchmark of the batched density-and-potential stage.

One step = the whole stage on a batched FoF catalogue: FP64 recentring,
octree, kNN (k = 32) + SPH density, TSC mesh + Gaussian smoothing + findDen,
and the Barnes-Hut self potential of every halo.  Workload: 4096 halos with
N_p ~ N^-1.9 on [100, 2e6], NFW with subhalos, 20% stars, per-halo TSC mesh of
64-256^3 (seeded synthetic catalogue standing in for RAMSES/opFoF output).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gf|reference]

The headline `value` and `e2e` run the catalogue as halo chunks on their own
CUDA streams and host threads (PipelinedStage), so one chunk's copies and
host-side syncs overlap the others' kernels; `single_stream` gives the same
numbers for one gf_stage_run call over the whole catalogue, and the
per-phase times and roofline come from that call.

Under torchrun each rank processes its own catalogue shard (independent
halos, no collective on the data path: weak scaling); rank 0 prints one JSON
line.  `--impl reference` times the reference's own NewGalFinder C
(oracle/_ref, compiled from its sources) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particles/s, kNN+TSC/FFT+potential; batched FP32 vs plain GPU at ≤1e-5 rel err"
UNIT = "particles/s"
K_NEIGH = 32
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per particle of
# each phase's dominant kernel, from one ncu capture of the 1024-halo
# catalogue (1,281,067 particles); the traffic scales with the particles
# processed.
TRAFFIC_PER_PARTICLE = {"knn": (59.67e6 + 115.437e6) / 1281067}
# What bounds the kNN kernel instead of HBM, from the same capture: the tree
# walk is latency- and issue-bound (its HBM traffic is the neighbour lists).
KNN_LIMITER = ("latency/issue: 68.7% of issue slots active, 35.9% of warp slots occupied (6 blocks of 4 "
               "warps per SM: 79 registers and 35.3 KB of heaps per block), dominant stall 'wait'; "
               "DRAM 0.69% of peak")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["gf", "reference"], default="gf")
    ap.add_argument("--nhalo", type=int, default=4096)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--chunks", type=int, default=12,
                    help="halo chunks (streams) of the pipelined stage (12: the best end-to-end time "
                         "on the 4096-halo catalogue; 8 chunks run 2 %% faster resident, 6 %% slower end to end)")
    ap.add_argument("--postprocessing", action="store_true",
                    help="run only the full post-processing workload (1e5 groups + centre refinement) and "
                         "print its line")
    ap.add_argument("--mesh-onchip", action="store_true",
                    help="run the 64^3 meshes through the opt-in on-chip cluster path")
    ap.add_argument("--configs", action="store_true",
                    help="also time the single-halo workloads (131072-particle halo, 5e7 cluster, 1e7 mixture)")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the comparison of sampled halos with the oracle")
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "source": "measured"}
    return {"hbm_gbs": PEAKS_FALLBACK["hbm_gbs"], "source": "fallback"}


# ------------------------------------------------------------------ clocks
class Clocks:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.tmp, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.tmp.flush()
        rows = []
        for line in Path(self.tmp.name).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) != 7:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[3:]))
            except ValueError:
                continue
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v == "Active"})
        loaded = [r[0] for r in rows]
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ reference (CPU)
# Halo-size strata (log N_p bins over the catalogue's range [100, 2e6]).  A
# CPU sample times halos from every stratum: up to STRATUM_BUDGET particles
# per stratum per step, at least one halo.  Halos above MAX_TIMED particles
# take the reference minutes each, so they are not timed; their stratum is
# extrapolated with the per-particle rate of the largest timed stratum, which
# overstates the reference's speed there (its kNN cost per particle grows
# with the halo size).
STRATA = (100, 316, 1000, 3162, 10_000, 31_623, 100_000, 316_228, 2_000_001)
STRATUM_BUDGET = 20_000
MAX_TIMED = 250_000
MESH_KW = dict(mode=2, nmin=64, nmax=256, rg=2.0, rg_in_cells=True)  # POW2 rule, 64-256^3


def halo_counts(hb):
    return np.diff(np.asarray(hb.pstart, np.int64))


def strata_of(hb):
    n = halo_counts(hb)
    return [np.flatnonzero((n >= a) & (n < b)) for a, b in zip(STRATA[:-1], STRATA[1:])]


def stratified_sample(hb, step: int, seed: int = 7):
    """Per stratum, the halos one CPU step times (seeded by the step)."""
    n = halo_counts(hb)
    rng = np.random.default_rng(seed + 1000 * step)
    out = []
    for halos in strata_of(hb):
        timed = halos[n[halos] <= MAX_TIMED]
        pick, tot = [], 0
        for h in rng.permutation(timed):
            pick.append(int(h))
            tot += int(n[h])
            if tot >= STRATUM_BUDGET:
                break
        out.append(pick)
    return out


def recentred_halo(hb, h):
    """Dump2BP's recentring of one halo after the periodic unwrap (FP64)."""
    a, b = int(hb.pstart[h]), int(hb.pstart[h + 1])
    p = np.stack([hb.x[a:b], hb.y[a:b], hb.z[a:b]], 1)
    for ax in range(3):
        c = p[:, ax]
        cs = np.where(c < 50.0, c + 100.0, c)
        if c.max() - c.min() > 50.0 and cs.max() - cs.min() < c.max() - c.min():
            p[:, ax] = cs
    return p - p.min(axis=0), a, b


def reference_halo_seconds(ref, hb, h, workers: int) -> float:
    """The reference's own functions on one halo, as subhalo_den drives them:
    findsphdensity (kNN + W4), assign_density_TSC, gaussian_Smoothing (FFTW
    unavailable: its FFTs timed with the scipy.fft stand-in), findDen and
    Self_Halo_Potent.  The mesh plan is the numpy restatement, so no repo
    library is loaded.  Returns seconds."""
    from oracle import fftw_standin, plan as oplan
    t0 = time.perf_counter()
    p, a, b = recentred_halo(hb, h)
    m = hb.mass[a:b]
    ref.findsphdensity(p[:, 0], p[:, 1], p[:, 2], m, min(K_NEIGH, b - a))
    mm = oplan.plan_one(p.max(0), **MESH_KW)
    n3 = (mm["nx"], mm["ny"], mm["nz"])
    o, cell = mm["xmin"], mm["cellsize"]
    den = ref.assign_density_TSC(p[:, 0], p[:, 1], p[:, 2], m, hb.type[a:b], *n3, o, o, o, cell, 5)
    fftw_standin.gaussian_smoothing(den, *n3, cell, mm["rg"], workers=workers)
    ref.findDen(p[:, 0], p[:, 1], p[:, 2], den, *n3, o, o, o, cell)
    ref.Self_Halo_Potent(p[:, 0], p[:, 1], p[:, 2], m.astype(np.float32))
    return time.perf_counter() - t0


def reference_step(ref, hb, step: int, workers: int) -> dict:
    """One CPU step: the stratified sample timed halo by halo, and the time the
    whole catalogue would take at each stratum's measured rate."""
    n = halo_counts(hb)
    sample = stratified_sample(hb, step)
    parts, secs = [], []
    for halos in sample:
        parts.append(int(n[halos].sum()) if halos else 0)
        secs.append(sum(reference_halo_seconds(ref, hb, h, workers) for h in halos))
    rates = [p / t if t > 0 else None for p, t in zip(parts, secs)]
    extrap, last = 0.0, None
    for s, halos in enumerate(strata_of(hb)):
        r = rates[s] if rates[s] is not None else last  # untimed: largest timed stratum's rate
        last = r if r is not None else last
        extrap += float(n[halos].sum()) / r
    return {"seconds": float(sum(secs)), "particles": int(sum(parts)), "extrap_s": extrap,
            "rates": rates, "halos": [len(x) for x in sample]}


def reference_baseline(hb, steps: int, warmup: int) -> dict:
    import oracle.oracle as orc
    ref = orc.Reference("fixed")
    cores = orc.cpu_threads()
    n = halo_counts(hb)
    small = [int(h) for h in np.argsort(n)[:2]]
    for _ in range(max(warmup, 1)):  # first touch of the reference's arena
        for h in small:
            reference_halo_seconds(ref, hb, h, cores)
    res = [reference_step(ref, hb, j, cores) for j in range(steps)]
    extrap = float(np.mean([r["extrap_s"] for r in res]))
    strata = []
    for s, halos in enumerate(strata_of(hb)):
        rs = [r["rates"][s] for r in res if r["rates"][s] is not None]
        strata.append({"n_p": [STRATA[s], STRATA[s + 1] - 1], "halos": int(len(halos)),
                       "particles": int(n[halos].sum()),
                       "timed_halos_per_step": float(np.mean([r["halos"][s] for r in res])),
                       "rate": float(np.mean(rs)) if rs else None})
    return {"value": float(hb.n) / extrap, "cores": cores, "extrap_s": extrap,
            "step_seconds": float(np.mean([r["seconds"] for r in res])),
            "step_particles": float(np.mean([r["particles"] for r in res])), "strata": strata}


def reference_sample_text(rb, hb) -> str:
    return (f"stratified by halo size: {len(STRATA) - 1} log N_p strata over [100, 2e6]; each step times up "
            f"to {STRATUM_BUDGET} particles (at least one halo) per stratum, halos of at most {MAX_TIMED} "
            f"particles, on average {rb['step_particles']:.0f} particles in {rb['step_seconds']:.1f} s; "
            f"the whole {hb.n}-particle catalogue's time is the sum of each stratum's particles over its "
            f"measured rate ({rb['extrap_s']:.0f} s); the {sum(1 for h in halo_counts(hb) if h > MAX_TIMED)} "
            f"halos above {MAX_TIMED} particles take the largest timed stratum's rate (which overstates "
            f"the reference's speed on them). findsphdensity + assign_density_TSC + gaussian_Smoothing + "
            f"findDen + Self_Halo_Potent; FFTW unavailable: the smoothing's FFTs run on scipy.fft "
            f"(single precision, all host threads) as the stand-in")


def reference_line(args, hb, base_cfg):
    try:
        rb = reference_baseline(hb, args.steps, args.warmup)
    except Exception as e:  # reference libraries missing on this host
        return {"impl": "reference", "unavailable": f"reference build missing: {e}"}
    line = dict(base_cfg)
    line.update({"impl": "reference", "value": rb["value"], "ms_per_step": rb["step_seconds"] * 1e3,
                 "cpu_baseline": {"value": rb["value"], "unit": UNIT, "cores": rb["cores"],
                                  "kind": "reference", "sample": reference_sample_text(rb, hb),
                                  "strata": rb["strata"], "catalogue_seconds": rb["extrap_s"]},
                 "e2e": {"value": rb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0},
                 "note": "ms_per_step is the measured time of one step's stratified sample; value is the "
                         "catalogue's particles over its time extrapolated stratum by stratum"})
    return line


def run_dropin_stage(hb, halos, mesh_rule):
    """The drop-in path a reference user gets by linking libgf: per halo,
    findsphdensity + assign_density_TSC + gaussian_Smoothing + findDen +
    Self_Halo_Potent through the reference signatures with host buffers (one
    halo per call, copies inside every call).  Inputs are built before the
    clock starts, as the reference has them in its own arrays.  Returns
    seconds."""
    from galaxyfinder_b200 import _lib, batch, dropin
    prepared = []
    for h in halos:
        p, a, b = recentred_halo(hb, h)
        bp = np.zeros(b - a, _lib.BP_DTYPE)
        bp["x"], bp["y"], bp["z"] = p[:, 0], p[:, 1], p[:, 2]
        bp["mass"], bp["type"] = hb.mass[a:b], hb.type[a:b]
        mesh, _ = batch.plan_meshes(p.max(0)[None, :], mesh_rule)
        mm = mesh[0]
        den = np.zeros(dropin.mesh_floats(int(mm["nx"]), int(mm["ny"]), int(mm["nz"])), np.float32)
        prepared.append((bp, p, hb.mass[a:b].astype(np.float32), mm, den, min(K_NEIGH, b - a)))
    t0 = time.perf_counter()
    for bp, p, m32, mm, den, k in prepared:
        n3 = (int(mm["nx"]), int(mm["ny"]), int(mm["nz"]))
        o, cell = float(mm["xmin"]), float(mm["cellsize"])
        dropin.findsphdensity(bp, k)
        den[:] = 0
        dropin.assign_density_TSC(bp, *n3, o, o, o, cell, _lib.TYPE_ALL, den=den)
        dropin.gaussian_Smoothing(den, *n3, cell, float(mm["rg"]))
        dropin.findDen(bp, den, *n3, o, o, o, cell)
        dropin.Self_Halo_Potent(p, m32)
    return time.perf_counter() - t0


def catalogue_mesh_cells(hb) -> int:
    """Mesh floats of the whole catalogue under the POW2 rule (numpy plan)."""
    from oracle import plan as oplan
    ext = np.array([recentred_halo(hb, h)[0].max(0) for h in range(hb.nhalo)])
    return int(oplan.plan(ext, **MESH_KW)[1])


def single_halo_configs(dev, steps: int = 3, warmup: int = 2) -> dict:
    """Throughput of the stage on the single-halo workloads: the 131072-particle
    NFW halo (fixed 128^3 mesh, Gaussian 2 cells), the 5e7-particle cluster
    (512^3, 2 cells) and the 1e7-particle Gaussian mixture (256^3, 1.5 cells),
    inputs resident, CUDA-event time per step; the first also through the plain
    FP64 stage."""
    import torch

    from galaxyfinder_b200 import _lib, batch, synth
    res = {}
    for name, make, nmesh, rg in (("single halo 131072, 128^3", synth.config1, 128, 2.0),
                                  ("cluster 5e7, 512^3", synth.config3, 512, 2.0),
                                  ("gaussian mixture 1e7, 256^3", synth.config4, 256, 1.5)):
        hb = make()
        ctx = batch.Context(dev.index or 0)
        db = batch.DeviceBatch.from_halobatch(hb, device=dev)
        rule = batch.mesh_rule(mode=_lib.MESH_FIXED, nfixed=nmesh, rg=rg, rg_in_cells=True)
        entry = {"particles": int(hb.n)}
        for label, cfg in (("batched_fp32", batch.stage_config(mesh=rule, knn_k=K_NEIGH)),
                           ("plain_fp64", batch.stage_config(mesh=rule, knn_k=K_NEIGH, plain_fp64=True))):
            if label == "plain_fp64" and hb.n > 1_000_000:
                continue
            out = batch.StageBuffers(hb.n, K_NEIGH, dev)
            for _ in range(warmup):
                batch.stage_run(ctx, db, cfg, out)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ctx.stream)
            for _ in range(steps):
                batch.stage_run(ctx, db, cfg, out)
            e1.record(ctx.stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            _, st = batch.stage_run(ctx, db, cfg, out, stats=True)
            entry[label] = {"value": hb.n / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
                            "phases_ms": {k[3:]: st[k] for k in st if k.startswith("ms_") and k != "ms_pad"}}
            del out
        if "plain_fp64" in entry:
            entry["batched_over_plain"] = entry["batched_fp32"]["value"] / entry["plain_fp64"]["value"]
        res[name] = entry
        ctx.close()
        del db, hb
        torch.cuda.empty_cache()
    return res


def postprocessing_workload(dev, steps: int, warmup: int, nchunk: int = 16, block: int = 2000) -> dict:
    """The full post-processing run: 1e5 FoF groups from the catalogue law on
    [50, 1e7] particles with 10 % unbound background particles, the batched
    stage over all of them (halo chunks on their own streams, inputs resident,
    CUDA-event time), then the gradient-ascent refinement (<= 20 steps of 0.1
    smoothing length) of the centre of every group's stellar body on its
    smoothed stellar mesh (64-256^3), all centres of a block of groups in one
    launch, and the refined centres against GalCenter's search-based ones
    (GalCenter/find_centers.c:25-104) on a sample of groups."""
    import torch

    from galaxyfinder_b200 import _lib, batch, centres, synth
    from oracle.oracle import GalCenterSearch
    t0 = time.perf_counter()
    hb = synth.postprocessing_catalogue()
    gen_s = time.perf_counter() - t0
    rule = batch.mesh_rule(mode=_lib.MESH_POW2, nmin=64, nmax=256, rg=2.0, rg_in_cells=True)
    cfg = batch.stage_config(mesh=rule, knn_k=K_NEIGH)
    pipe = batch.PipelinedStage(hb, cfg, nchunk=nchunk, device=dev.index or 0, k=K_NEIGH)
    pipe.run_resident(max(warmup, 1))
    torch.cuda.synchronize()
    p0, p1 = pipe.run_resident(steps)
    torch.cuda.synchronize()
    stage_ms = p0.elapsed_time(p1) / steps
    pipe.close()
    del pipe
    torch.cuda.empty_cache()
    # one galaxy per group with >= 30 stars: start at its stellar centre of mass
    n = halo_counts(hb)
    ctx = batch.Context(dev.index or 0)
    srule = batch.mesh_rule(mode=_lib.MESH_POW2, nmin=64, nmax=256, rg=2.0, rg_in_cells=True,
                            ptype=_lib.TYPE_STAR)
    refined = {}
    t0 = time.perf_counter()
    ngal = moved = 0
    for h0 in range(0, hb.nhalo, block):
        h1 = min(hb.nhalo, h0 + block)
        a, b = int(hb.pstart[h0]), int(hb.pstart[h1])
        sl = slice(a, b)
        ps = hb.pstart[h0:h1 + 1] - a
        starts, halo_of = [], []
        for h in range(h0, h1):
            p, ha, hb_ = recentred_halo(hb, h)
            st = hb.type[ha:hb_] == 1
            if st.sum() < 30:
                continue
            w = hb.mass[ha:hb_][st]
            c = (p[st] * w[:, None]).sum(0) / w.sum()
            off = np.array([hb.x[ha], hb.y[ha], hb.z[ha]]) - p[0]  # recentred -> box coordinates
            starts.append(np.mod(c + off, 100.0))
            halo_of.append(h - h0)
        if not starts:
            continue
        cen, rho, moves, aux = centres.refine_centres(ctx, hb.x[sl], hb.y[sl], hb.z[sl], hb.mass[sl],
                                                      hb.type[sl], ps, np.array(starts),
                                                      np.array(halo_of, np.int32), rule=srule)
        torch.cuda.synchronize()
        for i, hl in enumerate(halo_of):
            refined[h0 + hl] = (cen[i], float(aux["mesh"][hl]["rg"]))
        ngal += len(starts)
        moved += int(np.sum(moves > 0))
        del aux
    centre_s = time.perf_counter() - t0
    # against GalCenter's search on a sample of groups of up to 1e5 particles
    gc = GalCenterSearch()
    rng = np.random.default_rng(3)
    cand = [h for h in refined if n[h] <= 100_000]
    offs = []
    for h in rng.choice(cand, min(48, len(cand)), replace=False):
        a, b = int(hb.pstart[h]), int(hb.pstart[h + 1])
        g, _ = gc.find_centers(hb.x[a:b], hb.y[a:b], hb.z[a:b], hb.mass[a:b], hb.type[a:b])
        c, rg = refined[int(h)]
        d = c - g[:3]
        d -= 100.0 * np.round(d / 100.0)
        offs.append(np.linalg.norm(d) / rg)
    ctx.close()
    offs = np.array(offs)
    return {"particles": int(hb.n), "groups": int(hb.nhalo), "generation_s": gen_s,
            "stage": {"value": hb.n / (stage_ms / 1e3), "unit": UNIT, "ms_per_step": stage_ms,
                      "path": f"PipelinedStage, {nchunk} halo chunks, inputs resident"},
            "centres": {"galaxies": ngal, "moved": moved, "seconds": centre_s,
                        "path": "stellar TSC + smoothing (64-256^3) per block of 2000 groups, all centres of a "
                                "block in one gf_refine_centres launch (<= 20 steps of 0.1 R_G); seconds include "
                                "the host-side recentring and mesh planning",
                        "offset_vs_galcenter_over_rg": {"sample": int(len(offs)),
                                                        "median": float(np.median(offs)) if len(offs) else None,
                                                        "p90": float(np.quantile(offs, 0.9)) if len(offs) else None}}}


def graph_measurements(args, hb, cfg, ctx, db, out, total_particles, barrier, max_over_ranks) -> dict:
    """Throughput of CUDA-graph replays of the stage: the whole catalogue as
    one graph (gf_stage_graph on one stream), and the pipelined stage with
    one graph per halo chunk; a replay that no longer fits its plan would
    raise after the timed region."""
    import torch

    from galaxyfinder_b200 import batch
    if cfg.mesh_onchip:
        return {"skipped": "stage graphs capture device-memory meshes only (mesh_onchip is set)"}
    res = {}
    # a context on a stream of its own, so the events bracket the replays
    gctx = batch.Context(ctx.device, torch.cuda.Stream(device=db.x.device))
    g = batch.StageGraph(gctx, db, cfg, out)
    kernels, nodes = g.nodes()
    for _ in range(max(args.warmup, 3)):
        g.launch()
    g.sync()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(gctx.stream)
    for _ in range(args.steps):
        g.launch()
    e1.record(gctx.stream)
    g.sync()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    res["single_stream"] = {"value": total_particles / (ms / 1e3), "ms_per_step": ms,
                            "kernel_nodes": kernels, "graph_nodes": nodes, "replans": g.replans,
                            "path": "gf_stage_graph over the whole catalogue, one replay per step"}
    g.close()
    gctx.close()
    gp = batch.PipelinedStage(hb, cfg, nchunk=args.chunks, device=ctx.device, k=K_NEIGH, graph=True)
    gp_kernels = sum(c["graph"].nodes()[0] for c in gp.chunks)
    for mode in ("resident", "e2e"):
        runner = gp.run_resident if mode == "resident" else gp.run_e2e
        runner(max(args.warmup, 3))
        gp.check()
        barrier()
        p0, p1 = runner(args.steps)
        torch.cuda.synchronize()
        gp.check()
        pms = max_over_ranks(p0.elapsed_time(p1) / args.steps)
        res["pipelined_" + mode] = {"value": total_particles / (pms / 1e3), "ms_per_step": pms}
    res["pipelined_resident"]["path"] = (f"PipelinedStage(graph=True): {len(gp.chunks)} halo chunks, each "
                                         "replaying its own captured stage")
    res["pipelined_resident"]["kernel_nodes_per_step"] = int(gp_kernels)
    res["pipelined_resident"]["chunks"] = len(gp.chunks)
    gp.close()
    torch.cuda.synchronize()
    return res


def workload_config(args, hb, world: int, mesh_cells: int) -> dict:
    """The `config` object of both arms' JSON lines."""
    return {"workload": f"batched catalogue, {args.nhalo} FoF halos per GPU, N_p ~ N^-1.9 on [100, 2e6], "
                        "k=32, per-halo TSC mesh 64-256^3, Gaussian 2 cells, Barnes-Hut theta2=0.5",
            "nhalo": args.nhalo, "particles_per_gpu": int(hb.n), "mesh_cells": int(mesh_cells),
            "l2": "inputs and working set larger than L2 (no flush needed)",
            "parallelism": f"halo shards x{world} (no collective on the data path)"}


# ------------------------------------------------------------------ accuracy (oracle)
def accuracy_sample(hb, per_stratum: int = 9, seed: int = 11):
    """Halos of every size stratum (all of the largest), at least 64."""
    rng = np.random.default_rng(seed)
    pick = []
    for halos in strata_of(hb):
        pick += [int(h) for h in rng.permutation(halos)[:per_stratum]]
    return sorted(pick)


def accuracy_check(ctx, db, cfg, hb, mesh_rule, halos, rows_per_halo: int = 1500) -> dict:
    """The stage's outputs on sampled halos against the oracle: kNN lists and
    SPH densities against exact kNN (the C restatement, or for halos above
    40k particles a k-d tree over all the halo's FP32 positions, re-ranked in
    exact FP64 (d^2, index) order, on sampled rows); mesh density against the
    FP64 chain (TSC in FP64, FP64 spectral smoothing, findDen); the raw tree
    potential against an FP64 walk of the same tree on sampled particles."""
    import scipy.fft as sf
    import torch
    from scipy.spatial import cKDTree

    from galaxyfinder_b200 import _lib, batch
    from oracle import adjoint as A
    from oracle.oracle import Restatement

    R = Restatement()
    out = batch.StageBuffers(hb.n, K_NEIGH, db.x.device, keep_positions=True, keep_phi=True)
    _, st = batch.stage_run(ctx, db, cfg, out, stats=True)
    torch.cuda.synchronize()
    nn = int(st["nnode"])
    bh = np.zeros(nn, _lib.BH_NODE_DTYPE)
    tpos = np.zeros((hb.n, 4), np.float32)
    root = np.zeros(hb.nhalo, np.int32)
    rend = np.zeros(hb.nhalo, np.int32)
    _lib.check(_lib.lib().gf_tree_export(ctx.handle, _lib.ptr(bh), None, _lib.ptr(tpos), None,
                                         _lib.ptr(root), _lib.ptr(rend)))
    xr = np.stack([out.xr.cpu().numpy(), out.yr.cpu().numpy(), out.zr.cpu().numpy()], 1)
    near = out.nearindex.cpu().numpy()
    dsph = out.dens_sph.cpu().numpy()
    dmesh = out.dens_mesh.cpu().numpy()
    phi = out.phi.cpu().numpy().astype(np.float64)
    rng = np.random.default_rng(5)
    acc = {"halos": len(halos), "particles": 0, "knn_rows": 0, "knn_mismatch": 0, "sph_mismatch": 0,
           "sph_rel_max": 0.0, "mesh_particles": 0, "mesh_rel_max_dense": 0.0, "mesh_rel_max_rho_gt_1e-3": 0.0,
           "mesh_above_1e-5": 0,
           "mesh_rel": [], "pot_rows": 0, "potential_rel_max": 0.0, "pot_rel": []}
    for h in halos:
        a, b = int(hb.pstart[h]), int(hb.pstart[h + 1])
        n = b - a
        acc["particles"] += n
        p = xr[a:b]
        q = p.astype(np.float32)
        k = min(K_NEIGH, n)
        # kNN + SPH
        if n <= 40_000:
            rows = np.arange(n)
            idx, d2 = R.knn(q[:, 0], q[:, 1], q[:, 2], k)
        else:
            rows = np.sort(rng.choice(n, rows_per_halo, replace=False))
            q64 = q.astype(np.float64)
            _, cand = cKDTree(q64).query(q64[rows], k=k + 16, workers=-1)
            idx = np.zeros((len(rows), k), np.int64)
            d2 = np.zeros((len(rows), k))
            for r, i in enumerate(rows):
                c = cand[r]
                d = q64[c] - q64[i]
                dd = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
                o = np.lexsort((c, dd))
                idx[r], d2[r] = c[o[:k]], dd[o[:k]]
        acc["knn_rows"] += len(rows)
        acc["knn_mismatch"] += int(np.sum(np.any(near[a:b][rows, :k] != idx, axis=1)))
        sph = R.sph_density(d2)
        g = dsph[a:b][rows]
        acc["sph_mismatch"] += int(np.sum(g != sph))
        acc["sph_rel_max"] = max(acc["sph_rel_max"], float(np.max(np.abs(g.astype(np.float64) - sph) /
                                                                  np.maximum(np.abs(sph), 1e-300))))
        # mesh density: FP64 chain
        mm, _ = batch.plan_meshes(p.max(0)[None, :], mesh_rule)
        m = mm[0]
        n3 = (int(m["nx"]), int(m["ny"]), int(m["nz"]))
        o, cell = float(m["xmin"]), float(m["cellsize"])
        den = R.tsc(p[:, 0], p[:, 1], p[:, 2], hb.mass[a:b], hb.type[a:b], *n3, o, o, o, cell, 5,
                    acc_double=True)
        mesh = A.Mesh.from_desc(m)
        grid = np.asarray(den, np.float64).reshape(mesh.nz, mesh.ny, mesh.mx)[:, :, :mesh.nx]
        s = sf.irfftn(sf.rfftn(grid, workers=-1) * A._filter(mesh), s=(mesh.nz, mesh.ny, mesh.nx),
                      axes=(0, 1, 2), workers=-1)
        full = mesh.zeros()
        full[:, :, :mesh.nx] = s
        ref = R.find_den(p[:, 0], p[:, 1], p[:, 2], full.ravel().astype(np.float32), *n3, o, o, o,
                         cell).astype(np.float64)
        got = dmesh[a:b].astype(np.float64)
        pos = ref > 0
        rel = np.abs(got[pos] - ref[pos]) / ref[pos]
        # dense: rho > 1e-2 rho_max of the halo, the bar of the single-halo
        # tests; between 1e-3 and 1e-2 the FP32 mesh's absolute roundoff
        # (~2e-7 of its maximum) can approach 1e-5 of the local density
        dense = ref[pos] > 1e-2 * ref.max()
        mid = ref[pos] > 1e-3 * ref.max()
        acc["mesh_particles"] += int(pos.sum())
        acc["mesh_above_1e-5"] += int(np.sum(rel > 1e-5))
        acc["mesh_rel_max_dense"] = max(acc["mesh_rel_max_dense"], float(rel[dense].max()))
        acc["mesh_rel_max_rho_gt_1e-3"] = max(acc["mesh_rel_max_rho_gt_1e-3"], float(rel[mid].max()))
        acc["mesh_rel"].append(rel)
        # potential: raw phi vs FP64 walk of the same tree
        prow = np.arange(n) if n <= 2 * rows_per_halo else np.sort(rng.choice(n, rows_per_halo, replace=False))
        topen = np.full(len(prow), int(n < 100), np.int32)  # Self_Halo_Potent's direct branch
        f64 = R.tree_potential(bh, tpos, q[prow], np.full(len(prow), root[h], np.int32),
                               np.full(len(prow), rend[h], np.int32), topen)
        prel = np.abs(phi[a:b][prow] - f64) / np.abs(f64)
        acc["pot_rows"] += len(prow)
        acc["potential_rel_max"] = max(acc["potential_rel_max"], float(prel.max()))
        acc["pot_rel"].append(prel)
    mrel = np.concatenate(acc.pop("mesh_rel"))
    prel = np.concatenate(acc.pop("pot_rel"))
    acc["mesh_rel_p99"] = float(np.quantile(mrel, 0.99))
    acc["mesh_rel_median"] = float(np.median(mrel))
    acc["mesh_frac_above_1e-5"] = acc["mesh_above_1e-5"] / max(acc["mesh_particles"], 1)
    acc["potential_rel_median"] = float(np.median(prel))
    acc["largest_halo"] = int(max(halo_counts(hb)[halos]))
    acc["bars"] = {"knn": "bit-exact", "sph": "bit-exact", "mesh": "1e-5 relative where rho > 1e-2 rho_max of the halo "
                   "(below, the FP32 mesh's absolute roundoff; every particle is in the fraction beyond 1e-5)", "potential": "1e-6 relative (raw phi vs FP64 "
                   "walk of the same tree)"}
    acc["pass"] = bool(acc["knn_mismatch"] == 0 and acc["sph_mismatch"] == 0 and
                       acc["mesh_rel_max_dense"] < 1e-5 and acc["potential_rel_max"] < 1e-6)
    return acc


# ------------------------------------------------------------------ main
def main():
    args = parse()
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl" if args.impl == "gf" else "gloo",
                                timeout=datetime.timedelta(seconds=600))

    from galaxyfinder_b200 import _lib, batch, shard, synth

    mesh_rule = batch.mesh_rule(mode=_lib.MESH_POW2, nmin=64, nmax=256, rg=2.0, rg_in_cells=True)
    base = {"metric": METRIC, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (f64 recentring, f64 kNN distances)",
            "data": "synthetic (seeded NFW catalogue; no public dataset)"}

    if args.impl == "reference":
        if rank == 0:
            hb = synth.catalogue(seed=synth.SEED_BASE + 2, nhalo=args.nhalo)
            line = reference_line(args, hb, base)
            line["n_gpus"] = world
            line["config"] = workload_config(args, hb, world, catalogue_mesh_cells(hb))
            print(json.dumps(line), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.postprocessing:
        res = postprocessing_workload(dev, args.steps, args.warmup)
        line = dict(base)
        line.update({"value": res["stage"]["value"], "ms_per_step": res["stage"]["ms_per_step"],
                     "config": {"workload": "full post-processing run: 1e5 FoF groups, N_p ~ N^-1.9 on "
                                            "[50, 1e7], 10% unbound background, k=32, per-group TSC mesh "
                                            "64-256^3, Gaussian 2 cells, Barnes-Hut theta2=0.5, then centre "
                                            "refinement", "particles": res["particles"]},
                     "postprocessing": res})
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    hb = synth.catalogue(seed=synth.SEED_BASE + 2 + 1000 * rank, nhalo=args.nhalo)
    ctx = batch.Context(local)
    db = batch.DeviceBatch.from_halobatch(hb, device=dev)
    cfg = batch.stage_config(mesh=mesh_rule, knn_k=K_NEIGH, mesh_onchip=args.mesh_onchip)
    out = batch.StageBuffers(hb.n, K_NEIGH, dev)
    lib = _lib.lib()

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        return v if dist is None else shard.max_over_ranks(v, device=dev)

    def sum_over_ranks(v: float) -> float:
        return v if dist is None else shard.sum_over_ranks(v, device=dev)

    # ---- warm-up
    for _ in range(max(args.warmup, 3)):
        batch.stage_run(ctx, db, cfg, out)
    torch.cuda.synchronize()

    # ---- device-resident timing
    stream = ctx.stream
    barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    launches0 = lib.gf_kernel_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        batch.stage_run(ctx, db, cfg, out)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = (lib.gf_kernel_launch_count() - launches0) // max(args.steps, 1)
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    total_particles = sum_over_ranks(float(hb.n))
    value = total_particles / (ms / 1e3)

    # ---- per-phase times (CUDA events between the phases of one step), then
    # the work counters from a separately instrumented step
    _, st = batch.stage_run(ctx, db, cfg, out, stats=True)
    phases = {k[3:]: st[k] for k in st if k.startswith("ms_") and k != "ms_pad"}
    cfg_count = batch.stage_config(mesh=mesh_rule, knn_k=K_NEIGH, count_work=True, mesh_onchip=args.mesh_onchip)
    _, stc = batch.stage_run(ctx, db, cfg_count, out, stats=True)
    for key in ("pp_interactions", "pc_interactions", "knn_nodes", "knn_batches",
                "knn_candidates", "knn_single_inserts", "knn_bitonic_merges"):
        st[key] = stc[key]

    # ---- e2e through the public API with pinned host buffers
    hx = {k: torch.from_numpy(np.ascontiguousarray(getattr(hb, k))).pin_memory()
          for k in ("x", "y", "z", "mass")}
    htype = torch.from_numpy(hb.type).pin_memory()
    hps = torch.from_numpy(hb.pstart).pin_memory()
    o_host = {"nearindex": torch.empty((hb.n, K_NEIGH), dtype=torch.int32).pin_memory(),
              "dens_sph": torch.empty(hb.n, dtype=torch.float32).pin_memory(),
              "dens_mesh": torch.empty(hb.n, dtype=torch.float32).pin_memory(),
              "penergy": torch.empty(hb.n, dtype=torch.float32).pin_memory()}
    h2d = sum(t.numel() * t.element_size() for t in list(hx.values()) + [htype, hps])
    d2h = sum(t.numel() * t.element_size() for t in o_host.values())

    def e2e_step():
        with torch.cuda.stream(stream):
            for k in ("x", "y", "z", "mass"):
                getattr(db, k).copy_(hx[k], non_blocking=True)
            db.type.copy_(htype, non_blocking=True)
            db.pstart.copy_(hps, non_blocking=True)
        batch.stage_run(ctx, db, cfg, out)
        with torch.cuda.stream(stream):
            for k, t in o_host.items():
                t.copy_(getattr(out, k), non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1) / args.steps)
    e2e_value = total_particles / (e2e_ms / 1e3)

    # ---- the same two measurements through the pipelined stage: halo chunks
    # on their own streams and host threads, so copies and host-side syncs
    # of one chunk overlap the kernels of the others
    pipe = batch.PipelinedStage(hb, cfg, nchunk=args.chunks, device=local, k=K_NEIGH)
    pipe_res = {}
    for mode in ("resident", "e2e"):
        runner = pipe.run_resident if mode == "resident" else pipe.run_e2e
        runner(max(args.warmup, 3))
        torch.cuda.synchronize()
        barrier()
        l0 = lib.gf_kernel_launch_count()
        p0, p1 = runner(args.steps)  # each chunk streams its K passes back to back
        torch.cuda.synchronize()
        pms = max_over_ranks(p0.elapsed_time(p1) / args.steps)
        pipe_res[mode] = {"value": total_particles / (pms / 1e3), "ms_per_step": pms,
                          "launches": (lib.gf_kernel_launch_count() - l0) // max(args.steps, 1)}
    nchunks = len(pipe.chunks)
    pipe_h2d, pipe_d2h = int(pipe.h2d_bytes), int(pipe.d2h_bytes)
    pipe.close()
    del pipe

    # ---- the stage captured as CUDA graphs: the whole catalogue as one graph
    # on one stream, and each chunk of the pipelined stage as its own graph;
    # every replay runs every kernel of the stage on the resident inputs
    graph_res = graph_measurements(args, hb, cfg, ctx, db, out, total_particles, barrier, max_over_ranks)
    clk = clocks.stop()
    # the headline path: the pipelined stage replaying its captured graphs
    # (every kernel of the stage runs each pass); eager launches beside it
    use_graph = "pipelined_resident" in graph_res
    head = graph_res["pipelined_resident"] if use_graph else pipe_res["resident"]
    head_e2e = graph_res["pipelined_e2e"] if use_graph else pipe_res["e2e"]

    # ---- plain GPU path: every phase in FP64 (plain_fp64), one halo per
    # gf_stage_run call, inputs resident; and, for the batching's own gain,
    # the same FP32 kernels one halo per call
    def one_halo_per_call(c):
        views = batch.HaloViews(db, out, K_NEIGH, hb.pstart)
        views.run(ctx, c, halos=range(min(64, hb.nhalo)))
        torch.cuda.synchronize()
        barrier()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        views.run(ctx, c)
        g1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(g0.elapsed_time(g1))

    cfg64 = batch.stage_config(mesh=mesh_rule, knn_k=K_NEIGH, plain_fp64=True)
    plain_ms = one_halo_per_call(cfg64)
    plain32_ms = one_halo_per_call(cfg)
    headline = head["value"]
    plain = {"value": total_particles / (plain_ms / 1e3), "unit": UNIT, "ms_per_step": plain_ms,
             "path": "plain FP64 stage: every phase in FP64 (exact FP64 kNN, FP64 TSC/FFT/findDen meshes, "
                     "FP64 Barnes-Hut terms), one halo per gf_stage_run call, device-resident inputs",
             "batched_over_plain": headline / (total_particles / (plain_ms / 1e3)),
             "fp32_one_halo_per_call": {"value": total_particles / (plain32_ms / 1e3), "ms_per_step": plain32_ms,
                                        "batched_over_it": headline / (total_particles / (plain32_ms / 1e3))}}

    # ---- roofline of the dominant kernel
    pk = peaks()
    dom = max(phases, key=phases.get)
    n = hb.n
    cells = st["mesh_cells"]
    # algorithmic bytes per launch of each phase: recentre reads FP64 x, y, z,
    # m and writes FP64 x, y, z + float4 (52 B); kNN reads a float4 and
    # writes k int32 indices and a float density; TSC reads FP64 x, y, z, m
    # and writes the mesh once; smoothing reads and writes the mesh twice
    # (16 B per cell floor); findDen reads FP64 x, y, z, the mesh, writes a float
    # (its 27-cell stencils re-read the mesh the smoothing has just written,
    # shared between neighbouring particles: working set, not counted).
    # Meshes of 64^3 never reach device memory: the on-chip kernel (in the
    # smoothing phase) reads FP64 x, y, z, m and the type of their particles
    # for the deposit, x, y, z again for the interpolation, and writes a float
    dev_cells = st.get("mesh_cells_device", cells)
    n_chip = st.get("onchip_particles", 0)
    n_dev = n - n_chip
    alg = {"recentre": 52 * n, "tree": 0, "knn": (16 + 4 * K_NEIGH + 4) * n,
           "tsc": 32 * n_dev + 4 * dev_cells, "smooth": 16 * dev_cells + 64 * n_chip,
           "findden": 28 * n_dev, "potential": 0}
    # the whole stage's algorithmic bytes per step against HBM, for the
    # batched (pipelined and single-stream) and plain paths
    stage_bytes = float(sum(alg.values()))

    def stage_frac(ms_step):
        return {"achieved_gbs": stage_bytes / (ms_step / 1e3) / 1e9,
                "frac": stage_bytes / (ms_step / 1e3) / 1e9 / pk["hbm_gbs"]}
    plain["stage_roofline"] = stage_frac(plain_ms)
    roofline = None
    if alg.get(dom):
        achieved = alg[dom] / (phases[dom] / 1e3) / 1e9
        traffic = TRAFFIC_PER_PARTICLE.get(dom)
        roofline = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"],
                    "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                    "traffic": None if traffic is None else traffic * n,
                    "traffic_note": "bytes per launch, ncu capture of the 1024-halo catalogue scaled by particles",
                    "algorithmic_bytes": alg[dom], "peak_source": pk["source"]}
        if dom == "knn":
            roofline["limiter"] = KNN_LIMITER
    else:
        # dominant phase has no HBM-bound roofline (tree build / FP32 potential walk);
        # report the largest HBM-bound phase instead
        cand = {k: v for k, v in phases.items() if alg.get(k)}
        k2 = max(cand, key=cand.get)
        achieved = alg[k2] / (phases[k2] / 1e3) / 1e9
        roofline = {"kernel": k2, "bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"],
                    "unit": "GB/s", "frac": achieved / pk["hbm_gbs"], "traffic": None,
                    "peak_source": pk["source"], "dominant_phase": dom}

    # the kNN kernel's own work counters, per query
    algo = _lib.tuning_value("GF_KNN_ALGO")
    if algo in (1, 2):
        names = ("node_tests_per_bucket", "particle_tests_per_bucket", "heap_insertions",
                 "warp_insertion_steps_per_bucket",
                 "buckets_per_query" if algo == 1 else "uncertified_fraction")
        per = {"node_tests_per_bucket": 32, "particle_tests_per_bucket": 32,
               "warp_insertion_steps_per_bucket": 32}
        kernel = ("knn_bucket_kernel (lane = query, 32 tree-order queries per warp)" if algo == 1 else
                  "knn_fbucket_kernel (lane = query, float heap keys, exact FP64 certification; "
                  "uncertified queries redone by knn_kernel)")
    else:
        names = ("nodes", "batches", "candidates", "single_inserts", "bitonic_merges")
        per = {}
        kernel = "knn_kernel (warp = query)"
    knn_work = {"kernel": kernel}
    for nm, key in zip(names, ("knn_nodes", "knn_batches", "knn_candidates", "knn_single_inserts",
                               "knn_bitonic_merges")):
        knn_work[nm] = st[key] / max(hb.n, 1) * per.get(nm, 1)

    line = dict(base)
    line.update({
        "value": head["value"], "ms_per_step": head["ms_per_step"],
        "config": workload_config(args, hb, world, int(cells)),  # the same object as the reference arm's
        "pipeline": (f"{nchunks} halo chunks on their own streams and host threads"
                     + (", each replaying its stage captured as one CUDA graph" if use_graph else "")),
        "tree_nodes": int(st["nnode"]),
        "meshes": {"cells_planned": int(cells), "cells_in_device_memory": int(dev_cells),
                   "onchip_meshes": int(st.get("onchip_meshes", 0)), "onchip_particles": int(n_chip),
                   # the smoothing passes skip pencils that are all zero (outside
                   # the cells the TSC stencils reach) and, on the last pass, the
                   # columns no findDen stencil reads
                   "smoothing_pass_cells": int(st.get("mesh_pass_cells", 0)),
                   "smoothing_pass_fraction": (st.get("mesh_pass_cells", 0) / (3.0 * dev_cells)
                                               if dev_cells else None)},
        "e2e": {"value": head_e2e["value"], "unit": UNIT, "h2d_bytes_per_step": pipe_h2d,
                "d2h_bytes_per_step": pipe_d2h, "ms_per_step": head_e2e["ms_per_step"],
                "path": "PipelinedStage.run_e2e(K): pinned host inputs in, all outputs back to pinned host, "
                        "every pass; each chunk streams its K passes back to back"
                        + (" (graph replays)" if use_graph else "")},
        "eager_pipelined": {"value": pipe_res["resident"]["value"], "ms_per_step": pipe_res["resident"]["ms_per_step"],
                            "e2e": {"value": pipe_res["e2e"]["value"], "ms_per_step": pipe_res["e2e"]["ms_per_step"]},
                            "gpu_launches": int(pipe_res["resident"]["launches"]),
                            "path": "PipelinedStage with one gf_stage_run call per chunk and pass"},
        "stage_roofline": dict(stage_frac(head["ms_per_step"]), bytes_per_step=stage_bytes,
                               note="all phases' algorithmic bytes per step (tree and potential count none) "
                                    "over the step time, of measured HBM peak"),
        "single_stream": {"value": value, "ms_per_step": ms, "gpu_launches": int(launches),
                          "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                                  "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms},
                          "path": "one gf_stage_run call over the whole catalogue"},
        "roofline": roofline,
        "phases_ms": phases,
        "interactions": {"particle_particle": st["pp_interactions"],
                         "particle_cell": st["pc_interactions"]},
        "knn_work_per_query": knn_work,
        "plain": plain,
        # kernels of this repo per step: the kernel nodes of the chunks' graphs
        # (replays do not pass the host-side launch counter), else the launches
        "gpu_launches": int(head["kernel_nodes_per_step"]) if use_graph else int(pipe_res["resident"]["launches"]),
        "graph": graph_res,
        "clocks": clk,
    })

    # ---- CPU baseline (the reference's own code on a bounded stratified
    # sample), the drop-in path on one step of that sample, and the stage's
    # accuracy on sampled halos against the oracle
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rb = reference_baseline(hb, steps=1, warmup=1)
            line["cpu_baseline"] = {"value": rb["value"], "unit": UNIT, "cores": rb["cores"],
                                    "kind": "reference", "sample": reference_sample_text(rb, hb),
                                    "strata": rb["strata"], "catalogue_seconds": rb["extrap_s"]}
            halos = [h for s_ in stratified_sample(hb, 0) for h in s_]
            npart = int(halo_counts(hb)[halos].sum())
            # one untimed pass over the same halos first: the default context's
            # buffers grow to the largest halo once, as in a long-running caller
            run_dropin_stage(hb, halos, mesh_rule)
            td = run_dropin_stage(hb, halos, mesh_rule)
            line["plain"]["dropin"] = {
                "value": npart / td, "unit": UNIT, "seconds": td,
                "path": "reference signatures (findsphdensity, assign_density_TSC, "
                        "gaussian_Smoothing, findDen, Self_Halo_Potent), host buffers, "
                        "one halo per call, on one step of the cpu_baseline sample "
                        f"({len(halos)} halos, {npart} particles)"}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": None, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    if rank == 0 and world == 1 and not args.no_accuracy:
        halos = accuracy_sample(hb)
        line["accuracy"] = accuracy_check(ctx, db, cfg, hb, mesh_rule, halos)
    if rank == 0 and world == 1 and args.configs:
        line["single_halo_workloads"] = single_halo_configs(dev)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
