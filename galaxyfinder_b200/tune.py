"""Autotuner of libgf's compile-time launch parameters (csrc/gf_tuning.cuh).

    python -m galaxyfinder_b200.tune [--nhalo 4096] [--steps 5]     # on a GPU

For each group of parameters it builds variants of the one translation unit
that uses them (the other objects are reused), times the stage phase that the
group drives on a seeded catalogue (gf_stage_run's own per-phase CUDA-event
times, best of --steps after warm-up), and keeps the fastest; groups are
tuned one after another, each with the best values of the ones before.  The
result goes to galaxyfinder_b200/tuned.json (parameters, every measurement,
the GPU and the workload), which build.py turns into -D flags.

  group   parameters                                   phase
  knn     GF_KNN_ALGO x GF_KNNB_BLOCK (x GF_KNNB_ARITY), then GF_KNNB_SEEDS,
          GF_KNNB_LANECERT, GF_KNNB_DYN, GF_KNNB_WIN x GF_KNNB_MINB
          (node window against resident blocks), GF_KNNB_QUEUE and
          GF_KNNB_FILT x GF_KNNB_HEAPF (tile filter, heap order) for the
          float-key kernel; for the warp-per-query
          kernel GF_KNN_CHUNK, then GF_KNN_BLOCK x register cap   knn
  bh      GF_BH_DYN, GF_BH_ACC, GF_BH_TMA (leaf staging), GF_BH_LEAF4, GF_BH_BLOCK,
          then the register cap                        potential
  fft     GF_FFT_PENCILS                               smooth
  tsc     GF_TSC_TILE (0: direct global atomics)       tsc
  tree    GF_TREE_BLOCK                                tree

The register cap is expressed as GF_*_MINB = 65536 / (block * registers).
Leaf size is not a parameter: the octree follows the reference's node rule
(a node is split when it holds at least 10 particles, tree.h:20).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import datetime
import json
import os
import subprocess
import sys
from pathlib import Path

from . import build as B

TUNE_DIR = B.PKG / "_tune"
DEFAULTS = {"GF_KNN_ALGO": 2, "GF_KNNB_BLOCK": 64, "GF_KNNB_ARITY": 2, "GF_KNNB_SEEDS": 64, "GF_KNNB_QUEUE": 0, "GF_KNNB_LANECERT": 0,
            "GF_KNN_BLOCK": 256, "GF_KNN_MINB": 1, "GF_KNN_CHUNK": 32,
            "GF_BH_BLOCK": 128, "GF_BH_DYN": 0, "GF_BH_ACC": 0, "GF_BH_TMA": 0, "GF_BH_LEAF4": 0, "GF_KNNB_FILT": 0, "GF_KNNB_HEAPF": 0, "GF_KNNB_DYN": 0, "GF_KNNB_WIN": 32, "GF_KNNB_MINB": 1,
            "GF_BH_MINB": 1, "GF_FFT_PENCILS": 32, "GF_FFT_PENCILS_64": 32, "GF_FFT_PENCILS_128": 32, "GF_TSC_TILE": 0, "GF_TREE_BLOCK": 256}
REGCAPS = (255, 64, 48)


def minb(block: int, regs: int) -> int:
    return max(1, 65536 // (block * regs)) if regs < 255 else 1


# group -> stages; each stage maps the current best parameters to a list of
# overrides (an empty list skips the stage)
def stages(group: str):
    if group == "knn":
        return [lambda base: [{"GF_KNN_ALGO": a, "GF_KNNB_BLOCK": b, "GF_KNNB_ARITY": 2}
                              for a in (1, 2) for b in (32, 64, 128)] +
                [{"GF_KNN_ALGO": 1, "GF_KNNB_BLOCK": 32, "GF_KNNB_ARITY": 4}, {"GF_KNN_ALGO": 0}],
                lambda base: [] if base["GF_KNN_ALGO"] != 2 else [{"GF_KNNB_SEEDS": n} for n in (32, 48, 64, 80, 96)],
                lambda base: [] if base["GF_KNN_ALGO"] != 2 else [{"GF_KNNB_LANECERT": c} for c in (0, 1)],
                lambda base: [] if base["GF_KNN_ALGO"] != 2 else [{"GF_KNNB_DYN": d} for d in (0, 1)],
                lambda base: [] if base["GF_KNN_ALGO"] != 2 else
                [{"GF_KNNB_WIN": w, "GF_KNNB_MINB": mb} for w, mb in ((32, 1), (8, 6), (0, 6), (0, 1))],
                lambda base: [] if base["GF_KNN_ALGO"] != 2 else [{"GF_KNNB_QUEUE": q} for q in (0, 2, 4, 8)],
                lambda base: [] if base["GF_KNN_ALGO"] != 2 else
                [{"GF_KNNB_FILT": f, "GF_KNNB_HEAPF": h} for f in (0, 1) for h in (0, 1, 2, 3)],
                lambda base: [] if base["GF_KNN_ALGO"] != 0 else [{"GF_KNN_CHUNK": c} for c in (16, 32, 64)],
                lambda base: [] if base["GF_KNN_ALGO"] != 0 else
                [{"GF_KNN_BLOCK": b, "GF_KNN_MINB": minb(b, r)} for b in (128, 256) for r in REGCAPS]]
    if group == "bh":
        return [lambda base: [{"GF_BH_DYN": d} for d in (0, 1)],
                lambda base: [{"GF_BH_ACC": a} for a in (0, 1)],
                lambda base: [{"GF_BH_TMA": t} for t in (0, 1)],
                lambda base: [{"GF_BH_LEAF4": v} for v in (0, 1)],
                lambda base: [{"GF_BH_BLOCK": b, "GF_BH_MINB": 1} for b in (64, 128, 256)],
                lambda base: [{"GF_BH_MINB": minb(base["GF_BH_BLOCK"], r)} for r in REGCAPS]]
    if group == "fft":
        return [lambda base: [{"GF_FFT_PENCILS": p} for p in (16, 32)],
                lambda base: [{"GF_FFT_PENCILS_64": p} for p in (32, 64, 128)],
                lambda base: [{"GF_FFT_PENCILS_128": p} for p in (32, 64)]]
    if group == "tsc":
        return [lambda base: [{"GF_TSC_TILE": c} for c in (0, 4096, 8192)]]
    if group == "tree":
        return [lambda base: [{"GF_TREE_BLOCK": b} for b in (128, 256, 512)]]
    raise ValueError(group)


GROUPS = {"knn": ("gf_knn.cu", "knn"), "bh": ("gf_potent.cu", "potential"),
          "fft": ("gf_smooth.cu", "smooth"), "tsc": ("gf_tsc.cu", "tsc"), "tree": ("gf_tree.cu", "tree")}


def variant_name(params: dict) -> str:
    name = "_".join(f"{k[3:].lower()}{v}" for k, v in sorted(params.items()))
    if len(name) > 160:  # a directory name: keep it short, and unique by digest
        import hashlib
        name = "v" + hashlib.sha1(name.encode()).hexdigest()[:16]
    return name


def build_variant(src_name: str, params: dict) -> Path:
    """libgf with src_name compiled for params and every other object reused."""
    d = TUNE_DIR / variant_name(params)
    d.mkdir(parents=True, exist_ok=True)
    lib = d / "libgf.so"
    if lib.exists():
        return lib
    obj = d / (Path(src_name).stem + ".o")
    B.compile_one(B.CSRC / src_name, obj, params)
    objs = [obj if o.name == obj.name else o for o in sorted(B.BUILD.glob("*.o"))]
    B.link(objs, lib)
    return lib


def measure(lib: Path, nhalo: int, steps: int) -> dict:
    """Runs this module with --measure against lib in a fresh process."""
    env = dict(os.environ, GF_LIBGF=str(lib))
    out = subprocess.run([sys.executable, "-m", "galaxyfinder_b200.tune", "--measure", "--nhalo", str(nhalo),
                          "--steps", str(steps)], env=env, capture_output=True, text=True, check=True,
                         cwd=str(B.ROOT))
    return json.loads(out.stdout.strip().splitlines()[-1])


def _measure_main(nhalo: int, steps: int) -> None:
    import torch

    from . import _lib, batch, synth
    hb = synth.catalogue(seed=synth.SEED_BASE + 2, nhalo=nhalo)
    ctx = batch.Context(0)
    db = batch.DeviceBatch.from_halobatch(hb)
    rule = batch.mesh_rule(mode=_lib.MESH_POW2, nmin=64, nmax=256, rg=2.0, rg_in_cells=True)
    cfg = batch.stage_config(mesh=rule, knn_k=32)
    out = batch.StageBuffers(hb.n, 32, torch.device("cuda", 0))
    for _ in range(3):
        batch.stage_run(ctx, db, cfg, out)
    best = {}
    for _ in range(steps):
        _, st = batch.stage_run(ctx, db, cfg, out, stats=True)
        for k, v in st.items():
            if k.startswith("ms_") and k != "ms_pad":
                best[k[3:]] = min(best.get(k[3:], 1e30), v)
    torch.cuda.synchronize()
    print(json.dumps(best))


def tune(nhalo: int, steps: int, groups=("knn", "bh", "fft", "tsc", "tree")) -> dict:
    B.build()
    base = dict(DEFAULTS)
    base.update(B.tuned_params())
    log = {}
    for g in groups:
        src, phase = GROUPS[g]
        log[g] = []
        for stage_fn in stages(g):
            stage = stage_fn(base)
            if not stage:
                continue
            cands = [dict(base, **ov) for ov in stage]
            with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
                libs = list(ex.map(lambda p: build_variant(src, p), cands))
            keys = sorted(set().union(*(ov.keys() for ov in stage)))
            timed = []
            for p, lib in zip(cands, libs):
                ms = measure(lib, nhalo, steps)[phase]
                timed.append((ms, p))
                shown = {k: p[k] for k in keys}
                log[g].append({"params": shown, "ms": ms})
                print(f"{g}: {variant_name(shown)}: {phase} {ms:.3f} ms", flush=True)
            ref_ms = next(ms for ms, p in timed if p == base) if base in [p for _, p in timed] else None
            ms, p = min(timed, key=lambda t: t[0])
            if ref_ms is None or ms < 0.99 * ref_ms:  # keep the incumbent unless >1% faster
                base = p
    import torch
    if B.TUNED.exists():  # keep the measurements of the groups not re-run
        prev = json.loads(B.TUNED.read_text())
        log = {**prev.get("measured", {}), **log}
        groups = tuple(dict.fromkeys(list(prev.get("phase_of_group", {})) + list(groups)))
    res = {"params": base, "measured": log, "phase_of_group": {g: GROUPS[g][1] for g in groups},
           "workload": f"seeded catalogue, {nhalo} halos (N_p ~ N^-1.9 on [100, 2e6]), best of {steps} steps",
           "gpu": torch.cuda.get_device_name(0), "date": datetime.date.today().isoformat()}
    B.TUNED.write_text(json.dumps(res, indent=1) + "\n")
    return res


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--nhalo", type=int, default=4096)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--measure", action="store_true")
    ap.add_argument("--groups", default="knn,bh,fft,tsc,tree")
    a = ap.parse_args()
    if a.measure:
        _measure_main(a.nhalo, a.steps)
    else:
        res = tune(a.nhalo, a.steps, tuple(a.groups.split(",")))
        print(json.dumps(res["params"]))


if __name__ == "__main__":
    main()
