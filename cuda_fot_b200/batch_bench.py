"""Batch benchmark: many meshes of uneven size in one persistent launch.

    python -m cuda_fot_b200.batch_bench [--meshes 512] [--timesteps 100] [--seed 1]

Workload: `--meshes` meshes, half res_calc 2D quad meshes (edge -> cell
increment, FP64) and half volna shallow-water triangle meshes (edge flux
added to 2 cells, FP32), with cell counts drawn log-uniform between 4,000 and
1,000,000 from the seed.  The autotuner measures the batch under each plan
kind (atomic with / without warp aggregation, hierarchical with blocks of 64,
128, 256) and keeps the fastest, then:

  * batch_graph: a CUDA graph of `--timesteps` batched launches (one launch
    per timestep over all meshes' tiles), replayed;
  * batch_run:   the same timesteps as one Plan-like call (one launch);
  * loop_atomic: the plain method, one atomic launch per mesh per timestep
    from the host (`--meshes` x `--timesteps` launches);
  * loop_atomic_graph: those launches captured in one CUDA graph;
  * loop_hier:   one hierarchical launch per mesh per timestep.

GB/s counts each mesh's unique bytes once per timestep (as bench.py).  One
JSON line is printed.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np


def make_meshes(n: int, seed: int):
    from . import meshgen as mg
    rng = np.random.default_rng(seed)
    cells = np.exp(rng.uniform(np.log(4e3), np.log(1e6), n))
    out = []
    for i, c in enumerate(cells):
        if i % 2 == 0:
            s = max(2, int(round(np.sqrt(c))))
            out.append(mg.res_calc(s, s, seed * 100003 + i))
        else:
            s = max(2, int(round(np.sqrt(c / 2))))
            out.append(mg.volna(s, s, seed * 100003 + i))
    return out


def timed(fn, stream, reps=1):
    import torch
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        fn()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / 1e3 / reps


def run(meshes: int = 512, timesteps: int = 100, seed: int = 1) -> dict:
    """The batch benchmark; returns its JSON line as a dict."""
    a = argparse.Namespace(meshes=meshes, timesteps=timesteps, seed=seed)
    import torch
    from . import fot as F
    from . import meshgen as mg

    t0 = time.time()
    mds = make_meshes(a.meshes, a.seed)
    gen_s = time.time() - t0
    ub = float(sum(md.unique_bytes() for md in mds))
    n_cells = {"res_calc": int(sum(md.n_points[0] for md in mds if md.loop == mg.RES_CALC)),
               "volna": int(sum(md.n_points[0] for md in mds if md.loop == mg.VOLNA))}
    # two copies of every mesh on the GPU: hierarchical plans renumber their
    # problem's cells into colour order, atomic plans run on the given order
    t0 = time.time()
    probs_a = [F.Problem.from_mesh(md) for md in mds]
    probs_h = [F.Problem.from_mesh(md) for md in mds]
    upload_s = time.time() - t0
    st = torch.cuda.Stream()
    T = a.timesteps

    # the autotuner's choice of the batch's plan kind and block size
    kinds = [("atomic", F.EXEC_ATOMIC, 256, 0), ("atomic-plain", F.EXEC_ATOMIC, 256, F.PLAN_NO_AGGREGATE),
             ("hier/64", F.EXEC_HIER, 64, 0), ("hier/128", F.EXEC_HIER, 128, 0),
             ("hier/256", F.EXEC_HIER, 256, 0)]
    tune = {}
    best = None
    for name, ex, blk, flags in kinds:
        t1 = time.time()
        probs = probs_a if ex == F.EXEC_ATOMIC else probs_h
        plans = [p.plan(ex, blk, flags) for p in probs]
        plan_s = time.time() - t1
        b = F.Batch(plans)
        b.run(2, st)
        b.sync(st)
        secs = timed(lambda: b.run(5, st), st) / 5
        b.sync(st)
        tune[name] = {"us_per_step": secs * 1e6, "gbs": ub / secs / 1e9, "plan_build_s": round(plan_s, 2)}
        if best is None or secs < best[1]:
            best = ((name, ex, blk, flags), secs)
        del b, plans
    name, ex, blk, flags = best[0]
    plans = [p.plan(ex, blk, flags) for p in (probs_a if ex == F.EXEC_ATOMIC else probs_h)]
    batch = F.Batch(plans)
    batch.run(2, st)
    batch.sync(st)

    res = {}
    # one persistent launch per timestep, captured in a CUDA graph
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=st):
        for _ in range(T):
            batch.run(1, st)
    g.replay()
    torch.cuda.synchronize()
    secs = timed(g.replay, torch.cuda.current_stream(), 3) / T
    batch.sync(st)
    res["batch_graph"] = secs
    del g
    # all timesteps in one launch
    secs = timed(lambda: batch.run(T, st), st) / T
    batch.sync(st)
    res["batch_run"] = secs
    del batch, plans
    # per-mesh hierarchical launches from the host
    hplans = [p.plan(F.EXEC_HIER, 128) for p in probs_h]

    def loop_hier():
        for pl in hplans:
            pl.run(1, st)
    loop_hier()
    torch.cuda.synchronize()
    res["loop_hier"] = timed(loop_hier, st, 3)
    for p in probs_h:
        p.sync(st)
    del hplans
    # the plain method: one atomic launch per mesh per timestep
    aplans = [p.plan(F.EXEC_ATOMIC, 256, F.PLAN_NO_AGGREGATE) for p in probs_a]

    def loop_atomic():
        for pl in aplans:
            pl.run(1, st)
    loop_atomic()
    torch.cuda.synchronize()
    res["loop_atomic"] = timed(loop_atomic, st, min(T, 10))
    g2 = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g2, stream=st):
        for _ in range(min(T, 10)):
            loop_atomic()
    g2.replay()
    torch.cuda.synchronize()
    res["loop_atomic_graph"] = timed(g2.replay, torch.cuda.current_stream(), 3) / min(T, 10)
    del g2
    for p in probs_a:
        p.sync(st)

    line = {"metric": "batched indirect loops, aggregate GB/s of unique bytes",
            "unit": "GB/s", "meshes": a.meshes, "timesteps": T, "seed": a.seed,
            "cells": n_cells, "unique_bytes_per_step": ub,
            "batch_plan": name, "autotune": tune,
            "us_per_step": {k: v * 1e6 for k, v in res.items()},
            "gbs": {k: ub / v / 1e9 for k, v in res.items()},
            "speedup_batch_graph_vs_loop_atomic": res["loop_atomic"] / res["batch_graph"],
            "speedup_batch_graph_vs_loop_atomic_graph": res["loop_atomic_graph"] / res["batch_graph"],
            "host_s": {"mesh_generation": round(gen_s, 1), "upload": round(upload_s, 1)}}
    return line


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--meshes", type=int, default=512)
    ap.add_argument("--timesteps", type=int, default=100)
    ap.add_argument("--seed", type=int, default=1)
    a = ap.parse_args(argv)
    print(json.dumps(run(a.meshes, a.timesteps, a.seed)), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
