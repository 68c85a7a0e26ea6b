"""The configurations bench.py measures besides its headline (mini_aero 128^3).

Each function returns a dict for one key of bench.py's JSON line:

* ``res_calc_1000``  res_calc on the 1000 x 1000 quad grid (1,998,000 edges,
  152.0 MB of unique bytes per iteration): the plain atomic method on the
  given numbering, the exhaustive measured sweep's best, the best coloured
  (hierarchical) plan, the cost model's pick, and the best and best coloured
  plans timed again with the L2 flushed before every iteration (152 MB is
  only ~1.2x the 126 MB L2);
* ``lulesh_96``      LULESH 96^3 with a seeded random node numbering: plain
  atomics as given, then after RCM reordering and RCM + partitioning;
* ``batch_512``      512 uneven meshes (half res_calc, half volna) over 100
  timesteps: one batched launch per timestep in a CUDA graph vs one atomic
  launch per mesh and timestep (cuda_fot_b200.batch_bench);
* ``cost_model``     the learned plan model trained on the committed corpus's
  training seeds and evaluated on its held-out seed: regret against the
  exhaustive sweep, the fixed default plan's regret, tuning time saved;
* ``atomic_spread``  run-to-run spread of the atomic executor (normwise
  relative difference between repeated runs from the same inputs; the
  coloured executors are bit-reproducible);
* ``plan_build``     GPU ordering and plan-build wall time for res_calc 1000^2
  and mini_aero 128^3, beside the reference's host builder
  (HierarchicalColourMemory, colouring.hpp:44-147) timed on the same mesh;
* ``airfoil_1000``   the Airfoil solver iteration around res_calc (save_soln,
  then twice adt_calc, res_calc, bres_calc, update: fot_airfoil_run, whose
  per-cell loops run fused) on the 1000 x 1000 mesh, with res_calc through the best atomic plan and through a
  coloured one: time per iteration (launched call by call, and replayed as
  one CUDA graph of the time loop), GB/s of the iteration's unique bytes,
  and the share of res_calc in it.
"""
from __future__ import annotations

import time
from typing import Optional

import numpy as np

from . import fot as F
from . import meshgen as mg
from . import tune as T


def _frac(gbs: float, peak: float) -> float:
    return gbs / peak


def flushed_seconds(p, plan, iters: int, stream) -> float:
    """Seconds per iteration with the L2 flushed (a 256 MB write) before each
    iteration; CUDA events on the launching stream around each Plan.run(1)."""
    import torch
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")
    plan.run(2, stream)
    p.sync(stream)
    total = 0.0
    for _ in range(iters):
        flush.fill_(1)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        plan.run(1, stream)
        b.record(stream)
        b.synchronize()
        total += a.elapsed_time(b) / 1e3
    p.sync(stream)
    return total / iters


def _entry(r: dict, ub: int, peak: float, plain_s: Optional[float] = None) -> dict:
    d = {"plan": r["cand"].label(), "us": round(r["seconds"] * 1e6, 2), "gbs": round(r["gbs"], 1),
         "frac": round(_frac(r["gbs"], peak), 4)}
    if plain_s:
        d["speedup_vs_plain_atomics"] = round(plain_s / r["seconds"], 3)
    return d


def res_calc_1000(model, peak: float, stream) -> dict:
    from . import costmodel as CM
    md = mg.res_calc(1000, 1000, 1)
    ub = md.unique_bytes()
    cache = T.OrderedCache(md)
    plain = T.measure(cache, T.Candidate(None, 0, "atomic", 256, aggregate=False), iters=20)
    cands = T.default_candidates(md.loop)
    out = {"workload": "res_calc 1000x1000 quads, 1,998,000 edges, FP64, generator numbering",
           "unique_bytes_per_iteration": ub, "candidates": len(cands),
           "plain_atomics": _entry(plain, ub, peak)}
    pick = None
    if model is not None:
        t0 = time.perf_counter()
        pick = CM.pick(model, md, cands)
        out["model_pick_s"] = round(time.perf_counter() - t0, 2)
    t0 = time.perf_counter()
    res = T.sweep(md, cands, iters=20, cache=cache)
    out["sweep_s"] = round(time.perf_counter() - t0, 1)
    ok = [r for r in res if r["ok"]]
    best = min(ok, key=lambda r: r["seconds"])
    out["sweep_best"] = _entry(best, ub, peak, plain["seconds"])
    col = [r for r in ok if r["cand"].exec != "atomic"]
    bc = min(col, key=lambda r: r["seconds"]) if col else None
    if bc:
        out["best_coloured"] = _entry(bc, ub, peak, plain["seconds"])
    if pick is not None:
        pr = next((r for r in ok if r["cand"].label() == pick.label()), None)
        if pr:
            out["model_pick"] = _entry(pr, ub, peak, plain["seconds"])
            out["model_pick"]["regret"] = round(pr["seconds"] / best["seconds"] - 1.0, 4)
    flushed = {}
    for name, r in (("sweep_best", best), ("best_coloured", bc)):
        if r is None:
            continue
        p, plan = T.build(cache.get(r["cand"].order, r["cand"].partition), r["cand"])
        s = flushed_seconds(p, plan, 10, stream)
        flushed[name] = {"plan": r["cand"].label(), "us": round(s * 1e6, 2),
                         "gbs": round(ub / s / 1e9, 1), "frac": round(_frac(ub / s / 1e9, peak), 4)}
        del plan, p
    out["l2_flushed"] = flushed
    return out


def lulesh_96(peak: float) -> dict:
    md = mg.lulesh(96, 1, permute=True)
    ub = md.unique_bytes()
    cache = T.OrderedCache(md)
    plain = T.measure(cache, T.Candidate(None, 0, "atomic", 256, aggregate=False), iters=20)
    out = {"workload": "LULESH 96^3 hexes, 884,736 elements, FP64, seeded random node numbering",
           "unique_bytes_per_iteration": ub, "plain_atomics_random_numbering": _entry(plain, ub, peak)}
    for name, (order, part) in (("after_rcm", ("rcm", 0)), ("after_rcm_partition256", ("rcm", 256))):
        res = T.sweep(md, T.plan_candidates(order, part), iters=20, cache=cache)
        ok = [r for r in res if r["ok"]]
        b = min(ok, key=lambda r: r["seconds"])
        out[name] = {"best": _entry(b, ub, peak, plain["seconds"])}
        col = [r for r in ok if r["cand"].exec != "atomic"]
        if col:
            out[name]["best_coloured"] = _entry(min(col, key=lambda r: r["seconds"]), ub, peak,
                                                plain["seconds"])
    return out


def batch_512(meshes: int = 512, timesteps: int = 100) -> dict:
    from . import batch_bench
    r = batch_bench.run(meshes, timesteps, 1)
    return {"workload": f"{meshes} meshes (half res_calc, half volna), cells log-uniform in "
                        f"[4e3, 1e6], {timesteps} timesteps",
            "unique_bytes_per_timestep": r["unique_bytes_per_step"], "batch_plan": r["batch_plan"],
            "gbs": {k: round(v, 1) for k, v in r["gbs"].items()},
            "us_per_timestep": {k: round(v, 1) for k, v in r["us_per_step"].items()},
            "speedup_batch_graph_vs_loop_atomic": round(r["speedup_batch_graph_vs_loop_atomic"], 3),
            "speedup_batch_graph_vs_loop_atomic_graph":
                round(r["speedup_batch_graph_vs_loop_atomic_graph"], 3)}


def cost_model() -> dict:
    from . import costmodel as CM
    import json
    import os
    if not os.path.exists(CM.DEFAULT_CORPUS):
        return {"error": "no committed corpus"}
    data = CM.load_corpus()
    info = json.loads(str(data["info"]))
    t0 = time.perf_counter()
    _, ev = CM.train_and_evaluate(data)
    ev = {k: v for k, v in ev.items() if k != "picks"}
    ev["corpus_timings"] = int(len(data["y"]))
    ev["corpus_meshes"] = len(info)
    ev["train_and_evaluate_s"] = round(time.perf_counter() - t0, 1)
    return ev


def atomic_spread(md: mg.MeshData, cand: T.Candidate, runs: int = 6) -> dict:
    """Normwise relative spread of repeated atomic runs from the same inputs
    (the summation order of atomics varies from run to run)."""
    cache = T.OrderedCache(md)
    mdo = cache.get(cand.order, cand.partition, cand.layout)
    p, plan = T.build(mdo, cand)
    outs = []
    for _ in range(runs):
        p.set_point_data(0, mdo.point_data[0])
        plan.run(1)
        p.sync()
        outs.append(p.point_weights(0).astype(np.float64))
    ref = outs[0]
    den = np.abs(ref).max() or 1.0
    diffs = [float(np.abs(o - ref).max() / den) for o in outs[1:]]
    return {"plan": cand.label(), "runs": runs, "max_normwise_diff": max(diffs),
            "identical_runs": int(sum(d == 0.0 for d in diffs)) + 1}


def airfoil_unique_bytes(md: mg.MeshData, ex: dict) -> int:
    """Algorithmic bytes of one Airfoil iteration in its fused form: twice
    res_calc (its unique bytes) and bres_calc (boundary maps and flags, the
    boundary cells' q, adt and res), the stage-1 cell pass (update + adt_calc:
    qold, res and adt read, q written, res zeroed, the cell->node map and
    node coordinates read, adt written) and the stage-2 pass that also saves
    qold for the next iteration."""
    nc, nn = md.n_points[0], md.n_points[1]
    nb = len(ex["bedge_to_cell"])
    nbc = len(np.unique(ex["bedge_to_cell"]))
    bres = nb * (8 + 4 + 4) + nbc * (32 + 8 + 64)
    adt = nc * 16 + nn * 16 + nc * 8
    update = nc * (32 + 64 + 8 + 32)
    return 2 * (md.unique_bytes() + bres) + 2 * (update + adt) + nc * 32


def airfoil_setup(md: mg.MeshData, ex: dict, cand: T.Candidate):
    """A problem holding md, ordered / partitioned on the GPU as the
    candidate says, the candidate's res_calc plan and the Airfoil step on it
    (its maps given in md's numbering)."""
    p = F.Problem.from_mesh(md)
    if cand.order is not None:
        p.reorder(T.ORDERS[cand.order], seed=1)
    flags = 0
    if cand.partition:
        p.partition(cand.partition)
        p.reorder_to_partition()
        p.renumber_points()
        flags |= F.PLAN_USE_PARTITION
    if cand.layout != md.layout:
        p.set_layout(cand.layout)
    if cand.direct:
        flags |= F.PLAN_DIRECT_READS
    if cand.exec == "atomic" and not cand.aggregate:
        flags |= F.PLAN_NO_AGGREGATE
    plan = p.plan(T.EXECS[cand.exec], cand.block, flags)
    af = F.Airfoil(p, ex["cell_to_node"], ex["bedge_to_node"], ex["bedge_to_cell"],
                   ex["bound"], ex["qinf"], ex["cfl"])
    return p, plan, af


def airfoil_1000(peak: float, stream, iters: int = 20) -> dict:
    import torch
    md = mg.res_calc(1000, 1000, 1)
    ex = mg.airfoil_extras(md)
    ub = airfoil_unique_bytes(md, ex)
    out = {"workload": "Airfoil iteration: save_soln + 2 x (adt_calc, res_calc, bres_calc, update) "
                       "on res_calc 1000x1000 (1,998,000 edges, 4,000 boundary edges), FP64",
           "unique_bytes_per_iteration": ub}
    for name, cand in (("atomic", T.Candidate("rcm", 0, "atomic", 256, aggregate=False, layout="soa")),
                       ("coloured", T.Candidate("rcm", 256, "hier", 256))):
        p, plan, af = airfoil_setup(md, ex, cand)
        af.run(plan, 3, stream, rms=False)
        p.sync(stream)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        af.run(plan, iters, stream, rms=False)
        b.record(stream)
        b.synchronize()
        secs = a.elapsed_time(b) / 1e3 / iters
        rms = af.run(plan, 1, stream)
        g = af.graph(plan, iters, stream)
        g.launch(stream)
        p.sync(stream)
        a.record(stream)
        g.launch(stream)
        b.record(stream)
        b.synchronize()
        gsecs = a.elapsed_time(b) / 1e3 / iters
        del g
        loop_s = T.time_plan(p, plan, iters, 3, stream)
        out[name] = {"res_calc_plan": cand.label(), "us_per_iteration": round(secs * 1e6, 2),
                     "graph_us_per_iteration": round(gsecs * 1e6, 2),
                     "graph_gbs": round(ub / gsecs / 1e9, 1),
                     "gbs": round(ub / secs / 1e9, 1), "frac": round(_frac(ub / secs / 1e9, peak), 4),
                     "res_calc_share": round(2 * loop_s / secs, 3), "rms_after": rms}
        del af, plan, p
    return out


def plan_build() -> dict:
    """GPU wall time of the RCM ordering and of a hierarchical plan build
    (blocks of 256, both kernel forms' data), beside the reference's host
    plan builder on the same res_calc mesh."""
    from oracle import oracle_py as O
    out = {}
    for name, md in (("res_calc_1000", mg.res_calc(1000, 1000, 1)),
                     ("mini_aero_128", mg.mini_aero(128, 1, permute=True))):
        p = F.Problem.from_mesh(md)
        p.sync()
        t0 = time.perf_counter()
        p.reorder(F.ORDER_RCM)
        t1 = time.perf_counter()
        plan = p.plan(F.EXEC_HIER, 256)
        t2 = time.perf_counter()
        st = plan.stats()
        out[name] = {"rcm_s": round(t1 - t0, 3), "plan_build_s": round(t2 - t1, 3),
                     "blocks": st["n_blocks"], "block_colours": st["n_colours"]}
        if name == "res_calc_1000" and O.ref_available():
            r = O.ref_hier_plan(md, 256)
            out[name]["reference_host_plan_s"] = round(r["seconds"], 3)
            out[name]["reference_blocks"] = r["n_blocks"]
            out[name]["reference_block_colours"] = r["n_colours"]
        del plan, p
    return out
