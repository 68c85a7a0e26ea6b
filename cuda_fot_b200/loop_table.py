"""Per-loop measurement table: plain atomics vs the tuned plan, % of roofline.

    python -m cuda_fot_b200.loop_table [--loops res_calc mini_aero lulesh volna getacc]

For each benchmark mesh (seed 1):

  res_calc   1000 x 1000 quads, 1,998,000 edges, the generator's (natural) order
  mini_aero  128^3 hexes, 6,242,304 faces, seeded random cell numbering
  lulesh     96^3 hexes, seeded random node numbering (worst locality)
  volna      1024 x 1024 quads split into triangles
  getacc     1024 x 1024 quads

it measures the plain method (atomic executor without warp aggregation, on
the mesh as given), every candidate of the autotuner's default sweep (orderings
x executors x block sizes, partitioned variants), and the cost model's pick
when a trained model is present; it prints one JSON line per loop with
microseconds and GB/s of unique bytes per iteration, the fraction of the
measured HBM copy peak (MEASURED_PEAKS.json), the sweep's best, the model's
regret against it, and the speedups over the plain method.  Timing: CUDA
events around one Plan.run(K) call after warm-up (K iterations in one call).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

from . import meshgen as mg
from . import tune as T

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

MESHES = {
    "res_calc": lambda: mg.res_calc(1000, 1000, 1),
    "mini_aero": lambda: mg.mini_aero(128, 1, permute=True),
    "lulesh": lambda: mg.lulesh(96, 1, permute=True),
    "volna": lambda: mg.volna(1024, 1024, 1),
    "getacc": lambda: mg.getacc(1024, 1024, 1),
}


def peak_gbs() -> float:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except Exception:
        return 6650.0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--loops", nargs="+", default=list(MESHES))
    ap.add_argument("--iters", type=int, default=20)
    a = ap.parse_args(argv)
    from . import costmodel as CM
    model = CM.load_default()
    peak = peak_gbs()
    for name in a.loops:
        md = MESHES[name]()
        ub = md.unique_bytes()
        cache = T.OrderedCache(md)
        plain = T.measure(cache, T.Candidate(None, 0, "atomic", 256, aggregate=False), iters=a.iters)
        t0 = time.time()
        cands = T.default_candidates(md.loop)
        sweep = [T.measure(cache, c, iters=a.iters) for c in cands]
        sweep_s = time.time() - t0
        ok = [r for r in sweep if r["ok"]]
        best = min(ok, key=lambda r: r["seconds"])
        line = {"loop": name, "cells": int(md.n_cells), "unique_bytes": ub, "peak_gbs": peak,
                "plain_atomic": {"us": plain["seconds"] * 1e6, "gbs": plain["gbs"],
                                 "frac": plain["gbs"] / peak},
                "best": {"plan": best["cand"].label(), "us": best["seconds"] * 1e6, "gbs": best["gbs"],
                         "frac": best["gbs"] / peak,
                         "speedup_vs_plain": plain["seconds"] / best["seconds"]},
                "sweep_s": round(sweep_s, 1),
                "sweep": {r["cand"].label(): (round(r["seconds"] * 1e6, 1) if r["ok"] else None)
                          for r in sweep}}
        colour = [r for r in ok if r["cand"].exec != "atomic"]
        if colour:
            cb = min(colour, key=lambda r: r["seconds"])
            line["best_coloured"] = {"plan": cb["cand"].label(), "us": cb["seconds"] * 1e6, "gbs": cb["gbs"],
                                     "frac": cb["gbs"] / peak,
                                     "speedup_vs_plain": plain["seconds"] / cb["seconds"]}
        if model is not None:
            t1 = time.time()
            pick = CM.pick(model, md, cands)
            pick_s = time.time() - t1
            pr = next((r for r in sweep if r["cand"].label() == pick.label()), None)
            if pr is not None and pr["ok"]:
                line["model"] = {"plan": pick.label(), "us": pr["seconds"] * 1e6, "gbs": pr["gbs"],
                                 "frac": pr["gbs"] / peak, "regret": pr["seconds"] / best["seconds"] - 1.0,
                                 "speedup_vs_plain": plain["seconds"] / pr["seconds"],
                                 "pick_s": round(pick_s, 1)}
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
