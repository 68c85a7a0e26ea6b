"""Benchmark: indirect-loop GB/s of the tuned plan vs plain atomics.

Workload (one "step" = one iteration of the loop over the whole mesh; the K
timed steps run as one Plan.run(K) call, as the reference's
Problem::loop*(num) runs and times `num` iterations per call):
mini_aero-style 3D face flux, FP64, 128^3 hex cells, 6,242,304 interior faces,
cell numbering a seeded random permutation; the plan (ordering + executor +
block size + point-data layout, AOS or SOA as the reference's Problem<SOA>)
is picked by the cost model when one is trained and available,
otherwise by the measured sweep of the autotuner.  GB/s counts the algorithmic
("unique") bytes of one step: every indirectly read dataset once, the
incremented dataset read and written once, every direct dataset once, the
mapping once.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fot|reference]

Multi-GPU: the loop is single-GPU (the engine does not shard a mesh), so N
GPUs run N independent replicas ("scaling": "weak"); value = the bytes all
ranks processed / the max over ranks of the timed region.

At N=1 the line also carries the other configurations under their own keys
(cuda_fot_b200/bench_configs.py): res_calc 1000^2 with an L2-flushed timing,
LULESH 96^3 before and after reordering, the 512-mesh batch, the cost
model's held-out regret, the atomic executor's run-to-run spread, the
plan-build times and the Airfoil iteration around res_calc; --no-extras
skips them.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Indirect-loop GB/s (% of HBM roofline), learned-tuned plan vs plain atomics"
WORKLOAD = "mini_aero 128^3 face flux (FP64), random cell numbering"


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic(kernel_key):
    """Per-launch DRAM traffic (bytes) of the dominant kernel and where it
    comes from, from the committed ncu summary (profiles/traffic.json)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            j = json.load(f)
        e = j[kernel_key]
        return float(e["bytes_per_launch"]), e.get("source")
    except Exception:
        return None, None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 100 ms by one
    `nvidia-smi -lms` process that runs across the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self._proc = None
        self._t = None

    def _read(self):
        for line in self._proc.stdout:
            v = [x.strip() for x in line.strip().split(",")]
            if len(v) >= 7:
                self.rows.append(v)

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            time.sleep(0.3)  # first sample before the timed region starts
        except Exception:
            self._proc = None
        return self

    def __exit__(self, *a):
        if self._proc is not None:
            time.sleep(0.15)
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
            if self._t:
                self._t.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for n, v in zip(names, r[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def dist_setup(gpus):
    import torch
    if gpus > 1 or "RANK" in os.environ:
        import torch.distributed as dist
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        local = int(os.environ.get("LOCAL_RANK", "0"))
        # one process per GPU over NCCL; gloo where no GPU is visible (the
        # host-side tests of the replica path)
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
        return rank, world, local
    return 0, 1, 0


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_workload(args):
    from cuda_fot_b200 import meshgen as mg
    return mg.mini_aero(args.n, seed=args.seed, permute=True)


def cpu_baseline(md, impl_kind=None):
    """The reference's own compiled serial loop (oracle/_ref) on one core, or
    the oracle port, over a bounded sample: one iteration of the whole mesh."""
    from oracle import oracle_py as O
    ub = md.unique_bytes()
    if O.ref_available():
        _, _, secs = O.ref_serial(md, 1)
        kind = "reference"
    else:
        t0 = time.perf_counter()
        O.serial(md, 1)
        secs = time.perf_counter() - t0
        kind = "port"
    return {"value": ub / secs / 1e9, "unit": "GB/s", "cores": 1, "kind": kind,
            "sample": "1 iteration of the full mesh, serial loop in cell order"}


def run_reference(args):
    """Reference arm: the reference's own CPU loop (OpenMP over its global
    colouring, all host threads) on the same workload."""
    from oracle import oracle_py as O
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    md = make_workload(args)
    ub = md.unique_bytes()
    cores = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    if O.ref_available():
        kind = "reference"
        for _ in range(max(0, min(args.warmup, 1))):
            O.ref_omp(md, 1)
        # steps are timed until about 90 s of host time are spent, so the
        # default step count finishes within minutes
        times = []
        t_wall = time.perf_counter()
        for _ in range(args.steps):
            _, _, t_loop, _ = O.ref_omp(md, 1)
            times.append(t_loop)
            if time.perf_counter() - t_wall > 90.0:
                break
        secs = sum(times) / len(times)
        sample = (f"loopCPUCellCentredOMP, 1 iteration of the full mesh per step (colouring "
                  f"excluded), {len(times)} of {args.steps} steps timed (90 s host-time cap)")
    else:
        kind = "port"
        t0 = time.perf_counter()
        n = 0
        for _ in range(args.steps):
            O.serial(md, 1)
            n += 1
            if time.perf_counter() - t0 > 90.0:
                break
        secs = (time.perf_counter() - t0) / n
        cores = 1
        sample = f"oracle serial loop, 1 iteration of the full mesh per step, {n} of {args.steps} steps timed"
    v = ub / secs / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "faces": md.n_cells,
                                            "cells": md.n_points[0], "unique_bytes_per_step": ub},
            "cpu_baseline": {"value": v, "unit": "GB/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="fot", choices=["fot", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the other configurations (res_calc 1000^2, LULESH 96^3, the 512-mesh "
                         "batch, the cost model's held-out regret, the atomic spread, plan builds, "
                         "the Airfoil iteration)")
    ap.add_argument("--plan", default=None,
                    help="force a plan by its label, order[+partN]/exec[d][-plain]/block[@soa], "
                         "e.g. rcm/atomic-plain/256@soa")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    rank, world, local = dist_setup(args.gpus)
    from cuda_fot_b200 import fot as F
    from cuda_fot_b200 import meshgen as mg
    from cuda_fot_b200 import tune as T

    md = make_workload(args)
    ub = md.unique_bytes()
    stream = torch.cuda.current_stream()

    # plan choice: the cost model's pick when a trained model is present, else
    # the measured sweep; the sweep also measures the model's pick (regret)
    from cuda_fot_b200.profile_case import parse_plan
    choice_src = "sweep"
    choice_note = None
    chosen = None
    pick_s = None
    try:
        from cuda_fot_b200 import costmodel as CM
        model = None if args.plan else CM.load_default()  # a forced plan needs no pick
        if model is not None:
            t_pick = time.perf_counter()
            chosen = CM.pick(model, md, T.default_candidates(md.loop))
            pick_s = time.perf_counter() - t_pick
            choice_src = "cost model"
        elif not args.plan:
            choice_note = "no trained model for the current features (cuda_fot_b200/model/costmodel.npz)"
    except Exception as e:  # the measured sweep stays the fallback
        chosen = None
        choice_note = f"cost model unavailable: {e}"
    cache = T.OrderedCache(md)
    if args.plan:
        chosen = parse_plan(args.plan)
        choice_src = "forced"
    sweep_res = []
    if choice_src != "forced":
        # the exhaustive measured sweep over the same candidates the model
        # picks from: the fallback, and the yardstick of the model's pick
        cands = T.default_candidates(md.loop)
        if chosen is not None and chosen.label() not in [c.label() for c in cands]:
            cands.append(chosen)
        t_sweep = time.perf_counter()
        sweep_res = T.sweep(md, cands, iters=5, warmup=3, cache=cache)
        sweep_s = time.perf_counter() - t_sweep
        if chosen is None:
            chosen = T.best(sweep_res)["cand"]
    atomic_plain = T.measure(cache, T.Candidate(None, 0, "atomic", 256, aggregate=False),
                             iters=10, warmup=3)

    md_run = cache.get(chosen.order, chosen.partition, chosen.layout)
    p, plan = T.build(md_run, chosen)
    # launches of one Plan.run(K) call: the atomic executor launches once per
    # iteration; the split write-back kernels once per iteration plus one
    # combine-only launch when blocks share points; the other persistent
    # hierarchical kernels once per call; the per-colour form once per colour
    # and iteration
    st0 = plan.stats()
    if chosen.exec == "atomic":
        launches = args.steps
    elif chosen.exec == "hier" and st0["kernel"].startswith("split"):
        launches = args.steps + (1 if st0["shared_points"] else 0)
    elif chosen.exec == "hier":
        launches = 1
    else:
        launches = args.steps * st0["n_colours"]

    # ---- timed region: inputs resident in HBM -------------------------------
    # K steps = one Plan.run(K) call (K iterations of the loop), as the
    # reference's Problem::loop*(num) runs and times `num` iterations per call
    plan.run(args.warmup, stream)
    p.sync(stream)
    barrier(world)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    # NVTX ranges name the timed launches for a profiler's launch list
    # (ncu --nvtx --nvtx-include "bench_timed/")
    with ClockSampler(local) as clocks:
        torch.cuda.nvtx.range_push("bench_timed")
        start.record(stream)
        plan.run(args.steps, stream)
        end.record(stream)
        torch.cuda.nvtx.range_pop()
        end.synchronize()
    p.sync(stream)
    torch.cuda.synchronize()
    barrier(world)
    secs = start.elapsed_time(end) / 1e3
    secs_max = max_over_ranks(secs, world)
    value = ub * args.steps * world / secs_max / 1e9

    # ---- e2e: through the public API with host buffers ------------------------
    host_in = []
    for k in range(p.info.n_point_sets):
        host_in.append(("p", k, torch.from_numpy(np.ascontiguousarray(md_run.point_data[k])).pin_memory()))
    for j in range(p.info.n_cell_sets):
        host_in.append(("c", j, torch.from_numpy(np.ascontiguousarray(md_run.cell_data[j])).pin_memory()))
    host_out = torch.empty(md_run.point_data[0].shape, dtype=torch.float64).pin_memory()
    h2d = sum(t.numel() * t.element_size() for _, _, t in host_in)
    d2h = host_out.numel() * host_out.element_size()
    e2e_steps = max(3, min(args.steps, 10))

    def e2e_step():
        for kind, k, t in host_in:
            fn = F._lib.fot_set_point_data_async if kind == "p" else F._lib.fot_set_cell_data_async
            F._check(fn(p._h, k, F.C.c_void_p(t.data_ptr()), F.C.c_size_t(t.numel() * t.element_size()),
                        F._stream_ptr(stream)))
        plan.run(1, stream)
        F._check(F._lib.fot_get_point_data_async(p._h, 0, F.C.c_void_p(host_out.data_ptr()),
                                                 F.C.c_size_t(d2h), F._stream_ptr(stream)))

    e2e_step()
    p.sync(stream)
    barrier(world)
    torch.cuda.synchronize()
    s2 = torch.cuda.Event(enable_timing=True)
    e2 = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("bench_e2e")
    s2.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e2.record(stream)
    torch.cuda.nvtx.range_pop()
    e2.synchronize()
    p.sync(stream)
    e2e_secs = max_over_ranks(s2.elapsed_time(e2) / 1e3, world)
    e2e_value = ub * e2e_steps * world / e2e_secs / 1e9

    # the reference's sector model for the plan that ran (blocks of 256
    # consecutive cells for the atomic executor, as its global-colour loop
    # counts them; the plan's blocks otherwise): sectors x 32 B x 2 per
    # iteration is its "cache line" bandwidth (problem.hpp:189-192)
    try:
        if chosen.exec == "atomic":
            sectors, _ = p.sector_count(256)
        else:
            sectors, _ = plan.sector_count()
        sector_model = {"sectors_per_iteration": int(sectors), "bytes_per_iteration": int(sectors) * 64,
                        "gbs": int(sectors) * 64 / (secs / args.steps) / 1e9}
    except Exception as e:
        sector_model = {"error": str(e)}
    peak, peak_src = load_peaks()
    # algorithmic bytes per iteration / device time per iteration of this rank
    achieved = ub / (secs / args.steps) / 1e9
    kernel_key = chosen.label().split("/", 1)[1]  # kernel variant: executor, block, layout
    traffic, traffic_src = load_traffic(kernel_key)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(md)
    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        from cuda_fot_b200 import bench_configs as BC
        model = None
        try:
            model = CM.load_default()
        except Exception:
            pass
        jobs = [("res_calc_1000", lambda: BC.res_calc_1000(model, peak, stream)),
                ("lulesh_96", lambda: BC.lulesh_96(peak)),
                ("atomic_spread", lambda: {
                    "mini_aero_128": BC.atomic_spread(md, T.Candidate("rcm", 0, "atomic", 256, aggregate=False,
                                                                      layout="soa")),
                    "res_calc_1000": BC.atomic_spread(mg.res_calc(1000, 1000, 1),
                                                      T.Candidate("rcm", 0, "atomic", 256, aggregate=False,
                                                                  layout="soa"))}),
                ("plan_build", BC.plan_build),
                ("airfoil_1000", lambda: BC.airfoil_1000(peak, stream)),
                ("cost_model", BC.cost_model),
                ("batch_512", BC.batch_512)]
        for key, fn in jobs:
            t_job = time.perf_counter()
            try:
                extras[key] = fn()
            except Exception as e:  # one configuration failing does not lose the others
                extras[key] = {"error": f"{type(e).__name__}: {e}"}
            extras[key]["wall_s"] = round(time.perf_counter() - t_job, 1)

    if rank == 0:
        st = plan.stats()
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs_max / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "faces": md.n_cells, "cells": md.n_points[0],
                       "unique_bytes_per_step": ub, "seed": args.seed,
                       "l2": "inputs larger than L2 (%.2f GB per step vs 126 MB L2)" % (ub / 1e9),
                       "plan": chosen.label(), "plan_choice": choice_src,
                       "point_layout": chosen.layout.upper(),
                       "n_blocks": st["n_blocks"], "block_colours": st["n_colours"],
                       "timed_call": f"Plan.run({args.steps}): {args.steps} iterations in one call",
                       "parallelism": f"replicas x{world}"},
            "atomic_baseline": {"plan": "as-is/atomic-plain/256 (one thread per face, f64 "
                                        "atomics, no aggregation, on the given random numbering)",
                                "value": atomic_plain.get("gbs"), "unit": "GB/s"},
            "speedup_vs_atomic": (value / world) / atomic_plain["gbs"] if atomic_plain.get("ok") else None,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_src,
                         "traffic": traffic, "traffic_unit": "DRAM bytes per iteration",
                         "traffic_source": traffic_src},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "sector_model": sector_model,
            "gpu_launches": launches,
            "clocks": clocks.summary(),
        }
        if sweep_res:
            line["sweep"] = {r["cand"].label(): (round(r["gbs"], 1) if r["ok"] else None) for r in sweep_res}
            best = T.best(sweep_res)
            mine = next((r for r in sweep_res if r["cand"].label() == chosen.label() and r["ok"]), None)
            line["plan_judge"] = {"sweep_best": best["cand"].label(), "sweep_s": round(sweep_s, 1),
                                  "model_pick_s": round(pick_s, 1) if pick_s is not None else None,
                                  "regret": (mine["seconds"] / best["seconds"] - 1.0) if mine else None}
        if sweep_res:
            col = [r for r in sweep_res if r["ok"] and r["cand"].exec != "atomic"]
            if col:
                bc = min(col, key=lambda r: r["seconds"])
                line["coloured"] = {"plan": bc["cand"].label(), "gbs": round(bc["gbs"], 1),
                                    "frac": round(bc["gbs"] / peak, 4),
                                    "speedup_vs_plain_atomics": round(atomic_plain["seconds"] / bc["seconds"], 3)
                                    if atomic_plain.get("ok") else None}
        if choice_note:
            line["plan_note"] = choice_note
        line.update(extras)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
