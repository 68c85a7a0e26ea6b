"""Autotuner: candidate plans and their measured timings.

A candidate is (ordering, partition size, executor, block size, layout):

* ordering  -- None (keep the numbering), "natural" (cells sorted by point
  tuple), "random", "rcm" or "gps" (fot_reorder);
* partition -- 0, or the part size of fot_partition followed by
  fot_reorder_to_partition and fot_renumber_points (the reference's
  partition -> reorderToPartition -> renumberPoints sequence);
* executor  -- "atomic", "hier" (persistent; split write-back kernel,
  staged or -- with direct -- gathering rows straight from HBM/L2) or
  "hier_launch";
* block     -- cells per block (hierarchical) / threads per CTA (atomic);
* layout    -- "aos" or "soa" point data (the reference's Problem<SOA>).

``measure(md, cand)`` builds the candidate on a fresh problem and times
``iters`` iterations with CUDA events on the launching stream after warm-up.
The exhaustive sweep over a candidate list is the fallback and the yardstick of
the learned cost model (cuda_fot_b200/costmodel.py), and it produces that
model's training data.
"""
from __future__ import annotations

import time
from dataclasses import dataclass
from typing import Dict, List, Optional

from . import fot as F
from . import meshgen as mg

ORDERS = {None: None, "natural": F.ORDER_NATURAL, "random": F.ORDER_RANDOM,
          "rcm": F.ORDER_RCM, "gps": F.ORDER_GPS}
EXECS = {"atomic": F.EXEC_ATOMIC, "hier": F.EXEC_HIER, "hier_launch": F.EXEC_HIER_LAUNCH}


@dataclass(frozen=True)
class Candidate:
    order: Optional[str] = None
    partition: int = 0
    exec: str = "hier"
    block: int = 256
    direct: bool = False  # hierarchical: gather read rows from HBM/L2 (no staging)
    aggregate: bool = True  # atomic: warp aggregation of same-target lanes
    layout: str = "aos"     # point-data layout of the problem the plan runs on

    def label(self) -> str:
        o = self.order or "as-is"
        p = f"+part{self.partition}" if self.partition else ""
        d = "d" if self.direct and self.exec != "atomic" else ""
        a = "-plain" if self.exec == "atomic" and not self.aggregate else ""
        lay = "@soa" if self.layout == "soa" else ""
        return f"{o}{p}/{self.exec}{d}{a}/{self.block}{lay}"


def plan_candidates(order: Optional[str], part: int) -> List[Candidate]:
    """The plans of one (ordering, partition): for both point layouts, the
    atomic executor with and without warp aggregation and the hierarchical
    executor's staged and direct split write-back kernels (blocks of 128, 256,
    512 and 128, 256 cells; on a partition, blocks of the part size)."""
    out = []
    for lay in ("aos", "soa"):
        out.append(Candidate(order, part, "atomic", 256, layout=lay))
        out.append(Candidate(order, part, "atomic", 256, aggregate=False, layout=lay))
        if part:
            out.append(Candidate(order, part, "hier", part, layout=lay))
            out.append(Candidate(order, part, "hier", part, True, layout=lay))
            continue
        for b in (128, 256, 512):
            out.append(Candidate(order, 0, "hier", b, layout=lay))
        for b in (128, 256):
            out.append(Candidate(order, 0, "hier", b, True, layout=lay))
    return out


def default_candidates(loop: int, quick: bool = False) -> List[Candidate]:
    """The sweep: plan_candidates over the orderings (quick: RCM and GPS, and
    RCM with parts of 256 cells; else also the given numbering, a random one
    and GPS with parts of 128, 256 and 512)."""
    orderings = [("gps", 0), ("rcm", 0), ("rcm", 256)] if quick else \
        [(None, 0), ("random", 0), ("rcm", 0), ("gps", 0), ("gps", 128), ("gps", 256),
         ("rcm", 256), ("gps", 512)]
    out = []
    for o, part in orderings:
        out.extend(plan_candidates(o, part))
    return out


class OrderedCache:
    """Host copies of a mesh after each ordering / partition, so that every
    plan candidate starts from the same cell order."""

    def __init__(self, md: mg.MeshData):
        self.md = md
        self._cache: Dict = {}

    def drop(self, order: Optional[str], partition: int) -> None:
        """Forget the host copies of one ordering (both layouts)."""
        for k in [k for k in self._cache if k[0] == order and k[1] == partition]:
            del self._cache[k]

    def get(self, order: Optional[str], partition: int, layout: Optional[str] = None) -> mg.MeshData:
        if layout is not None and layout != self.md.layout:
            key = (order, partition, layout)
            if key not in self._cache:
                self._cache[key] = self.get(order, partition).to_layout(layout)
            return self._cache[key]
        key = (order, partition)
        if key not in self._cache:
            p = F.Problem.from_mesh(self.md)
            t0 = time.perf_counter()
            if order is not None:
                p.reorder(ORDERS[order], seed=1)
            if partition:
                p.partition(partition)
                p.reorder_to_partition()
                p.renumber_points()
            t_order = time.perf_counter() - t0
            md2 = p.mesh_data()
            md2.meta = dict(self.md.meta, order=order, partition=partition, order_s=t_order)
            if partition:
                md2.meta["partition_vector"] = p.partition_vector()
            self._cache[key] = md2
        return self._cache[key]


def build(md: mg.MeshData, cand: Candidate, stream=None):
    """A problem holding md (already ordered; converted to the candidate's
    point layout on the GPU when it is not in it) and the candidate's plan."""
    p = F.Problem.from_mesh(md)
    if md.layout != cand.layout:
        p.set_layout(cand.layout)
    flags = 0
    if cand.partition:
        p.set_partition(md.meta["partition_vector"])
        flags |= F.PLAN_USE_PARTITION
    if cand.direct:
        flags |= F.PLAN_DIRECT_READS
    if cand.exec == "atomic" and not cand.aggregate:
        flags |= F.PLAN_NO_AGGREGATE
    plan = p.plan(EXECS[cand.exec], cand.block, flags)
    return p, plan


def time_plan(p, plan, iters: int = 10, warmup: int = 3, stream=None) -> float:
    """Seconds per iteration (CUDA events on the launching stream)."""
    import torch
    st = stream or torch.cuda.current_stream()
    plan.run(warmup, st)
    p.sync(st)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(st)
    plan.run(iters, st)
    end.record(st)
    end.synchronize()
    p.sync(st)
    return start.elapsed_time(end) / 1e3 / iters


def measure(cache: OrderedCache, cand: Candidate, iters: int = 10, warmup: int = 3) -> dict:
    md = cache.get(cand.order, cand.partition)
    try:
        t0 = time.perf_counter()
        p, plan = build(md, cand)
        t_plan = time.perf_counter() - t0
        secs = time_plan(p, plan, iters, warmup)
        st = plan.stats()
        ok = True
    except F.FotError as e:
        return {"cand": cand, "ok": False, "error": str(e)}
    ub = cache.md.unique_bytes()
    return {"cand": cand, "ok": ok, "seconds": secs, "gbs": ub / secs / 1e9,
            "plan_s": t_plan, "order_s": md.meta.get("order_s", 0.0), "stats": st}


def sweep(md: mg.MeshData, cands: List[Candidate], iters: int = 10, warmup: int = 3,
          verbose: bool = False, cache: Optional[OrderedCache] = None) -> List[dict]:
    """Measure every candidate, one (ordering, partition) at a time; the
    host copies of an ordering are dropped once its candidates are measured
    (the given cache keeps the unordered mesh only)."""
    cache = cache or OrderedCache(md)
    out = [None] * len(cands)
    groups: Dict = {}
    for i, c in enumerate(cands):
        groups.setdefault((c.order, c.partition), []).append(i)
    for key, idx in groups.items():
        for i in idx:
            out[i] = measure(cache, cands[i], iters, warmup)
        cache.drop(*key)
    for c, r in zip(cands, out):
        if verbose:
            if r["ok"]:
                print(f"  {c.label():28s} {r['seconds']*1e6:9.1f} us  {r['gbs']:8.1f} GB/s", flush=True)
            else:
                print(f"  {c.label():28s} failed: {r['error']}", flush=True)
    return out


def best(results: List[dict]) -> dict:
    ok = [r for r in results if r["ok"]]
    return min(ok, key=lambda r: r["seconds"])
