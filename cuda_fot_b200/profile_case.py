"""A small profiling case: one plan on one seeded mesh, run as separate launches.

    python -m cuda_fot_b200.profile_case --loop mini_aero --n 96 \
        --plan rcm/atomic/256 [--launches 6]

Builds the mesh and the plan, then calls Plan.run(1) `--launches` times, so a
profiler can skip the first launches (-s) and capture one to three (-c) of the
same kernel.  With --airfoil (res_calc only) it runs that many Airfoil
solver iterations around the plan instead (fot_airfoil_run: the cell passes
k_cells, k_bres_calc, k_rms and the plan's res_calc kernel).  Plan labels are those of cuda_fot_b200.tune.Candidate.label():
`order[+partN]/exec[d][-plain]/block[@soa]`, e.g. `gps/hier/128`,
`gps+part256/hierd/256`, `as-is/atomic-plain/256@soa`.  Sizes: res_calc/volna/getacc take --n as the grid edge
(n x n), mini_aero/lulesh as the hex edge (n^3).
"""
from __future__ import annotations

import argparse
import sys

from . import meshgen as mg
from . import tune as T


def parse_plan(label: str) -> T.Candidate:
    layout = "aos"
    if label.endswith("@soa"):
        label, layout = label[: -len("@soa")], "soa"
    order, ex, block = label.split("/")
    part = 0
    if "+part" in order:
        order, p = order.split("+part")
        part = int(p)
    aggregate = True
    if ex.endswith("-plain"):
        aggregate = False
        ex = ex[: -len("-plain")]
    direct = False
    if ex in ("hierd", "hier_launchd"):
        direct = True
        ex = ex[:-1]
    return T.Candidate(None if order == "as-is" else order, part, ex, int(block), direct, aggregate, layout)


def make_mesh(loop: str, n: int, seed: int) -> mg.MeshData:
    if loop == "res_calc":
        return mg.res_calc(n, n, seed)
    if loop == "mini_aero":
        return mg.mini_aero(n, seed, permute=True)
    if loop == "lulesh":
        return mg.lulesh(n, seed, permute=True)
    if loop == "volna":
        return mg.volna(n, n, seed)
    if loop == "getacc":
        return mg.getacc(n, n, seed)
    raise SystemExit(f"unknown loop {loop}")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--loop", default="mini_aero")
    ap.add_argument("--n", type=int, default=96)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--plan", default="rcm/atomic/256")
    ap.add_argument("--launches", type=int, default=6)
    ap.add_argument("--airfoil", action="store_true",
                    help="res_calc only: run `--launches` Airfoil iterations (fot_airfoil_run) "
                         "around the plan instead of bare loop iterations")
    a = ap.parse_args(argv)
    md = make_mesh(a.loop, a.n, a.seed)
    cand = parse_plan(a.plan)
    if a.airfoil:
        if a.loop != "res_calc":
            raise SystemExit("--airfoil needs --loop res_calc")
        from . import bench_configs as BC
        ex = mg.airfoil_extras(md)
        p, plan, af = BC.airfoil_setup(md, ex, cand)
        rms = None
        for _ in range(a.launches):
            rms = af.run(plan, 1)
        print(f"airfoil res_calc n={a.n} cells={md.n_points[0]} edges={md.n_cells} plan={cand.label()} "
              f"iterations={a.launches} rms={rms}")
        return 0
    cache = T.OrderedCache(md)
    p, plan = T.build(cache.get(cand.order, cand.partition, cand.layout), cand)
    for _ in range(a.launches):
        plan.run(1)
    p.sync()
    st = plan.stats()
    print(f"{a.loop} n={a.n} cells={md.n_cells} plan={cand.label()} unique_bytes={md.unique_bytes()} "
          f"blocks={st['n_blocks']} colours={st['n_colours']} smem={st['smem_bytes']} grid={st['grid']}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
