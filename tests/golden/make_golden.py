"""Generates the golden fixtures in this directory.

Each fixture holds the inputs of a small seeded mesh (cuda_fot_b200.meshgen)
and the outputs of the REFERENCE'S OWN serial loop on them
(``Problem::loopCPUCellCentred<StepSeq>``, problem.hpp:362-380), compiled from
the reference sources by ``make -C oracle ref`` into oracle/_ref/libref.so.
The fixtures pin the oracle (tests/test_oracle.py) and, through it, the GPU
executors; sectors.json holds the reference's own sector model
(countCacheLinesForBlock, problem.hpp:654-672) on the same meshes.  Run from the repository root where the reference sources exist:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cuda_fot_b200 import meshgen as mg  # noqa: E402
from oracle import oracle_py as O  # noqa: E402

ITERS = 3
CASES = [
    # (loop, generator kwargs, layout)
    (mg.RES_CALC, dict(nx=24, ny=20), "aos"),
    (mg.RES_CALC, dict(nx=24, ny=20), "soa"),
    (mg.MINI_AERO, dict(n=7), "aos"),
    (mg.MINI_AERO, dict(n=7), "soa"),
    (mg.LULESH, dict(n=6), "aos"),
    (mg.LULESH, dict(n=6), "soa"),
    (mg.VOLNA, dict(nx=16, ny=12), "aos"),
    (mg.GETACC, dict(nx=16, ny=12), "aos"),
]


def fixture_name(loop, layout):
    return f"{mg.LOOP_NAMES[loop]}_{layout}.npz"


SECTOR_BLOCKS = (32, 256)


def sector_fixtures(here):
    """sectors.json: the reference's own sector model (countCacheLinesForBlock
    over blocks of consecutive cells) on the fixture meshes, both layouts."""
    import json
    out = []
    for loop, kw, layout in CASES:
        if layout != "aos":
            continue
        md = mg.GENERATORS[loop](seed=1, layout=layout, **kw)
        dim = md.point_data[0].shape[1]
        ts = md.point_data[0].dtype.itemsize
        for soa in (False, True):
            for b in SECTOR_BLOCKS:
                out.append({"loop": mg.LOOP_NAMES[loop], "kwargs": kw, "cells_per_block": b,
                            "soa": soa, "dim": dim, "type_size": ts,
                            "sectors": O.ref_sector_count(md.maps[0], b, dim, ts, soa)})
    path = os.path.join(here, "sectors.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(path, len(out), "sector cases")


def main():
    O.build_ref()
    here = os.path.dirname(os.path.abspath(__file__))
    for loop, kw, layout in CASES:
        md = mg.GENERATORS[loop](seed=1, layout=layout, **kw)
        pd, cd, _ = O.ref_serial(md, ITERS)
        arrays = {"loop": np.int32(loop), "n_cells": np.int64(md.n_cells),
                  "n_points": np.array(md.n_points, dtype=np.int64),
                  "iters": np.int32(ITERS), "layout": np.array(layout)}
        for k, m in enumerate(md.maps):
            arrays[f"map{k}"] = m
        for k, d in enumerate(md.point_data):
            arrays[f"point_in{k}"] = d
            arrays[f"point_out{k}"] = pd[k]
        for j, d in enumerate(md.cell_data):
            arrays[f"cell_in{j}"] = d
            arrays[f"cell_out{j}"] = cd[j]
        path = os.path.join(here, fixture_name(loop, layout))
        np.savez_compressed(path, **arrays)
        print(path, md.n_cells, "cells")
    sector_fixtures(here)


if __name__ == "__main__":
    main()
