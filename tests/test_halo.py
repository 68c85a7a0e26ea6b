"""CPU tests of the partitioned (multi-GPU) path's host side
(cuda_fot_b200/halo.py): the split of a mesh into rank-local meshes, and the
halo exchange over torch.distributed with gloo ranks on the CPU, each rank's
loop run by the oracle.  The owners' assembled rows equal the serial loop
over the whole mesh (to rounding: the halo sums add in another order)."""
import os
import socket

import numpy as np
import pytest

from cuda_fot_b200 import halo as H
from cuda_fot_b200 import meshgen as mg
from oracle import oracle_py as O
from tests.helpers import rel_err

MESHES = {"res_calc": lambda: mg.res_calc(30, 20, 1), "mini_aero": lambda: mg.mini_aero(6, 1, permute=True),
          "lulesh": lambda: mg.lulesh(5, 1, permute=True), "volna": lambda: mg.volna(12, 10, 1),
          "getacc": lambda: mg.getacc(12, 10, 1)}


def tol(md):
    return 1e-5 if md.loop == mg.VOLNA else 1e-12


def parts(md, n_ranks, kind):
    if kind == "blocks":
        return np.arange(md.n_cells) * n_ranks // md.n_cells
    return np.random.default_rng(3).integers(0, n_ranks, md.n_cells)


@pytest.mark.parametrize("kind", ["blocks", "random"])
@pytest.mark.parametrize("n_ranks", [1, 2, 4])
def test_split_is_consistent(n_ranks, kind):
    md = mg.res_calc(24, 18, 2)
    part = parts(md, n_ranks, kind)
    lms = H.split_mesh(md, part, n_ranks)
    # every cell in exactly one part, local maps resolve to the global points
    assert sorted(np.concatenate([lm.cells for lm in lms]).tolist()) == list(range(md.n_cells))
    owners = np.zeros(md.n_points[0], dtype=int)
    for lm in lms:
        for k, m in enumerate(md.maps):
            assert np.array_equal(lm.points[k][lm.md.maps[k]], m[lm.cells])
        owners[lm.points[0][lm.owned]] += 1
        halo = ~lm.owned
        assert not np.any(lm.md.point_data[0][halo])
        assert np.array_equal(lm.md.point_data[0][lm.owned], md.point_data[0][lm.points[0][lm.owned]])
        for o, rows in lm.send.items():
            assert o < lm.rank  # the owner is the lowest rank touching the point
            assert np.array_equal(lms[o].points[0][lms[o].recv[lm.rank]], lm.points[0][rows])
            assert lms[o].owned[lms[o].recv[lm.rank]].all()
    touched = np.unique(md.maps[0])
    assert np.array_equal(owners[touched], np.ones(len(touched)))


@pytest.mark.parametrize("layout", ["aos", "soa"])
@pytest.mark.parametrize("loop", list(MESHES))
def test_assembled_parts_equal_the_whole(loop, layout):
    md = MESHES[loop]().to_layout(layout)
    lms = H.split_mesh(md, parts(md, 3, "random"), 3)
    outs = [O.serial(lm.md, 2)[0][0] for lm in lms]
    for o in range(3):
        for s in range(3):
            if o in lms[s].send:
                src = H._rows(outs[s], lms[s].send[o], layout)
                if layout == "aos":
                    outs[o][lms[o].recv[s]] += src
                else:
                    outs[o][:, lms[o].recv[s]] += src
    ser = O.serial(md, 2)[0][0]
    assert rel_err(H.assemble(md, lms, outs), ser) <= tol(md)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, loop, layout, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        md = MESHES[loop]().to_layout(layout)
        lms = H.split_mesh(md, parts(md, world, "random"), world)
        lm = lms[rank]
        out = O.serial(lm.md, 2)[0][0]
        dt = torch.from_numpy(out).dtype

        def gather(o):
            # packed rows are AOS (row-major), whatever the dataset layout
            rows = H._rows(out, lm.send[o], layout)
            return torch.from_numpy(np.ascontiguousarray(rows if layout == "aos" else rows.T).ravel())

        def scatter_add(s, t):
            rows = t.numpy().reshape(len(lm.recv[s]), -1) if layout == "aos" else \
                t.numpy().reshape(len(lm.recv[s]), -1).T
            if layout == "aos":
                out[lm.recv[s]] += rows
            else:
                out[:, lm.recv[s]] += rows

        H.exchange(lm, gather, scatter_add, lambda n: torch.empty(n, dtype=dt))
        got = [None] * world
        dist.all_gather_object(got, out)
        if rank == 0:
            ser = O.serial(md, 2)[0][0]
            q.put(float(rel_err(H.assemble(md, lms, got), ser)) <= tol(md))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("loop,layout,world", [("res_calc", "aos", 2), ("mini_aero", "soa", 3),
                                                ("volna", "aos", 2), ("getacc", "soa", 2)])
def test_gloo_ranks_exchange_halo(loop, layout, world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, loop, layout, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=10) is True
