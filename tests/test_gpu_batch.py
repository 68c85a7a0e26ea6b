"""GPU parity of the batched executors (fot_batch): many meshes of uneven
size in ONE launch.

Hierarchical plans: each mesh's tiles run in its own plan's colour order,
with the thread-colour accumulation of the hierarchical executor, so every
mesh's result is BIT-IDENTICAL to the oracle's CPU replay of its own plan,
and within 1e-12 (FP64) / 1e-5 (FP32 volna) of the serial loop; a CUDA graph
of batched launches equals the same launches issued directly.  Atomic plans:
every mesh within the same tolerances of its serial loop.
"""
import pytest

from cuda_fot_b200 import meshgen as mg
from oracle import oracle_py as O
from tests.helpers import bitwise_equal, rel_err

pytestmark = pytest.mark.gpu


def F():
    from cuda_fot_b200 import fot
    return fot


def tol(loop):
    return 1e-5 if loop == mg.VOLNA else 1e-12


def mixed_meshes():
    """res_calc and volna meshes of very different sizes (4 to 3,000 cells)."""
    out = []
    for i, (a, b) in enumerate([(8, 6), (40, 30), (17, 9), (64, 48), (2, 2), (30, 70)]):
        out.append(mg.res_calc(a, b, 10 + i))
        out.append(mg.volna(a + 3, b + 1, 20 + i))
    return out


def single_kind(loop):
    if loop == mg.MINI_AERO:
        return [mg.mini_aero(n, 30 + n) for n in (4, 9, 6)]
    if loop == mg.LULESH:
        return [mg.lulesh(n, 40 + n) for n in (3, 10, 6)]
    if loop == mg.GETACC:
        return [mg.getacc(a, b, 50 + a) for a, b in ((5, 4), (33, 21), (12, 40))]
    if loop == mg.VOLNA:
        return [mg.volna(a, b, 60 + a) for a, b in ((5, 4), (33, 21), (12, 40))]
    return [mg.res_calc(a, b, 70 + a) for a, b in ((5, 4), (33, 21), (12, 40))]


def run_and_check(mds, block, iters_split=(2, 1)):
    probs = [F().Problem.from_mesh(md) for md in mds]
    plans = [p.plan(F().EXEC_HIER, block) for p in probs]
    exs = [pl.export() for pl in plans]
    b = F().Batch(plans)
    for k in iters_split:
        b.run(k)
    b.sync()
    iters = sum(iters_split)
    for md, p, ex in zip(mds, probs, exs):
        rep, _ = O.replay_hier(md, ex, iters)
        assert bitwise_equal(p.point_weights(0), rep[0]), (mg.LOOP_NAMES[md.loop], md.n_cells)
        ser, _ = O.serial(md, iters)
        assert rel_err(p.point_weights(0), ser[0]) <= tol(md.loop)
    return probs


@pytest.mark.parametrize("block", [64, 128, 256])
def test_mixed_res_calc_volna_batch_matches_replay(block):
    run_and_check(mixed_meshes(), block)


@pytest.mark.parametrize("loop", range(5))
def test_single_kind_batch_matches_replay(loop):
    run_and_check(single_kind(loop), 128)


def test_batch_graph_equals_direct_launches():
    import torch
    mds = mixed_meshes()[:6]
    direct = [F().Problem.from_mesh(md) for md in mds]
    b1 = F().Batch([p.plan(F().EXEC_HIER, 128) for p in direct])
    for _ in range(4):
        b1.run(1)
    b1.sync()
    graphed = [F().Problem.from_mesh(md) for md in mds]
    b2 = F().Batch([p.plan(F().EXEC_HIER, 128) for p in graphed])
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b2.run(1, s)
        b2.run(1, s)
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    b2.sync()
    for p1, p2 in zip(direct, graphed):
        assert bitwise_equal(p1.point_weights(0), p2.point_weights(0))
    del g


@pytest.mark.parametrize("aggregate", [True, False])
def test_atomic_batch_matches_serial(aggregate):
    """Atomic plans of many meshes in one launch: each mesh within the
    atomic tolerance of its serial loop (summation order is not fixed)."""
    mds = mixed_meshes()
    probs = [F().Problem.from_mesh(md) for md in mds]
    flags = 0 if aggregate else F().PLAN_NO_AGGREGATE
    b = F().Batch([p.plan(F().EXEC_ATOMIC, 256, flags) for p in probs])
    b.run(2)
    b.run(1)
    b.sync()
    for md, p in zip(mds, probs):
        ser, _ = O.serial(md, 3)
        assert rel_err(p.point_weights(0), ser[0]) <= tol(md.loop), (mg.LOOP_NAMES[md.loop], md.n_cells)


@pytest.mark.parametrize("loop", [mg.MINI_AERO, mg.LULESH, mg.GETACC])
def test_single_kind_atomic_batch_matches_serial(loop):
    mds = single_kind(loop)
    probs = [F().Problem.from_mesh(md) for md in mds]
    b = F().Batch([p.plan(F().EXEC_ATOMIC, 256) for p in probs])
    b.run(3)
    b.sync()
    for md, p in zip(mds, probs):
        ser, ser_cd = O.serial(md, 3)
        assert rel_err(p.point_weights(0), ser[0]) <= tol(md.loop)
        for j, ref in enumerate(ser_cd):  # lulesh's element volumes (contracted FMA)
            assert rel_err(p.cell_weights(j), ref) <= tol(md.loop)


def test_batch_rejects_mixed_executors_and_kinds():
    md1, md2 = mg.res_calc(6, 5, 1), mg.lulesh(3, 2)
    p1, p2 = F().Problem.from_mesh(md1), F().Problem.from_mesh(md2)
    p3 = F().Problem.from_mesh(mg.res_calc(7, 5, 3))
    with pytest.raises(F().FotError):
        F().Batch([p1.plan(F().EXEC_ATOMIC, 256), p3.plan(F().EXEC_HIER, 64)])
    with pytest.raises(F().FotError):
        F().Batch([p1.plan(F().EXEC_HIER, 64), p2.plan(F().EXEC_HIER, 64)])
