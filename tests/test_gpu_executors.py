"""GPU parity of the two executors, through the C ABI (libfot.so).

* atomic executor vs the oracle's serial loop: <= 1e-12 normwise relative
  error for the FP64 loops, <= 1e-5 for the FP32 volna loop (the summation
  order of atomics is not fixed, and its units contract multiply-adds), for
  the incremented dataset and for cell data the functor writes;
* hierarchical executors: the exported plan passes the oracle's exact checks
  and the GPU result is BIT-IDENTICAL to the oracle's CPU replay of the same
  colour order, and within the same tolerances of the serial loop;
* golden fixtures (outputs of the reference's own serial loop);
* the benchmark-size meshes (res_calc 1000x1000, mini_aero 128^3 and LULESH
  96^3 with random numbering) against the serial loop.
"""
import numpy as np
import pytest

from cuda_fot_b200 import meshgen as mg
from oracle import oracle_py as O
from tests.helpers import bitwise_equal, golden_names, load_golden, rel_err

pytestmark = pytest.mark.gpu


def F():
    from cuda_fot_b200 import fot
    return fot


def tol(loop):
    return 1e-5 if loop == mg.VOLNA else 1e-12


def medium(loop, layout="aos", seed=3):
    if loop == mg.RES_CALC:
        return mg.res_calc(64, 48, seed, layout)
    if loop == mg.MINI_AERO:
        return mg.mini_aero(14, seed, layout)
    if loop == mg.LULESH:
        return mg.lulesh(12, seed, layout)
    if loop == mg.VOLNA:
        return mg.volna(40, 30, seed, layout)
    return mg.getacc(40, 30, seed, layout)


def unpermute_cells(arr, cell_id):
    out = np.empty_like(arr)
    out[:, cell_id] = arr
    return out


@pytest.mark.parametrize("layout", ["aos", "soa"])
@pytest.mark.parametrize("loop", range(5))
@pytest.mark.parametrize("aggregate", [True, False])
def test_atomic_matches_serial(loop, layout, aggregate):
    md = medium(loop, layout)
    p = F().Problem.from_mesh(md)
    p.loop_gpu_cell_centred(3, aggregate=aggregate)
    ser, ser_cd = O.serial(md, 3)
    assert rel_err(p.point_weights(0), ser[0]) <= tol(loop)
    # cell data the functor writes (lulesh's element volumes): the atomic
    # executor is compiled with multiply-add contraction, so within tolerance
    for j, ref in enumerate(ser_cd):
        assert rel_err(p.cell_weights(j), ref) <= tol(loop)


KERNELS = {  # executor, plan flags
    "split": (1, 0), "split_direct": (1, 4), "pipelined": (1, 16), "simple": (1, 8),
    "simple_direct": (1, 12), "per_colour": (2, 0),
}


@pytest.mark.parametrize("layout", ["aos", "soa"])
@pytest.mark.parametrize("loop", range(5))
@pytest.mark.parametrize("block", [32, 128, 256])
@pytest.mark.parametrize("kernel", list(KERNELS))
def test_hierarchical_bit_exact_replay(loop, layout, block, kernel):
    md = medium(loop, layout)
    p = F().Problem.from_mesh(md)
    exec_, flags = KERNELS[kernel]
    plan = p.plan(exec_, block, flags)
    ex = plan.export()
    rc, msg = O.check_plan(ex, md.maps[0], md.n_points[0], block)
    assert rc == 0, msg
    # the problem's cells now follow plan order
    assert np.array_equal(p.mapping(0), md.maps[0][ex["cell_id"]])
    assert np.array_equal(p.cell_order(), ex["cell_id"])
    plan.run(3)
    p.sync()
    rep, rep_cd = O.replay_hier(md, ex, 3)
    assert bitwise_equal(p.point_weights(0), rep[0])
    for j, ref in enumerate(rep_cd):
        assert bitwise_equal(unpermute_cells(p.cell_weights(j), ex["cell_id"]), ref)
    ser, _ = O.serial(md, 3)
    assert rel_err(p.point_weights(0), ser[0]) <= tol(loop)


@pytest.mark.parametrize("name", golden_names())
def test_golden_fixtures_on_gpu(name):
    md, out_pd, out_cd, iters = load_golden(name)
    for exec_ in (F().EXEC_ATOMIC, F().EXEC_HIER):
        p = F().Problem.from_mesh(md)
        plan = p.plan(exec_, 64)
        plan.run(iters)
        p.sync()
        assert rel_err(p.point_weights(0), out_pd[0]) <= tol(md.loop), (name, exec_)
        order = p.cell_order()
        for j, ref in enumerate(out_cd):
            got = unpermute_cells(p.cell_weights(j), order)
            if exec_ == F().EXEC_ATOMIC:  # contracted multiply-adds
                assert rel_err(got, ref) <= tol(md.loop), (name, j)
            else:
                assert bitwise_equal(got, ref), (name, j)


def test_repeated_runs_are_deterministic_and_graph_equals_run():
    md = medium(mg.RES_CALC)
    p1 = F().Problem.from_mesh(md)
    plan1 = p1.plan(F().EXEC_HIER, 128)
    plan1.run(2)
    plan1.run(3)
    p1.sync()
    p2 = F().Problem.from_mesh(md)
    plan2 = p2.plan(F().EXEC_HIER, 128)
    g = plan2.graph(5)
    g.launch()
    p2.sync()
    assert bitwise_equal(p1.point_weights(0), p2.point_weights(0))


def test_stale_plan_is_rejected():
    md = medium(mg.RES_CALC)
    p = F().Problem.from_mesh(md)
    old = p.plan(F().EXEC_HIER, 64)
    p.plan(F().EXEC_HIER, 128)  # reorders the cells again
    with pytest.raises(F().FotError) as e:
        old.run(1)
    assert e.value.code == -3


def test_bad_mapping_is_rejected():
    md = mg.small(mg.MINI_AERO)
    maps = [m.copy() for m in md.maps]
    maps[1][0, 0] = (maps[1][0, 0] + 1) % md.n_points[1]
    with pytest.raises(F().FotError):
        F().Problem(md.loop, md.n_cells, md.n_points, maps)
    maps = [m.copy() for m in md.maps]
    maps[0][3, 1] = md.n_points[0]
    with pytest.raises(F().FotError):
        F().Problem(md.loop, md.n_cells, md.n_points, maps)


@pytest.mark.parametrize("loop,gen", [
    (mg.RES_CALC, lambda: mg.res_calc(1000, 1000)),
    (mg.LULESH, lambda: mg.lulesh(96)),
    (mg.MINI_AERO, lambda: mg.mini_aero(128)),
])
def test_benchmark_sizes_against_serial(loop, gen):
    md = gen()
    ser, _ = O.serial(md, 1)
    pa = F().Problem.from_mesh(md)
    pa.loop_gpu_cell_centred(1)
    assert rel_err(pa.point_weights(0), ser[0]) <= 1e-12
    ph = F().Problem.from_mesh(md)
    ph.loop_gpu_hierarchical(1, 256)
    assert rel_err(ph.point_weights(0), ser[0]) <= 1e-12


@pytest.mark.parametrize("loop", range(5))
@pytest.mark.parametrize("layout", ["aos", "soa"])
@pytest.mark.parametrize("direct", [False, True])
def test_split_writeback_repeated_launches_match_replay(loop, layout, direct):
    """The split write-back kernels run one launch per iteration, each
    combining the previous iteration's shared points, and a flush launch at
    the end of a call: one call of 4 iterations (chained launches) and 4 calls
    of 1 iteration both equal the CPU replay of 4 iterations, and the plan has
    points shared by several blocks to exercise the combine."""
    md = medium(loop, layout)
    outs = []
    for calls in ((4,), (1, 1, 1, 1)):
        p = F().Problem.from_mesh(md)
        plan = p.plan(F().EXEC_HIER, 64, F().PLAN_DIRECT_READS if direct else 0)
        st = plan.stats()
        assert st["kernel"] == ("split write-back, direct" if direct else "split write-back")
        assert st["shared_points"] > 0 and st["partial_slots"] > st["shared_points"]
        ex = plan.export()
        for k in calls:
            plan.run(k)
        p.sync()
        outs.append(p.point_weights(0))
    rep, _ = O.replay_hier(md, ex, 4)
    assert bitwise_equal(outs[0], rep[0])
    assert bitwise_equal(outs[1], rep[0])
