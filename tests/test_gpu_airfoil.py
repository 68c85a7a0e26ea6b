"""GPU parity of the Airfoil iteration around res_calc (fot_airfoil_run)
against its oracle (orc_airfoil_run):

* with a hierarchical res_calc plan (every kernel form): q, adt and res are
  BIT-IDENTICAL to the oracle replaying the same colour order, the rms
  (a tree sum on the GPU, a cell-order sum on the CPU) within 1e-12;
* with the atomic plan: within 1e-11 normwise of the oracle's serial order;
* maps given in the original numbering follow a reordered problem, also
  when the problem is reordered after the Airfoil step was created;
* bad input and a destroyed problem are refused with an error code;
* the time loop captured as one CUDA graph replays to the same results.
"""
import numpy as np
import pytest

from cuda_fot_b200 import meshgen as mg
from oracle import oracle_py as O
from tests.helpers import bitwise_equal, rel_err

pytestmark = pytest.mark.gpu


def F():
    from cuda_fot_b200 import fot
    return fot


def airfoil(p, ex):
    return F().Airfoil(p, ex["cell_to_node"], ex["bedge_to_node"], ex["bedge_to_cell"],
                       ex["bound"], ex["qinf"], ex["cfl"])


def unpermute_points(arr, perm, layout):
    """Rows (AOS) or columns (SOA) back to the original point numbering;
    perm[orig] = current."""
    return arr[perm] if layout == "aos" else arr[:, perm]


FLAGS = {"split": 0, "split_direct": 4, "pipelined": 16, "simple": 8}


@pytest.mark.parametrize("layout", ["aos", "soa"])
@pytest.mark.parametrize("kernel", list(FLAGS))
def test_coloured_bit_exact_to_replay(layout, kernel):
    md = mg.res_calc(48, 40, 5, layout)
    ex = mg.airfoil_extras(md)
    p = F().Problem.from_mesh(md)
    plan = p.plan(F().EXEC_HIER, 128, FLAGS[kernel])
    exp = plan.export()
    af = airfoil(p, ex)
    rms = af.run(plan, 3)
    p.sync()
    ref, ref_rms = O.airfoil(md, ex, 3, plan=exp)
    for k in (0, 2, 3):
        assert bitwise_equal(p.point_weights(k), ref[k]), f"point set {k}"
    assert abs(rms - ref_rms) <= 1e-12 * ref_rms
    ser, _ = O.airfoil(md, ex, 3)
    assert rel_err(p.point_weights(2), ser[2]) <= 1e-11


def test_coloured_runs_are_reproducible():
    md = mg.res_calc(40, 32, 6)
    ex = mg.airfoil_extras(md)
    outs = []
    for calls in ((4,), (1, 3)):
        p = F().Problem.from_mesh(md)
        plan = p.plan(F().EXEC_HIER, 128)
        af = airfoil(p, ex)
        rms = [af.run(plan, k) for k in calls]
        outs.append((p.point_weights(2), rms[-1]))
    assert bitwise_equal(outs[0][0], outs[1][0])
    assert outs[0][1] == outs[1][1]


@pytest.mark.parametrize("layout", ["aos", "soa"])
def test_atomic_within_tolerance(layout):
    md = mg.res_calc(64, 48, 7, layout)
    ex = mg.airfoil_extras(md)
    p = F().Problem.from_mesh(md)
    plan = p.plan(F().EXEC_ATOMIC, 256, F().PLAN_NO_AGGREGATE)
    rms = af_rms = airfoil(p, ex).run(plan, 5)
    ser, ref_rms = O.airfoil(md, ex, 5)
    assert rel_err(p.point_weights(2), ser[2]) <= 1e-11
    assert rel_err(p.point_weights(3), ser[3]) <= 1e-11
    assert abs(af_rms - ref_rms) <= 1e-9 * ref_rms
    assert rms > 0


@pytest.mark.parametrize("reorder_after", [False, True])
def test_reordered_problem(reorder_after):
    md = mg.res_calc(50, 36, 8)
    ex = mg.airfoil_extras(md)
    p = F().Problem.from_mesh(md)
    if reorder_after:
        af = airfoil(p, ex)
        p.reorder(F().ORDER_RCM)
    else:
        p.reorder(F().ORDER_RCM)
        af = airfoil(p, ex)
    plan = p.plan(F().EXEC_ATOMIC, 256)
    af.run(plan, 3)
    q = unpermute_points(p.point_weights(2), p.point_permutation(0), "aos")
    ser, _ = O.airfoil(md, ex, 3)
    assert rel_err(q, ser[2]) <= 1e-11


def test_rejects_bad_input():
    md = mg.res_calc(10, 8, 1)
    ex = mg.airfoil_extras(md)
    p = F().Problem.from_mesh(md)
    bad = dict(ex)
    bad["cell_to_node"] = ex["cell_to_node"].copy()
    bad["cell_to_node"][3, 2] = md.n_points[1]
    with pytest.raises(F().FotError):
        airfoil(p, bad)
    bad = dict(ex)
    bad["bedge_to_cell"] = ex["bedge_to_cell"].copy()
    bad["bedge_to_cell"][0] = md.n_points[0]
    with pytest.raises(F().FotError):
        airfoil(p, bad)
    other = F().Problem.from_mesh(mg.getacc(8, 8, 1))
    with pytest.raises(F().FotError):
        airfoil(other, ex)


def test_destroyed_problem_is_refused():
    md = mg.res_calc(10, 8, 1)
    ex = mg.airfoil_extras(md)
    p = F().Problem.from_mesh(md)
    plan = p.plan(F().EXEC_ATOMIC, 256)
    af = airfoil(p, ex)
    F()._lib.fot_problem_destroy(p._h)
    p._h = None
    with pytest.raises(F().FotError) as e:
        af.run(plan, 1)
    assert e.value.code == -3  # FOT_ERR_STATE


@pytest.mark.parametrize("exec_", ["hier", "atomic"])
def test_graph_replays_the_time_loop(exec_):
    """The time loop captured as one CUDA graph gives the run's results
    (bit for bit with a coloured plan)."""
    md = mg.res_calc(40, 32, 9)
    ex = mg.airfoil_extras(md)
    out = []
    for use_graph in (False, True):
        p = F().Problem.from_mesh(md)
        plan = (p.plan(F().EXEC_HIER, 128) if exec_ == "hier"
                else p.plan(F().EXEC_ATOMIC, 256, F().PLAN_NO_AGGREGATE))
        af = airfoil(p, ex)
        if use_graph:
            g = af.graph(plan, 3)
            g.launch()
            g.launch()
            rms = af.rms()
        else:
            af.run(plan, 3)
            rms = af.run(plan, 3)
        p.sync()
        out.append((p.point_weights(2), rms))
    if exec_ == "hier":
        assert bitwise_equal(out[0][0], out[1][0])
        assert out[0][1] == out[1][1]
    else:
        assert rel_err(out[1][0], out[0][0]) <= 1e-11
    ref, ref_rms = O.airfoil(md, ex, 6)
    assert rel_err(out[1][0], ref[2]) <= 1e-11
    assert abs(out[1][1] - ref_rms) <= 1e-9 * ref_rms
