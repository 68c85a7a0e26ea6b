"""Failure detection of the persistent executor, without a GPU fault.

A block's completion flag is zeroed from the host (a flag that nothing will
set again).  The next run's tiles that depend on the block wait for it until
their bounded wait runs out (about 2 s of wall time); the kernel then returns
early with an error status, fot_sync reports FOT_ERR_DEVICE and resets the
plan's queue and flags, and both the CUDA context and the plan stay usable:
a fresh run of the same plan is again bit-identical to the CPU replay.
"""
import time

import pytest

from cuda_fot_b200 import meshgen as mg
from oracle import oracle_py as O
from tests.helpers import bitwise_equal

pytestmark = pytest.mark.gpu


def F():
    from cuda_fot_b200 import fot
    return fot


def test_lost_completion_flag_is_reported_and_recovered():
    md = mg.res_calc(64, 48, 5)
    p = F().Problem.from_mesh(md)
    plan = p.plan(F().EXEC_HIER, 128, F().PLAN_BLOCK_FLAGS)
    ex = plan.export()
    with pytest.raises(F().FotError) as e:
        plan.inject_lost_flag(0)  # nothing has run yet
    assert e.value.code == -3
    plan.run(1)
    p.sync()
    plan.inject_lost_flag(ex["n_blocks"] // 2)
    t0 = time.time()
    plan.run(1)
    with pytest.raises(F().FotError) as e:
        p.sync()
    assert e.value.code == -5, e.value
    assert time.time() - t0 < 60
    # the plan was reset: restore the inputs and run again from scratch
    for k, d in enumerate(md.point_data):
        p.set_point_data(k, d)
    plan.run(2)
    p.sync()
    rep, _ = O.replay_hier(md, ex, 2)
    assert bitwise_equal(p.point_weights(0), rep[0])


def test_other_work_runs_after_a_failed_run():
    md = mg.volna(40, 30, 6)
    p = F().Problem.from_mesh(md)
    plan = p.plan(F().EXEC_HIER, 64, F().PLAN_BLOCK_FLAGS)
    plan.run(1)
    p.sync()
    plan.inject_lost_flag(0)
    plan.run(1)
    with pytest.raises(F().FotError):
        p.sync()
    # an unrelated problem on the same device is unaffected
    md2 = mg.getacc(30, 20, 7)
    p2 = F().Problem.from_mesh(md2)
    plan2 = p2.plan(F().EXEC_HIER, 64)
    ex2 = plan2.export()
    plan2.run(2)
    p2.sync()
    rep, _ = O.replay_hier(md2, ex2, 2)
    assert bitwise_equal(p2.point_weights(0), rep[0])


def test_sync_reports_an_earlier_plans_failure_once():
    """fot_sync checks every plan run since the previous sync, not only the
    last one: a failed hierarchical run followed by an atomic run on the same
    problem is still reported, and the next sync is clean."""
    md = mg.res_calc(64, 48, 9)
    p = F().Problem.from_mesh(md)
    bad = p.plan(F().EXEC_HIER, 128, F().PLAN_BLOCK_FLAGS)
    n_blocks = bad.export()["n_blocks"]
    bad.run(1)
    p.sync()
    bad.inject_lost_flag(n_blocks // 3)
    bad.run(1)
    atomic = p.plan(F().EXEC_ATOMIC, 256)
    atomic.run(1)
    with pytest.raises(F().FotError) as e:
        p.sync()
    assert e.value.code == -5
    p.sync()  # reported once; the plan was reset


def test_flag_injection_needs_a_block_flag_plan():
    """The split write-back kernels wait on no flag: injecting into such a
    plan is refused."""
    p = F().Problem.from_mesh(mg.res_calc(32, 24, 3))
    plan = p.plan(F().EXEC_HIER, 64)
    plan.run(1)
    p.sync()
    with pytest.raises(F().FotError) as e:
        plan.inject_lost_flag(0)
    assert e.value.code == -3
