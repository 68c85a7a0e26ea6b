"""Edge cases of every executor on the GPU: meshes of one cell, meshes whose
cell count is not a multiple of a warp or a block, blocks larger than the
whole mesh, points no cell touches, and input the engine refuses.
Coloured runs are bit-identical to the CPU replay of their plan, atomic runs
within the usual tolerance of the serial loop."""
import numpy as np
import pytest

from cuda_fot_b200 import meshgen as mg
from oracle import oracle_py as O
from tests.helpers import bitwise_equal, rel_err

pytestmark = pytest.mark.gpu


def F():
    from cuda_fot_b200 import fot
    return fot


TINY = {
    "res_calc_1edge": lambda: mg.res_calc(2, 1, 4),
    "res_calc_58": lambda: mg.res_calc(7, 5, 4),
    "mini_aero_54": lambda: mg.mini_aero(3, 4, permute=True),
    "lulesh_27": lambda: mg.lulesh(3, 4, permute=True),
    "volna_small": lambda: mg.volna(5, 3, 4),
    "getacc_6": lambda: mg.getacc(3, 2, 4),
}

# executor, flags
KINDS = {"atomic": (0, 0), "atomic_plain": (0, 1), "split": (1, 0), "split_direct": (1, 4),
         "pipelined": (1, 16), "simple": (1, 8), "per_colour": (2, 0)}


def tol(md):
    return 1e-5 if md.loop == mg.VOLNA else 1e-12


@pytest.mark.parametrize("block", [64, 512])
@pytest.mark.parametrize("kind", list(KINDS))
@pytest.mark.parametrize("name", list(TINY))
def test_tiny_and_ragged_meshes(name, kind, block):
    md = TINY[name]()
    p = F().Problem.from_mesh(md)
    exec_, flags = KINDS[kind]
    if exec_ == 0:
        plan = p.plan(exec_, 256, flags)
        plan.run(3)
        p.sync()
        assert rel_err(p.point_weights(0), O.serial(md, 3)[0][0]) <= tol(md)
        return
    plan = p.plan(exec_, block, flags)
    ex = plan.export()
    rc, msg = O.check_plan(ex, md.maps[0], md.n_points[0], block)
    assert rc == 0, msg
    plan.run(3)
    p.sync()
    rep, _ = O.replay_hier(md, ex, 3)
    assert bitwise_equal(p.point_weights(0), rep[0])


@pytest.mark.parametrize("kind", ["atomic", "split", "split_direct"])
def test_untouched_points_keep_their_values(kind):
    md = mg.getacc(12, 9, 5)
    extra = 7
    d0 = md.point_data[0]
    tail = np.random.default_rng(2).standard_normal((extra, d0.shape[1]))
    md.point_data[0] = np.concatenate([d0, tail])
    md.n_points = [md.n_points[0] + extra] + md.n_points[1:]
    p = F().Problem.from_mesh(md)
    exec_, flags = KINDS[kind]
    plan = p.plan(exec_, 128 if exec_ else 256, flags)
    plan.run(2)
    p.sync()
    out = p.point_weights(0)
    assert bitwise_equal(out[-extra:], tail)
    assert rel_err(out, O.serial(md, 2)[0][0]) <= 1e-12


def test_refused_input():
    md = mg.res_calc(6, 4, 1)
    maps = [m.copy() for m in md.maps]
    with pytest.raises(F().FotError):  # no cells
        F().Problem(md.loop, 0, md.n_points, [m[:0] for m in maps])
    bad = [m.copy() for m in maps]
    bad[1][3, 1] = md.n_points[1]
    with pytest.raises(F().FotError):  # mapping entry out of range
        F().Problem(md.loop, md.n_cells, md.n_points, bad)
    bad = [m.copy() for m in maps]
    bad[2][0, 0] = (bad[2][0, 0] + 1) % md.n_points[2]
    with pytest.raises(F().FotError):  # q's mapping differs from mapping 0
        F().Problem(md.loop, md.n_cells, md.n_points, bad)
    p = F().Problem.from_mesh(md)
    with pytest.raises(F().FotError):  # wrong dataset size
        p.set_point_data(0, np.zeros((3, 4)))


@pytest.mark.parametrize("name", ["res_calc_58", "lulesh_27", "mini_aero_54"])
@pytest.mark.parametrize("block", [1, 1024])
def test_block_size_limits(name, block):
    """The smallest (one cell per block) and largest block sizes run and
    replay bit for bit; sizes outside [1, 1024] are refused."""
    md = TINY[name]()
    p = F().Problem.from_mesh(md)
    plan = p.plan(F().EXEC_HIER, block, 0)
    ex = plan.export()
    plan.run(2)
    p.sync()
    rep, _ = O.replay_hier(md, ex, 2)
    assert bitwise_equal(p.point_weights(0), rep[0])
    for bad in (0, 1025):
        with pytest.raises(F().FotError) as e:
            p.plan(F().EXEC_HIER, bad, 0)
        assert e.value.code == -1  # FOT_ERR_ARG


@pytest.mark.parametrize("exec_", [0, 1])
def test_stale_graph_is_refused(exec_):
    """A captured graph replays the buffers it was captured with: after the
    problem is renumbered its launch is refused, not replayed."""
    md = mg.res_calc(10, 8, 1)
    p = F().Problem.from_mesh(md)
    plan = p.plan(exec_, 256 if exec_ == 0 else 64, 0)
    g = plan.graph(2)
    g.launch()
    p.sync()
    p.reorder(F().ORDER_RCM)
    with pytest.raises(F().FotError) as e:
        g.launch()
    assert e.value.code == -3  # FOT_ERR_STATE
    del g
