"""CPU tests of the oracle: pinned bit-exactly to the golden fixtures made by
the reference's own compiled serial loop, the reference's Catch KATs for the
point graph, and the coloured-plan replay and plan checks (with mistakes
planted in CPU-side plans)."""
import numpy as np
import pytest

from cuda_fot_b200 import meshgen as mg
from oracle import oracle_py as O
from tests.helpers import (bitwise_equal, golden_names, load_golden, py_plan,
                           rel_err)


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference_serial_loop_bit_exact(name):
    md, out_pd, out_cd, iters = load_golden(name)
    pd, cd = O.serial(md, iters)
    for k, (a, b) in enumerate(zip(pd, out_pd)):
        assert bitwise_equal(a, b), f"{name}: point data {k} differs"
    for j, (a, b) in enumerate(zip(cd, out_cd)):
        assert bitwise_equal(a, b), f"{name}: cell data {j} differs"


@pytest.mark.parametrize("name", golden_names())
def test_golden_outputs_are_nontrivial(name):
    md, out_pd, _, _ = load_golden(name)
    assert np.abs(out_pd[0]).max() > 0
    assert not np.array_equal(out_pd[0], md.point_data[0])


def test_point_graph_reorder_inverse_kat():
    """catch_heuristical_partition.cu:33-51: the point graph of the 4-edge
    mesh "0 1, 0 2, 1 2, 2 3", renumbered by the inverse permutation
    {3, 1, 0, 2}, has adjacency {{3}, {2, 3}, {1, 3}, {0, 1, 2}}."""
    mapping = np.array([[0, 1], [0, 2], [1, 2], [2, 3]], dtype=np.uint32)
    ind, ends = O.point_graph(4, mapping)
    assert np.all(np.diff(ind.astype(np.int64)) >= 0)  # sanity check (:20-31)
    adj = [set(ends[ind[i]:ind[i + 1]].tolist()) for i in range(4)]
    inv = [3, 1, 0, 2]
    perm = np.argsort(inv)
    got = [sorted(perm[list(adj[inv[i]])].tolist()) for i in range(4)]
    assert got == [[3], [2, 3], [1, 3], [0, 1, 2]]


def test_bandwidth_profile_natural_vs_random():
    md = mg.res_calc(30, 30)
    bw_nat, prof_nat = O.bandwidth_profile(md.n_points[0], md.maps[0])
    perm = mg.rng(5).permutation(md.n_points[0])
    bw_rnd, prof_rnd = O.bandwidth_profile(md.n_points[0], perm[md.maps[0]])
    assert bw_nat <= 31 and bw_rnd > 10 * bw_nat and prof_rnd > 10 * prof_nat


@pytest.mark.parametrize("loop", range(5))
@pytest.mark.parametrize("layout", ["aos", "soa"])
def test_replay_of_python_plan_matches_serial(loop, layout):
    md = mg.small(loop, layout=layout)
    plan = py_plan(md, 32)
    rc, msg = O.check_plan(plan, md.maps[0], md.n_points[0], 32)
    assert rc == 0, msg
    ser, ser_cd = O.serial(md, 2)
    rep, rep_cd = O.replay_hier(md, plan, 2)
    tol = 1e-5 if loop == mg.VOLNA else 1e-12
    assert rel_err(rep[0], ser[0]) <= tol
    for a, b in zip(rep_cd, ser_cd):
        assert bitwise_equal(a, b)  # direct outputs do not depend on order


def test_replay_is_deterministic_and_order_sensitive():
    md = mg.small(mg.RES_CALC)
    plan = py_plan(md, 16)
    a, _ = O.replay_hier(md, plan, 3)
    b, _ = O.replay_hier(md, plan, 3)
    assert bitwise_equal(a[0], b[0])


def _planted(plan, **changes):
    p = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in plan.items()}
    p.update(changes)
    return p


def test_check_plan_catches_planted_mistakes():
    md = mg.small(mg.RES_CALC)
    plan = py_plan(md, 32)
    n0 = md.n_points[0]
    assert O.check_plan(plan, md.maps[0], n0, 32)[0] == 0
    # 1: positions not a permutation
    cid = plan["cell_id"].copy()
    cid[1] = cid[0]
    assert O.check_plan(_planted(plan, cell_id=cid), md.maps[0], n0, 32)[0] == 1
    # 3: block larger than the block size
    assert O.check_plan(plan, md.maps[0], n0, 8)[0] == 3
    # 5: a local index that points at the wrong point
    lidx = plan["lidx"].copy()
    lidx[0, 0] = (int(lidx[0, 0]) + 1) % (plan["pts_off"][1])
    assert O.check_plan(_planted(plan, lidx=lidx), md.maps[0], n0, 32)[0] == 5
    # 7: two cells of one thread colour writing the same point
    tcol = np.zeros_like(plan["tcol"])
    ntc = np.ones_like(plan["block_ntcol"])
    assert O.check_plan(_planted(plan, tcol=tcol, block_ntcol=ntc), md.maps[0], n0, 32)[0] == 7
    # 8: two blocks of one block colour writing the same point
    one = np.array([0, plan["n_blocks"]], dtype=np.uint32)
    assert O.check_plan(_planted(plan, n_colours=1, colour_offsets=one), md.maps[0], n0, 32)[0] == 8


def test_is_permutation():
    assert O.is_permutation(np.array([2, 0, 1]))
    assert not O.is_permutation(np.array([2, 0, 2]))
    assert not O.is_permutation(np.array([3, 0, 1]))


def _sector_cases():
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "sectors.json")) as f:
        return json.load(f)


def test_sector_model_matches_the_reference():
    """The numpy restatement of the reference's sector model
    (countCacheLinesForBlock) equals the reference's own counts on the
    fixture meshes (tests/golden/sectors.json), both layouts, two block
    sizes."""
    for c in _sector_cases():
        md = mg.GENERATORS[mg.LOOP_NAMES.index(c["loop"])](seed=1, **c["kwargs"])
        got = O.sector_count(md.maps[0], c["cells_per_block"], c["dim"], c["type_size"], c["soa"])
        assert got == c["sectors"], c
