"""GPU orderings and partitions (fot_reorder / fot_partition /
fot_reorder_to_partition / fot_renumber_points).

The reference computes these with SCOTCH and METIS, which are absent, so the
exact orderings are not pinned; they are checked by properties:
* every permutation is a bijection; the problem's mappings and datasets are
  exactly the originals renumbered by the reported permutations;
* RCM / GPS shrink the bandwidth and profile of a randomly numbered mesh;
* partitions cover every cell with parts of at most the requested size, and
  reorder_to_partition makes parts contiguous;
* loop results after any sequence of reorderings, un-permuted, equal the
  serial loop on the original numbering (<= 1e-12, FP32 <= 1e-5), and a
  hierarchical plan built on the reordered problem is bit-exact to the CPU
  replay of its colour order.
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


def tol(loop):
    return 1e-5 if loop == mg.VOLNA else 1e-12


def check_consistent(p, md):
    """The problem's state equals md renumbered by the reported permutations."""
    perm = [p.point_permutation(k) for k in range(p.info.n_mappings)]
    order = p.cell_order()
    assert O.is_permutation(order)
    for k in range(p.info.n_mappings):
        assert O.is_permutation(perm[k])
        expect = perm[k][md.maps[k][order]]
        assert np.array_equal(p.mapping(k), expect), k
    for k in range(p.info.n_point_sets):
        cur = p.point_weights(k)
        if k == 0:
            continue  # the incremented dataset, checked by the loop results
        if md.layout == "aos":
            assert bitwise_equal(cur[perm[k]], md.point_data[k])
        else:
            assert bitwise_equal(cur[:, perm[k]], md.point_data[k])
    for j in range(p.info.n_cell_sets):
        assert bitwise_equal(p.cell_weights(j), md.cell_data[j][:, order])


def unpermuted_out(p):
    out = p.point_weights(0)
    perm = p.point_permutation(0)
    return out[perm] if p.layout == "aos" else out[:, perm]


@pytest.mark.parametrize("order", [0, 1, 2, 3])
@pytest.mark.parametrize("loop", range(5))
def test_reorder_consistency_and_results(loop, order):
    md = mg.small(loop, seed=4) if loop != mg.RES_CALC else mg.res_calc(30, 20, 4)
    p = F().Problem.from_mesh(md)
    p.reorder(order, seed=9)
    check_consistent(p, md)
    plan = p.plan(F().EXEC_HIER, 64)
    p.loop_gpu_cell_centred(1)
    plan.run(1)
    p.sync()
    ser, _ = O.serial(md, 2)
    assert rel_err(unpermuted_out(p), ser[0]) <= tol(loop)


@pytest.mark.parametrize("order", [2, 3])
def test_bandwidth_reduction_of_random_numbering(order):
    md = mg.mini_aero(20, seed=2, permute=True)
    bw0, prof0 = O.bandwidth_profile(md.n_points[0], md.maps[0])
    p = F().Problem.from_mesh(md)
    p.reorder(order)
    m = p.mapping(0)
    bw, prof = O.bandwidth_profile(md.n_points[0], m)
    assert bw < bw0 / 5 and prof < prof0 / 5
    # within a factor of 2 of the structured numbering's bandwidth (n^2 = 400)
    assert bw <= 2 * 20 * 20 + 40


def test_rcm_close_to_scipy():
    scipy_sparse = pytest.importorskip("scipy.sparse")
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    md = mg.lulesh(10, seed=3, permute=True)
    n = md.n_points[0]
    ind, ends = O.point_graph(n, md.maps[0])
    a = scipy_sparse.csr_matrix((np.ones(ends.size), ends, ind), shape=(n, n))
    sp = np.asarray(reverse_cuthill_mckee(a, symmetric_mode=True))
    perm_sp = np.empty(n, np.uint32)
    perm_sp[sp] = np.arange(n)
    bw_sp, _ = O.bandwidth_profile(n, perm_sp[md.maps[0]])
    p = F().Problem.from_mesh(md)
    p.reorder(F().ORDER_RCM)
    bw, _ = O.bandwidth_profile(n, p.mapping(0))
    assert bw <= 1.25 * bw_sp


@pytest.mark.parametrize("loop", [mg.RES_CALC, mg.MINI_AERO, mg.LULESH, mg.GETACC])
def test_partition_reorder_renumber(loop):
    md = {mg.RES_CALC: lambda: mg.res_calc(40, 30, 2), mg.MINI_AERO: lambda: mg.mini_aero(10, 2),
          mg.LULESH: lambda: mg.lulesh(9, 2), mg.GETACC: lambda: mg.getacc(30, 25, 2)}[loop]()
    p = F().Problem.from_mesh(md)
    p.reorder(F().ORDER_GPS)
    p.partition(64)
    part = p.partition_vector()
    counts = np.bincount(part)
    # ceil(n / 64) parts within one cell of the mean: the reference's METIS
    # balance (tolerance 1.001) up to integral sizes
    nparts = int(np.ceil(md.n_cells / 64))
    assert counts.size == nparts and counts.sum() == md.n_cells
    mean = md.n_cells / nparts
    assert counts.max() <= min(64, np.ceil(mean)) and counts.min() >= np.floor(mean)
    p.reorder_to_partition()
    part2 = p.partition_vector()
    assert np.all(np.diff(part2.astype(np.int64)) >= 0)
    p.renumber_points()
    check_consistent(p, md)
    plan = p.plan(F().EXEC_HIER, 64, F().PLAN_USE_PARTITION)
    ex = plan.export()
    before = p.mesh_data()  # state after the plan reordered the cells
    plan.run(2)
    p.sync()
    ser, _ = O.serial(md, 2)
    assert rel_err(unpermuted_out(p), ser[0]) <= tol(loop)
    st = plan.stats()
    assert st["n_blocks"] >= md.n_cells // 64


def test_partition_blocks_follow_parts():
    md = mg.res_calc(40, 30, 2)
    p = F().Problem.from_mesh(md)
    p.partition(48)
    part = p.partition_vector().copy()
    mdp = p.mesh_data()
    plan = p.plan(F().EXEC_HIER, 64, F().PLAN_USE_PARTITION)
    ex = plan.export()
    rc, msg = O.check_plan(ex, mdp.maps[0], mdp.n_points[0], 64)
    assert rc == 0, msg
    # every block holds cells of one part
    for b in range(ex["n_blocks"]):
        cells = ex["cell_id"][ex["block_start"][b]:ex["block_start"][b + 1]]
        assert np.unique(part[cells]).size == 1
    plan.run(2)
    p.sync()
    rep, _ = O.replay_hier(mdp, ex, 2)
    assert bitwise_equal(p.point_weights(0), rep[0])


def quality_numpy(map0, part):
    """(part, point) pairs per point and the fraction of shared points, from
    the mapping and a partition (restated on the CPU)."""
    pairs = np.unique(np.stack([map0.astype(np.int64).ravel(),
                                np.repeat(part.astype(np.int64), map0.shape[1])], 1), axis=0)
    pts, cnt = np.unique(pairs[:, 0], return_counts=True)
    return len(pairs) / len(pts), float((cnt > 1).mean())


@pytest.mark.parametrize("loop", [mg.RES_CALC, mg.LULESH, mg.GETACC, mg.MINI_AERO])
def test_partition_quality_beats_contiguous_blocks(loop):
    """The bisection's parts share fewer points than blocks of consecutive
    cells of the RCM order (what the plan would form without a partition)
    and than the region-growing parts; fot_partition_quality agrees with the
    CPU restatement."""
    md = {mg.RES_CALC: lambda: mg.res_calc(80, 60, 3), mg.MINI_AERO: lambda: mg.mini_aero(14, 3),
          mg.LULESH: lambda: mg.lulesh(14, 3), mg.GETACC: lambda: mg.getacc(70, 50, 3)}[loop]()
    res = {}
    for method in ("bisect", "grow"):
        p = F().Problem.from_mesh(md)
        p.reorder(F().ORDER_RCM)
        p.partition(128, method=method)
        q = p.partition_quality()
        ppp, shared = quality_numpy(p.mapping(0), p.partition_vector())
        assert abs(q["pairs_per_point"] - ppp) < 1e-12 and abs(q["shared_points"] - shared) < 1e-12
        res[method] = q
    p = F().Problem.from_mesh(md)
    p.reorder(F().ORDER_RCM)
    contiguous, _ = quality_numpy(p.mapping(0), np.arange(md.n_cells) // 128)
    assert res["bisect"]["parts"] == int(np.ceil(md.n_cells / 128))
    assert res["bisect"]["max_over_mean"] <= 1.0 + res["bisect"]["parts"] / md.n_cells + 1e-12
    assert res["bisect"]["pairs_per_point"] < contiguous
    assert res["bisect"]["pairs_per_point"] <= res["grow"]["pairs_per_point"]


def test_partition_tolerance_is_checked():
    p = F().Problem.from_mesh(mg.res_calc(20, 20, 1))
    with pytest.raises(F().FotError) as e:
        p.partition(32, tolerance=0.9)
    assert e.value.code == -1
    p.partition(32, tolerance=1.0)
    counts = np.bincount(p.partition_vector())
    assert counts.max() - counts.min() <= 1
