"""GPU mesh statistics through the C ABI: the sector model (the reference's
countCacheLinesForBlock, problem.hpp:654-672) equals the reference's own
counts (tests/golden/sectors.json) and the oracle's restatement, over runs of
cells and over a hierarchical plan's blocks; the mapping-spread and
point-degree features equal numpy's."""
import json
import os

import numpy as np
import pytest

from cuda_fot_b200 import meshgen as mg
from oracle import oracle_py as O

pytestmark = pytest.mark.gpu


def F():
    from cuda_fot_b200 import fot
    return fot


def cases():
    with open(os.path.join(os.path.dirname(__file__), "golden", "sectors.json")) as f:
        return json.load(f)


def test_sector_count_matches_reference_fixture():
    for c in cases():
        md = mg.GENERATORS[mg.LOOP_NAMES.index(c["loop"])](seed=1, **c["kwargs"])
        p = F().Problem.from_mesh(md)
        sec, nb = p.sector_count(c["cells_per_block"], "soa" if c["soa"] else "aos")
        assert sec == c["sectors"], c
        assert nb == -(-md.n_cells // c["cells_per_block"])


@pytest.mark.parametrize("loop", range(5))
def test_sector_count_after_reorder_and_plan_blocks(loop):
    md = {mg.RES_CALC: lambda: mg.res_calc(60, 40, 2), mg.MINI_AERO: lambda: mg.mini_aero(12, 2),
          mg.LULESH: lambda: mg.lulesh(10, 2), mg.VOLNA: lambda: mg.volna(40, 30, 2),
          mg.GETACC: lambda: mg.getacc(40, 30, 2)}[loop]()
    dim, ts = md.point_data[0].shape[1], md.point_data[0].dtype.itemsize
    p = F().Problem.from_mesh(md)
    p.reorder(F().ORDER_RCM)
    m0 = p.mapping(0)
    for b in (32, 100, 256):
        for soa in (False, True):
            got, _ = p.sector_count(b, "soa" if soa else "aos")
            assert got == O.sector_count(m0, b, dim, ts, soa), (b, soa)
    plan = p.plan(F().EXEC_HIER, 128)
    ex = plan.export()
    for soa in (False, True):
        got, nb = plan.sector_count("soa" if soa else "aos")
        assert nb == ex["n_blocks"]
        want = 0
        per = 32 // ts
        for b in range(ex["n_blocks"]):
            pts = ex["pts"][ex["pts_off"][b]:ex["pts_off"][b + 1]].astype(np.int64)
            if soa:
                want += dim * len(np.unique(pts // per))
            else:
                want += len(np.unique((pts[:, None] * dim + np.arange(dim)).ravel() // per))
        assert got == want, soa


def test_mesh_features_match_numpy():
    md = mg.lulesh(9, 4, permute=True)
    p = F().Problem.from_mesh(md)
    p.reorder(F().ORDER_GPS)
    m0 = p.mapping(0).astype(np.int64)
    f = p.mesh_features()
    span = m0.max(axis=1) - m0.min(axis=1)
    assert f["span_max"] == span.max()
    assert abs(f["span_mean"] - span.mean()) <= 1e-9 * span.mean()
    deg = np.bincount(m0.ravel(), minlength=md.n_points[0])
    want = [(deg <= 2).mean(), ((deg >= 3) & (deg <= 4)).mean(), ((deg >= 5) & (deg <= 6)).mean(),
            (deg >= 7).mean()]
    assert np.allclose(f["deg_hist"], want, rtol=0, atol=1e-12)


@pytest.mark.parametrize("loop", range(5))
def test_set_layout_matches_host_conversion_and_runs(loop):
    """fot_set_layout converts every point dataset on the GPU, bit-identical
    to the host conversion (the reference's AOStoSOA), both ways; plans built
    before are stale; a plan on the converted problem gives the same result
    as one on a problem created in SOA."""
    from tests.helpers import bitwise_equal
    md = {mg.RES_CALC: lambda: mg.res_calc(40, 30, 5), mg.MINI_AERO: lambda: mg.mini_aero(9, 5),
          mg.LULESH: lambda: mg.lulesh(8, 5), mg.VOLNA: lambda: mg.volna(30, 20, 5),
          mg.GETACC: lambda: mg.getacc(30, 20, 5)}[loop]()
    soa = md.to_layout("soa")
    p = F().Problem.from_mesh(md)
    old = p.plan(F().EXEC_ATOMIC, 256)
    p.set_layout("soa")
    for k, d in enumerate(soa.point_data):
        assert bitwise_equal(p.point_weights(k), d), k
    with pytest.raises(F().FotError) as e:
        old.run(1)
    assert e.value.code == -3
    plan = p.plan(F().EXEC_HIER, 64)
    plan.run(2)
    p.sync()
    q = F().Problem.from_mesh(soa)
    plan_q = q.plan(F().EXEC_HIER, 64)
    plan_q.run(2)
    q.sync()
    assert bitwise_equal(p.point_weights(0), q.point_weights(0))
    p.set_layout("aos")
    for k in range(1, len(md.point_data)):
        assert bitwise_equal(p.point_weights(k), md.point_data[k]), k
