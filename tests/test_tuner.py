"""The autotuner's candidates: labels round-trip through the profiling
entry point's parser (CPU), and a candidate in either point layout builds a
problem whose run matches the serial loop (GPU)."""
import pytest

from cuda_fot_b200 import meshgen as mg
from oracle import oracle_py as O
from tests.helpers import rel_err


def test_candidate_labels_round_trip():
    from cuda_fot_b200 import tune as T
    from cuda_fot_b200.profile_case import parse_plan
    full, quick = T.default_candidates(mg.RES_CALC), T.default_candidates(mg.MINI_AERO, quick=True)
    for cs in (full, quick):
        assert len({c.label() for c in cs}) == len(cs)  # labels are unique
    for c in full + quick:
        assert parse_plan(c.label()) == c, c.label()
    assert {c.layout for c in full} == {"aos", "soa"}


@pytest.mark.gpu
@pytest.mark.parametrize("label", ["gps/atomic/256@soa", "rcm/atomic-plain/256", "gps/hier/128@soa",
                                   "gps+part128/hier/128@soa", "as-is/hierd/128"])
def test_candidate_builds_and_matches_serial(label):
    from cuda_fot_b200 import tune as T
    from cuda_fot_b200.profile_case import parse_plan
    md = mg.res_calc(48, 40, 4)
    cache = T.OrderedCache(md)
    cand = parse_plan(label)
    mdo = cache.get(cand.order, cand.partition, cand.layout)
    assert mdo.layout == cand.layout
    p, plan = T.build(mdo, cand)
    plan.run(2)
    p.sync()
    ser, _ = O.serial(mdo, 2)
    assert rel_err(p.point_weights(0), ser[0]) <= 1e-12
