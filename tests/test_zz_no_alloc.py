"""fot_model_predict_noalloc: the cost model's forward pass with its device
scratch in a fixed file-scope array instead of per-call allocations.

Collected last on purpose (file name): it must pass alone and after every
other test.  Two calls in a row give the same predictions as
fot_model_predict; more rows than the fixed array holds are rejected.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _model_and_rows(n, seed=5):
    from cuda_fot_b200 import costmodel as CM
    m = CM.CostModel(seed=seed)
    rng = np.random.default_rng(seed)
    m.set_normalisation(rng.normal(size=CM.N_FEATURES).astype(np.float32),
                        rng.uniform(0.5, 2.0, CM.N_FEATURES).astype(np.float32))
    X = rng.normal(size=(n, CM.N_FEATURES)).astype(np.float32)
    return m, X


def test_noalloc_predict_matches_predict_twice_in_a_row():
    from cuda_fot_b200 import costmodel as CM
    m, X = _model_and_rows(1000)
    ref = m.predict(X)
    y1 = m.predict_noalloc(X)
    y2 = m.predict_noalloc(X[:700])
    np.testing.assert_allclose(y1, ref, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(y2, ref[:700], rtol=1e-6, atol=1e-6)
    # the full capacity in one call
    m2, X2 = _model_and_rows(CM.NOALLOC_MAX_ROWS, seed=6)
    np.testing.assert_allclose(m2.predict_noalloc(X2), m2.predict(X2), rtol=1e-6, atol=1e-6)


def test_noalloc_predict_rejects_more_rows_than_its_scratch():
    from cuda_fot_b200 import costmodel as CM
    from cuda_fot_b200 import fot as F
    m, X = _model_and_rows(CM.NOALLOC_MAX_ROWS + 1)
    with pytest.raises(F.FotError) as e:
        m.predict_noalloc(X)
    assert e.value.code == -4 and "at most" in str(e.value)
