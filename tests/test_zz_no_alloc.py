"""ptc_sizer_predict_noalloc, the sizer inference entry point that allocates no device memory.

It serves callers that cannot allocate device memory where they need a prediction (another
allocator owns the device, or an allocation would synchronize or is not allowed there); its
scratch is a static device array sized for 65536 feature rows.  Its predictions must equal those
of ptc_sizer_predict (the allocating entry point), call after call, because every call
overwrites the shared scratch.  This file is named to run last.
"""
import numpy as np
import pytest

from partc_b200 import _lib

pytestmark = pytest.mark.gpu


def test_noalloc_predictions_equal_the_allocating_entry_point(engine):
    rng = np.random.default_rng(123)
    s = _lib.Sizer.create(seed=21)
    x1 = rng.random((5000, 16), dtype=np.float32) * 2
    x2 = rng.random((777, 16), dtype=np.float32)
    ref1, ref2 = s.predict(x1), s.predict(x2)
    a = s.predict_noalloc(x1)   # first call: also looks up the scratch array on this device
    b = s.predict_noalloc(x2)   # second call in a row: the scratch holds the first call's data
    np.testing.assert_allclose(a, ref1, rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(b, ref2, rtol=1e-4, atol=1e-4)
    c = s.predict_noalloc(x1)
    np.testing.assert_allclose(c, ref1, rtol=1e-4, atol=1e-4)


def test_noalloc_rejects_more_rows_than_its_scratch_holds(engine):
    s = _lib.Sizer.create(seed=22)
    x = np.zeros((65537, 16), dtype=np.float32)
    with pytest.raises(_lib.PtcError) as e:
        s.predict_noalloc(x)
    assert e.value.name == "PTC_ERR_INVALID_ARGUMENT"
    # the largest allowed call works
    y = s.predict_noalloc(np.ones((65536, 16), dtype=np.float32))
    assert y.shape == (65536,) and np.isfinite(y).all()
