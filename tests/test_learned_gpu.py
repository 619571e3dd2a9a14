"""The learned path: the sizer's predictions replace the symbolic pass; parts whose prediction was
too small rerun exactly, so results stay identical to the reference's."""
import os

import numpy as np
import pytest

from helpers import assert_same_output
from oracle import sizer_ref
from partc_b200 import _lib, gen

pytestmark = pytest.mark.gpu

CASE = ([120, 140, 900, 17], 200_000, [1.1] * 4, 51, "uniform01", 2, [0, 1, 2, 3])


@pytest.fixture(scope="module")
def trained():
    xs, ts = [], []
    for seed in range(4):
        w = gen.sizer_member(seed, nnz_scale=0.05)
        x, y = _lib.sizer_collect(w.tensor, None, w.c, w.modes)
        xs.append(x)
        ts.append(y)
    s = _lib.Sizer.create(seed=9)
    s.train(np.concatenate(xs), np.concatenate(ts), epochs=40, batch=1024, lr=3e-3)
    return s


def _run(engine, oracle_mod, sizer, **kw):
    dims, nnz, alphas, seed, values, c, modes = CASE
    t = gen.random_coo(dims, nnz, alphas, seed, values)
    o = oracle_mod.contract(t, None, c, modes)
    idx, vals, st = engine.contract(t, None, c, modes, path="learned", sizer=sizer.h.value, **kw)
    assert_same_output(idx, vals, o["idx"], o["vals"], bit_exact=True)
    assert st["out_nnz"] == o["nnz"]
    return st


def test_learned_path_is_exact(engine, oracle_mod, trained):
    st = _run(engine, oracle_mod, trained)
    assert st["rows_hash"] > 0
    assert st["sizer_mean_abs_log2_err"] < 2.0


def test_learned_path_with_a_sizer_that_predicts_one_entry(engine, oracle_mod):
    """Every prediction far too small: every part overflows and reruns exactly."""
    s = _lib.Sizer.create(seed=1)
    p = np.zeros(sizer_ref.NPARAM, np.float32)
    p[-1] = 1.0  # b3: log2(1 + D) = 1 -> D = 1
    s.set_params(p)
    st = _run(engine, oracle_mod, s)
    assert st["rerun_rows"] > 0


def test_learned_path_with_a_sizer_that_overestimates(engine, oracle_mod):
    s = _lib.Sizer.create(seed=2)
    p = np.zeros(sizer_ref.NPARAM, np.float32)
    p[-1] = 30.0
    s.set_params(p)
    st = _run(engine, oracle_mod, s)
    assert st["rerun_rows"] == 0


def test_learned_path_without_sizer_is_an_error_or_uses_the_default(engine):
    dims, nnz, alphas, seed, values, c, modes = CASE
    t = gen.random_coo(dims, 20_000, alphas, seed, values)
    try:
        engine.contract(t, None, c, modes, path="learned")
    except engine.PtcError as e:
        assert e.name == "PTC_ERR_INVALID_ARGUMENT"


def test_trained_sizer_gains_over_an_untrained_one(engine, oracle_mod):
    """What training buys: on a held-out Zipf contraction the shipped sizer (trained on the seeded
    training contractions) predicts row sizes closely and needs no exact rerun, while the same
    network with its initial weights is far off and reruns rows; both stay exact, and both skip
    the exact symbolic pass of the large rows that the two-phase path runs."""
    t = gen.random_coo([2482, 2862, 14036, 17], 400_000, [1.1] * 4, 2024, "uniform01")
    o = oracle_mod.contract(t, None, 2, [0, 1, 2, 3])
    trained = _lib.Sizer.load(os.path.join(os.path.dirname(_lib.LIB_PATH), "sizer_default.bin"))
    untrained = _lib.Sizer.create(seed=5)
    res = {}
    for name, s in (("trained", trained), ("untrained", untrained)):
        idx, vals, st = engine.contract(t, None, 2, [0, 1, 2, 3], path="learned", sizer=s.h.value)
        assert_same_output(idx, vals, o["idx"], o["vals"], bit_exact=True)
        res[name] = st
    assert res["trained"]["sizer_mean_abs_log2_err"] < 0.25
    assert res["trained"]["rerun_rows"] == 0
    assert res["untrained"]["sizer_mean_abs_log2_err"] > 4 * res["trained"]["sizer_mean_abs_log2_err"]
