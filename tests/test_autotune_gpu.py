"""The autotuner picks the tuning knobs by timing; results must not depend on them."""
import pytest

from helpers import assert_same_output
from partc_b200 import _lib, gen

pytestmark = pytest.mark.gpu


def test_autotune_picks_knobs_and_results_stay_exact(engine, oracle_mod):
    work = [gen.Workload("a", gen.random_coo([60, 70, 80], 20000, [1.2] * 3, 11, "uniform01"), 1, [0, 1, 2]),
            gen.Workload("b", gen.random_coo([40, 30, 20, 9], 15000, [1.0] * 4, 12, "normal"), 2, [3, 0, 1, 2])]
    keep = []
    items = _lib.batch_items(work, keep)
    knobs, rep = _lib.autotune(items, repeats=1)
    assert rep["trials"] >= 10
    assert rep["best_ms"] <= rep["default_ms"]
    assert set(knobs) == set(_lib.TUNE_KNOBS)
    res, _ = _lib.batch_contract(items, **knobs)
    for (idx, vals), w in zip(res, work):
        o = oracle_mod.contract(w.tensor, None, w.c, w.modes)
        assert_same_output(idx, vals, o["idx"], o["vals"], bit_exact=True)


@pytest.mark.parametrize("knobs", [dict(large_rows="panels", panel_width=64, warp_task_max_len=1),
                                   dict(small_max_products=128, sort_max_avg_products=64, hash_load_pct=50),
                                   dict(large_rows="panels", panel_width=1024), dict(large_rows="bitmap")])
def test_every_knob_setting_gives_the_same_result(engine, oracle_mod, knobs):
    t = gen.random_coo([300, 200, 40], 60000, [1.3, 1.0, 1.1], 13, "uniform11")
    o = oracle_mod.contract(t, None, 1, [2, 0, 1])
    idx, vals, _ = engine.contract(t, None, 1, [2, 0, 1], **knobs)
    assert_same_output(idx, vals, o["idx"], o["vals"], bit_exact=True)
