"""Failure paths of the cuckoo build, injected from the host (marked gpu).

The reference rehashes a bucket with new kDict multipliers and a larger table when its cuckoo
insertion fails (rehash, fksCuckoo.hpp:297-442) and exits with "None of the keys in kDict worked"
when no pair works (:439-441).  Here the build of B's fiber table fails an attempt when an
insertion's eviction chain runs out; the host then rebuilds with new seeds (and twice the buckets
after every two failures), and gives up with PTC_ERR_HASH_BUILD after cuckoo_max_attempts builds.
A chain bound of 0 (no eviction) at 90% load makes the first attempts fail on purpose.
"""
import pytest

from helpers import assert_same_output
from partc_b200 import gen

pytestmark = pytest.mark.gpu

# 200x200x50 uniform, 60k nonzeros, contracted over modes {0,1}: about 31k fibers, so a 90% load
# target gives 2048 buckets of 16 slots, and some first-choice bucket overflows
DIMS, NNZ, C, MODES = [200, 200, 50], 60_000, 2, [0, 1, 2]


@pytest.fixture(scope="module")
def case(oracle_mod):
    t = gen.random_coo(DIMS, NNZ, [None] * 3, 301, "uniform01")
    return t, oracle_mod.contract(t, None, C, MODES)


def test_rebuild_after_failed_attempts_stays_exact(engine, case):
    t, o = case
    idx, vals, st = engine.contract(t, None, C, MODES, cuckoo_max_chain=0, hash_load_pct=90)
    assert st["hash_attempts"] > 1, "the injected chain bound should fail the first build"
    assert st["nfibers"] == o["nfibers"]
    assert_same_output(idx, vals, o["idx"], o["vals"], bit_exact=True)
    # the default bound builds at the first attempt
    idx, vals, st = engine.contract(t, None, C, MODES)
    assert st["hash_attempts"] == 1
    assert_same_output(idx, vals, o["idx"], o["vals"], bit_exact=True)


@pytest.mark.parametrize("path", ["two_phase", "learned"])
def test_exhausted_attempts_return_hash_build_and_free_everything(engine, case, path):
    t, _ = case
    before = engine.device_pool_in_use()
    with pytest.raises(engine.PtcError) as e:
        engine.contract(t, None, C, MODES, cuckoo_max_chain=0, cuckoo_max_attempts=1, hash_load_pct=90, path=path)
    assert e.value.name == "PTC_ERR_HASH_BUILD"
    assert engine.device_pool_in_use() == before, "the failed call left device memory allocated"
    # the library is usable afterwards
    _, _, st = engine.contract(t, None, C, MODES, path=path)
    assert st["hash_attempts"] == 1
    assert engine.device_pool_in_use() == before


def test_batch_reports_hash_build_failure(engine, case):
    t, _ = case
    keep = []
    items = engine.batch_items([gen.Workload("a", t, C, MODES), gen.Workload("b", t, C, MODES)], keep)
    before = engine.device_pool_in_use()
    with pytest.raises(engine.PtcError) as e:
        engine.batch_contract(items, outputs="none", cuckoo_max_chain=0, cuckoo_max_attempts=1, hash_load_pct=90)
    assert e.value.name == "PTC_ERR_HASH_BUILD"
    assert engine.device_pool_in_use() == before
