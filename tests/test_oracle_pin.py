"""Pin the C restatement of the reference (oracle/) to the reference itself.

(1) against the golden fixtures made by the reference (tests/golden/make_golden.py);
(2) where oracle/_ref exists (the reference compiled from its sources), against fresh runs of
    the reference on more seeded cases, including row-sampled A operands.
All comparisons are bit-exact: the restatement sums in the reference's order.
"""
import glob
import os

import numpy as np
import pytest

from helpers import assert_same_output, load_golden
from partc_b200 import gen

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_golden(oracle_mod, path):
    t, c, modes, gi, gv = load_golden(path)
    o = oracle_mod.contract(t, None, c, modes)
    assert_same_output(o["idx"], o["vals"], gi, gv, bit_exact=True)
    assert o["nnz"] == gi.shape[0]
    # the per-row exact counts agree with the output
    assert int(o["row_nnz"].sum()) == gi.shape[0]


REF_CASES = [
    ([50, 40, 30], 3_000, [None, None, None], 101, "uniform01", 2, [0, 1, 2]),
    ([50, 40, 30], 3_000, [None, None, None], 102, "uniform01", 1, [2, 0, 1]),
    ([30, 40, 50, 6], 4_000, [1.2, 1.0, 1.1, 0.8], 103, "uniform01", 2, [3, 1, 0, 2]),
    ([100, 20, 100], 5_000, [None, 1.4, None], 104, "normal", 2, [0, 2, 1]),
    ([8, 9, 10, 11, 12], 3_000, [0.9] * 5, 105, "uniform11", 2, [4, 3, 2, 1, 0]),
]


@pytest.mark.parametrize("case", REF_CASES, ids=[f"ref{i}" for i in range(len(REF_CASES))])
def test_oracle_matches_reference(oracle_mod, case):
    if not oracle_mod.ref_available():
        pytest.skip("reference not compiled here (oracle/_ref)")
    dims, nnz, alphas, seed, values, c, modes = case
    t = gen.random_coo(dims, nnz, alphas, seed, values)
    r = oracle_mod.ref_self_contract(t, c, modes)
    o = oracle_mod.contract(t, None, c, modes)
    assert_same_output(o["idx"], o["vals"], r["idx"], r["vals"], bit_exact=True)


def test_oracle_matches_reference_row_sample(oracle_mod):
    """The reference with only some rows of A kept (B whole) equals the restatement of A_subset x B."""
    if not oracle_mod.ref_available():
        pytest.skip("reference not compiled here (oracle/_ref)")
    t = gen.random_coo([40, 50, 60, 7], 6_000, [1.1] * 4, 106, "uniform01")
    c, modes = 2, [0, 1, 2, 3]
    fkey = t.idx[:, 2].astype(np.int64) * 7 + t.idx[:, 3]
    rng = np.random.default_rng(0)
    chosen = rng.choice(np.unique(fkey), size=40, replace=False)
    keep = np.isin(fkey, chosen)
    r = oracle_mod.ref_self_contract(t, c, modes, keep_mask=keep)
    sub = gen.CooTensor(idx=t.idx[keep], vals=t.vals[keep], dims=t.dims)
    o = oracle_mod.contract(sub, t, c, modes, modes)
    assert_same_output(o["idx"], o["vals"], r["idx"], r["vals"], bit_exact=True)


def test_oracle_flop_count(oracle_mod):
    """flops = sum over A nonzeros of the matching fiber length (fksCuckooTC.hpp:94-154)."""
    t = gen.random_coo([30, 30, 30], 2_000, [None, None, None], 107, "uniform01")
    o = oracle_mod.contract(t, None, 2, [0, 1, 2], mode=oracle_mod.FLOPS_ONLY)
    key = t.idx[:, 0].astype(np.int64) * 30 + t.idx[:, 1]
    _, cnt = np.unique(key, return_counts=True)
    assert o["flops"] == int((cnt.astype(np.int64) ** 2).sum())


def test_oracle_rejects_bad_input(oracle_mod):
    t = gen.random_coo([10, 10, 10], 100, [None] * 3, 108, "uniform01")
    bad = gen.CooTensor(idx=t.idx.copy(), vals=t.vals, dims=t.dims)
    bad.idx[5, 1] = 10
    with pytest.raises(ValueError):
        oracle_mod.contract(bad, None, 2, [0, 1, 2])
