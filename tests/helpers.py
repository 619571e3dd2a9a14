"""Shared helpers for the tests (canonical comparison of COO outputs)."""
import numpy as np


def canonical(idx, vals):
    if idx.shape[0] == 0:
        return idx, vals
    order = np.lexsort(idx.T[::-1])
    return idx[order], vals[order]


def assert_same_output(idx_a, vals_a, idx_b, vals_b, bit_exact=True, rtol=1e-12):
    """Index sets must be identical; values bit-identical (or within rtol of the larger of |v| and
    the sum of |terms|, when a test states a summation order different from the reference)."""
    ia, va = canonical(idx_a, vals_a)
    ib, vb = canonical(idx_b, vals_b)
    assert ia.shape == ib.shape, f"nnz {ia.shape[0]} != {ib.shape[0]}"
    assert np.array_equal(ia, ib), "index sets differ"
    if bit_exact:
        same = (va.view(np.uint64) == vb.view(np.uint64))
        if not same.all():
            bad = np.flatnonzero(~same)[:5]
            raise AssertionError(f"{(~same).sum()} values differ, e.g. {va[bad]} vs {vb[bad]}")
    else:
        np.testing.assert_allclose(va, vb, rtol=rtol, atol=0)


def load_golden(path):
    from partc_b200.gen import CooTensor
    z = np.load(path)
    t = CooTensor(idx=z["idx"], vals=z["vals"], dims=z["dims"])
    return t, int(z["c"]), [int(x) for x in z["modes"]], z["out_idx"], z["out_vals"]
