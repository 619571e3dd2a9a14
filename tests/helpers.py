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


def digest(idx, vals):
    """sha256 of an output tensor in canonical order (index tuples, then value bits)."""
    import hashlib
    ci, cv = canonical(np.ascontiguousarray(idx, dtype=np.uint32), np.ascontiguousarray(vals, dtype=np.float64))
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(ci).tobytes())
    h.update(np.ascontiguousarray(cv).view(np.uint64).tobytes())
    return h.hexdigest()


def input_digest(t):
    """sha256 of a generated COO tensor (indices, values, mode sizes)."""
    import hashlib
    h = hashlib.sha256()
    for a in (t.idx, t.vals, t.dims):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def free_keys(t, modes):
    """Linearized key of every nonzero over the given modes (first mode most significant)."""
    k = np.zeros(t.nnz, dtype=np.uint64)
    for m in modes:
        k = k * np.uint64(t.dims[m]) + t.idx[:, m].astype(np.uint64)
    return k


def sample_rows(row_keys, row_nnz, n_top=10, n_random=1000, seed=20):
    """Row keys of a seeded sample: the n_top rows with the most output entries and n_random
    other rows drawn uniformly."""
    order = np.argsort(-row_nnz.astype(np.int64), kind="stable")
    top = order[:n_top]
    rest = order[n_top:]
    rng = np.random.default_rng(seed)
    pick = rng.choice(rest, size=min(n_random, rest.size), replace=False)
    return np.sort(row_keys[np.concatenate([top, pick])])
