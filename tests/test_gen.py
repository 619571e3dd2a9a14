"""The seeded workload generator: determinism, distinct coordinates, bounds, file formats."""
import numpy as np

from partc_b200 import gen


def test_deterministic_and_distinct():
    a = gen.random_coo([50, 60, 70, 5], 20_000, [1.1] * 4, 7, "uniform01")
    b = gen.random_coo([50, 60, 70, 5], 20_000, [1.1] * 4, 7, "uniform01")
    assert np.array_equal(a.idx, b.idx) and np.array_equal(a.vals, b.vals)
    key = ((a.idx[:, 0].astype(np.int64) * 60 + a.idx[:, 1]) * 70 + a.idx[:, 2]) * 5 + a.idx[:, 3]
    assert np.unique(key).size == a.nnz
    assert (a.idx < a.dims[None, :]).all()
    assert ((a.vals >= 0) & (a.vals < 1)).all()


def test_value_distributions():
    n = gen.random_coo([100, 100, 100], 10_000, [None] * 3, 1, "normal")
    assert abs(n.vals.mean()) < 0.05 and abs(n.vals.std() - 1) < 0.05
    u = gen.random_coo([100, 100, 100], 10_000, [None] * 3, 1, "uniform11")
    assert u.vals.min() >= -1 and u.vals.max() < 1 and u.vals.min() < -0.9


def test_zipf_skew():
    t = gen.random_coo([1000, 1000], 50_000, [1.3, None], 3, "uniform01")
    counts = np.bincount(t.idx[:, 0], minlength=1000)
    assert counts[0] > 20 * np.median(counts)


def test_tns_and_meta_roundtrip(tmp_path):
    t = gen.random_coo([7, 8, 9], 50, [None] * 3, 5, "uniform01")
    p = str(tmp_path / "t.tns")
    gen.write_tns(p, t)
    r = gen.read_tns(p)
    assert np.array_equal(r.idx, t.idx) and np.array_equal(r.vals, t.vals)
    assert (r.dims <= t.dims).all()
    m = str(tmp_path / "t.meta")
    gen.write_meta(m, 2, [1, 2, 0])
    assert gen.read_meta(m, 3) == (2, [1, 2, 0])


def test_batch_member_shapes():
    for s in range(5):
        w = gen.batch_member(s)
        assert w.tensor.order in (3, 4)
        assert 1 <= w.c <= 2
        assert (64 <= w.tensor.dims).all() and (w.tensor.dims <= 4096).all()
        assert 1 <= w.tensor.nnz <= 200_000


def test_every_named_workload_has_a_one_line_description():
    for name in gen.WORKLOADS:
        d = gen.describe(name)
        assert d and "\n" not in d and not d.endswith(".")
