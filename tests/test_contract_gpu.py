"""Parity of the CUDA engine (through the C ABI) with the reference and its C restatement.

Indices and nnz must be identical as sets; values must be bit-identical (the engine sums in the
reference's order: per output entry, a left fold over the row's A nonzeros in COO input order).
"""
import glob
import os

import numpy as np
import pytest

from helpers import assert_same_output, canonical, load_golden
from partc_b200 import gen

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_golden(engine, path):
    t, c, modes, gi, gv = load_golden(path)
    idx, vals, st = engine.contract(t, None, c, modes)
    assert_same_output(idx, vals, gi, gv, bit_exact=True)
    assert st["out_nnz"] == gi.shape[0]


CASES = [
    # dims, nnz, alphas, seed, values, c, modes
    ([500, 400, 300], 50_000, [None] * 3, 0, "uniform01", 2, [0, 1, 2]),
    ([120, 140, 900, 17], 200_000, [1.1] * 4, 21, "uniform01", 2, [0, 1, 2, 3]),
    ([120, 140, 900, 17], 200_000, [1.1] * 4, 21, "uniform01", 2, [1, 2, 0, 3]),
    ([2000, 900, 3000], 300_000, [None, 1.3, None], 22, "normal", 2, [0, 2, 1]),
    ([300, 200, 100], 40_000, [None] * 3, 23, "uniform11", 1, [2, 0, 1]),
    ([20, 30, 25, 40, 10], 60_000, [0.9] * 5, 24, "uniform01", 3, [4, 0, 2, 1, 3]),
]


_ORACLE = {}


def _case_and_oracle(oracle_mod, i):
    """Case i's tensor and the restatement's output (computed once per test session)."""
    if i not in _ORACLE:
        dims, nnz, alphas, seed, values, c, modes = CASES[i]
        t = gen.random_coo(dims, nnz, alphas, seed, values)
        _ORACLE[i] = (t, oracle_mod.contract(t, None, c, modes))
    return _ORACLE[i]


# large-row accumulators: the row bitmap kernel, and the panel kernels (warp tasks and block
# parts) at the automatic, narrowest and widest panel widths
KERNELS = [("bitmap", 0), ("panels", 0), ("panels", 64), ("panels", 4096)]


@pytest.mark.parametrize("case", range(len(CASES)), ids=[f"c{i}" for i in range(len(CASES))])
@pytest.mark.parametrize("kernel", KERNELS, ids=[f"{k}{p}" for k, p in KERNELS])
@pytest.mark.parametrize("path", ["two_phase", "learned"])
def test_against_oracle(engine, oracle_mod, case, kernel, path):
    t, o = _case_and_oracle(oracle_mod, case)
    _, _, _, _, _, c, modes = CASES[case]
    large_rows, panel = kernel
    idx, vals, st = engine.contract(t, None, c, modes, panel_width=panel, large_rows=large_rows, path=path)
    assert st["mult_adds"] == o["flops"]
    assert st["nrows"] == o["nrows"] and st["nfibers"] == o["nfibers"]
    assert_same_output(idx, vals, o["idx"], o["vals"], bit_exact=True)


@pytest.mark.parametrize("path", ["two_phase", "learned"])
def test_dense_tasks_fuller_than_the_slot_list(engine, oracle_mod, path):
    """Rows of ~200 A nonzeros (warp tasks) over 2000 columns that all appear: dense tasks of 768
    columns fill every slot, more than a warp's list of filled slots holds, so their emission
    lists and writes the table a part at a time."""
    t = gen.random_coo([60, 50, 2000], 400_000, [None] * 3, 39, "uniform01")
    o = oracle_mod.contract(t, None, 2, [0, 1, 2])
    idx, vals, st = engine.contract(t, None, 2, [0, 1, 2], large_rows="panels", path=path)
    assert st["mult_adds"] == o["flops"]
    assert st["out_nnz"] == o["nnz"] > 0.99 * 2000 * 2000
    assert_same_output(idx, vals, o["idx"], o["vals"], bit_exact=True)


def test_general_two_tensors(engine, oracle_mod):
    """A x B with different tensors and different mode positions (the reference's
    tc_fksCuckoo signature takes two tensors)."""
    A = gen.random_coo([40, 300, 50], 30_000, [None, 1.1, None], 31, "uniform01")
    B = gen.random_coo([50, 60, 40, 8], 40_000, [None, 1.0, None, None], 32, "uniform11")
    # contract A's modes (0, 2) with B's modes (2, 0); free: A mode 1, B modes 1, 3
    o = oracle_mod.contract(A, B, 2, [0, 2, 1], [2, 0, 3, 1])
    idx, vals, st = engine.contract(A, B, 2, [0, 2, 1], [2, 0, 3, 1])
    assert_same_output(idx, vals, o["idx"], o["vals"], bit_exact=True)


@pytest.mark.parametrize("path", ["two_phase", "learned"])
def test_more_than_two_million_columns(engine, oracle_mod, path):
    """B with about 2.6M distinct free keys (columns): more than one shared-memory bitmap holds, so
    the exact symbolic pass sweeps each row in column windows.  The reference sizes each row's
    accumulator by the row alone (fksCuckooSPA.hpp:637-645) and has no column limit either."""
    B = gen.random_coo([4000, 3000, 3000], 3_000_000, [None] * 3, 41, "uniform01")
    A = gen.random_coo([4000, 50], 2_000, [None, None], 42, "uniform11")
    o = oracle_mod.contract(A, B, 1, [0, 1], [0, 1, 2])
    idx, vals, st = engine.contract(A, B, 1, [0, 1], [0, 1, 2], path=path)
    assert st["ncols"] > 2_000_000
    assert st["mult_adds"] == o["flops"]
    assert_same_output(idx, vals, o["idx"], o["vals"], bit_exact=True)


def _one_entry_contraction(products):
    """A (K x 1) times B (K x 1) over mode 0 with b = 1: one output entry whose products are
    `products` in this order (the left fold's order: A's COO order)."""
    K = len(products)
    A = gen.CooTensor(idx=np.stack([np.arange(K), np.zeros(K, np.int64)], 1).astype(np.uint32),
                      vals=np.asarray(products, np.float64), dims=np.array([K, 1], np.uint32))
    B = gen.CooTensor(idx=np.stack([np.arange(K), np.zeros(K, np.int64)], 1).astype(np.uint32),
                      vals=np.ones(K), dims=np.array([K, 1], np.uint32))
    return A, B


@pytest.mark.parametrize("kind", ["squares", "signs", "magnitudes", "ties", "cancel"])
def test_long_runs_fold_exactly(engine, oracle_mod, kind):
    """An output entry that 100k+ products meet is folded by a block on the grid of the running
    value's ulp; the result must still be the sequential left fold to the bit, whatever the
    values: ties broken by parity, binade crossings, cancellation, magnitudes far apart."""
    rng = np.random.default_rng(61)
    n = 120_000
    if kind == "squares":
        p = rng.standard_normal(n) ** 2
    elif kind == "signs":
        p = rng.standard_normal(n)
    elif kind == "magnitudes":
        p = rng.standard_normal(n) * np.exp(rng.uniform(-40, 40, n))
    elif kind == "ties":
        p = np.concatenate([[1.0], np.tile([2.0 ** -53, 3 * 2.0 ** -53, 2.0 ** -52, 5 * 2.0 ** -54], n // 4),
                            rng.random(1000)])
    else:
        p = np.tile([1e16, 1.0, -1e16, 3.0, 0.5, -0.25], n // 6).astype(np.float64)
    A, B = _one_entry_contraction(p)
    o = oracle_mod.contract(A, B, 1, [0, 1], [0, 1])
    idx, vals, st = engine.contract(A, B, 1, [0, 1], [0, 1])
    assert st["out_nnz"] == 1 and o["nnz"] == 1
    seq = p[0]
    for x in p[1:].tolist():
        seq = seq + x
    assert vals.view(np.uint64)[0] == np.float64(seq).view(np.uint64) == o["vals"].view(np.uint64)[0]


def test_output_is_canonical_for_panel_rows(engine, oracle_mod):
    """Rows come out in increasing free-key order; panel rows in increasing column order."""
    t = gen.random_coo([50, 40, 3000], 100_000, [None, None, 1.0], 33, "uniform01")
    idx, vals, st = engine.contract(t, None, 2, [0, 1, 2], panel_width=1024)
    ci, cv = canonical(idx, vals)
    # every row's entries are contiguous in the engine's output
    rows = idx[:, 0]
    changes = np.count_nonzero(np.diff(rows.astype(np.int64)) != 0) + 1
    assert changes == np.unique(rows).size


def test_device_output_and_inputs(engine, oracle_mod):
    import torch
    t = gen.random_coo([100, 80, 60], 20_000, [None] * 3, 34, "uniform01")
    o = oracle_mod.contract(t, None, 2, [0, 1, 2])
    di = torch.from_numpy(t.idx.astype(np.int32)).cuda()
    dv = torch.from_numpy(t.vals).cuda()
    keep = []
    ca = engine.device_coo(di.data_ptr(), dv.data_ptr(), t.nnz, t.dims, keep)
    out, st = engine.contract_coo(ca, None, 2, [0, 1, 2], output_location="device")
    try:
        n, d = out.nnz, out.order
        idx = _wrap(out.idx, n * d, torch.int32).cpu().numpy().astype(np.uint32).reshape(n, d)
        vals = _wrap(out.vals, n, torch.float64).cpu().numpy()
    finally:
        engine.free(out)
    assert_same_output(idx, vals, o["idx"], o["vals"], bit_exact=True)


def _wrap(ptr, n, dtype):
    """A torch view of n elements at a raw device pointer."""
    import ctypes

    import torch
    addr = ctypes.cast(ptr, ctypes.c_void_p).value

    class _CAI:
        __cuda_array_interface__ = {
            "shape": (n,), "typestr": {torch.int32: "<i4", torch.float64: "<f8"}[dtype],
            "data": (addr, False), "version": 3, "strides": None,
        }
    return torch.as_tensor(_CAI(), device="cuda")


def test_error_empty_contraction(engine):
    # contracted keys of A never meet a fiber of B
    A = gen.random_coo([10, 10, 10], 50, [None] * 3, 35, "uniform01")
    B = gen.CooTensor(idx=A.idx.copy(), vals=A.vals.copy(), dims=A.dims.copy())
    A.idx[:, 0] = 0
    B.idx[:, 0] = 1
    B.idx[:, 2] = np.arange(B.nnz) % 10  # keep B free of accidental duplicates of A
    with pytest.raises(engine.PtcError) as e:
        engine.contract(A, B, 1, [0, 1, 2], [0, 1, 2])
    assert e.value.name == "PTC_ERR_EMPTY_CONTRACTION"


def test_error_index_range(engine):
    t = gen.random_coo([10, 10, 10], 200, [None] * 3, 36, "uniform01")
    bad = gen.CooTensor(idx=t.idx.copy(), vals=t.vals, dims=t.dims)
    bad.idx[17, 2] = 10
    with pytest.raises(engine.PtcError) as e:
        engine.contract(bad, None, 2, [0, 1, 2])
    assert e.value.name == "PTC_ERR_INDEX_RANGE"


def test_repeatable(engine):
    """Values are deterministic (fixed summation order); within a row the entry order is hash
    order, which may differ between runs, as in the reference."""
    t = gen.random_coo([120, 140, 900, 17], 100_000, [1.1] * 4, 37, "uniform01")
    a = engine.contract(t, None, 2, [0, 1, 2, 3])
    b = engine.contract(t, None, 2, [0, 1, 2, 3])
    assert_same_output(a[0], a[1], b[0], b[1], bit_exact=True)
    # rows appear in the same order (increasing free key) in both runs
    ra = a[0][:, :2]
    rb = b[0][:, :2]
    assert np.array_equal(ra, rb)


def test_dropin_driver(engine, oracle_mod, tmp_path):
    """The drop-in driver takes the reference's command line and prints its lines."""
    import subprocess

    from partc_b200 import build as b
    t = gen.random_coo([60, 70, 80, 9], 20_000, [1.1] * 4, 38, "uniform01")
    tns, meta = str(tmp_path / "t.tns"), str(tmp_path / "t.meta")
    gen.write_tns(tns, t)
    gen.write_meta(meta, 2, [1, 2, 0, 3])
    r = subprocess.run([b.BIN, tns, meta, "0", "1"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert lines[0].split() == [str(int(x)) for x in t.idx.max(axis=0) + 1]
    for name in ("Number of elements inserted", "Total time for insertion", "Total time for preprocessing",
                 "Total time for tensor contraction"):
        assert any(l.startswith(name) for l in lines), name
    nnz = int([l for l in lines if l.startswith("Total number of nonzeros in the output tensor")][0].split("=")[1])
    dims = (t.idx.max(axis=0) + 1).astype(np.uint32)
    o = oracle_mod.contract(gen.CooTensor(idx=t.idx, vals=t.vals, dims=dims), None, 2, [1, 2, 0, 3])
    assert nnz == o["nnz"]


@pytest.mark.parametrize("path", ["two_phase", "learned"])
def test_sort_rows_gives_canonical_order(engine, oracle_mod, path):
    """sort_rows=1: rows in increasing free-key order, each row in increasing column order --
    the lexicographic order of the output tuples when free keys follow the modes' order."""
    t = gen.random_coo([80, 60, 300], 40000, [1.2, 1.0, 1.1], 21, "uniform01")
    o = oracle_mod.contract(t, None, 1, [0, 1, 2])
    idx, vals, _ = engine.contract(t, None, 1, [0, 1, 2], sort_rows=1, path=path)
    assert_same_output(idx, vals, o["idx"], o["vals"], bit_exact=True)
    order = np.lexsort(idx.T[::-1])
    assert np.array_equal(order, np.arange(len(order)))
