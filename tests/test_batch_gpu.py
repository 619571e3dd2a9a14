"""Batched contraction (ptc_batch_contract): many uneven contractions as one problem.  Every
item's output must equal the oracle's for that item alone -- same entries, bit-identical values --
whatever the waves, the output mode or the path."""
import ctypes as C

import numpy as np
import pytest

from helpers import assert_same_output
from oracle import sizer_ref
from partc_b200 import _lib, gen

pytestmark = pytest.mark.gpu


def _items():
    """Self-contractions of 3-D and 4-D tensors with 1-2 contracted modes, an A x B item of
    different orders, an item with no matching fiber, an item with one nonzero and an empty one."""
    W = gen.Workload
    R = gen.random_coo
    work, bs = [], []
    specs = [
        ([40, 50, 60], 3000, [1.1] * 3, 1, 1, [0, 1, 2]),
        ([40, 50, 60], 5000, [None] * 3, 2, 2, [2, 0, 1]),
        ([30, 20, 25, 9], 4000, [1.2] * 4, 3, 1, [3, 1, 0, 2]),
        ([30, 20, 25, 9], 2000, [0.9] * 4, 4, 2, [1, 2, 0, 3]),
        ([300, 200, 9], 20000, [1.3, 1.0, 1.0], 5, 1, [2, 0, 1]),
        ([64, 64, 64], 1, [None] * 3, 6, 1, [0, 1, 2]),
    ]
    for dims, nnz, al, seed, c, modes in specs:
        work.append(W(f"s{seed}", R(dims, nnz, al, seed, "uniform11"), c, modes))
        bs.append(None)
    # A (3-D) x B (4-D) over one mode of size 35
    a = R([35, 40, 12], 3000, [1.1] * 3, 7, "normal")
    b = R([9, 35, 7, 11], 5000, [1.0] * 4, 8, "normal")
    work.append(W("ab", a, 1, [0, 2, 1]))
    bs.append((b, [1, 0, 3, 2]))
    # A x B with disjoint contracted indices: no matching fiber
    a2 = gen.CooTensor(idx=np.array([[0, 1], [1, 2]], np.uint32), vals=np.array([1.0, 2.0]), dims=np.array([4, 5]))
    b2 = gen.CooTensor(idx=np.array([[2, 0], [3, 4]], np.uint32), vals=np.array([3.0, 4.0]), dims=np.array([4, 5]))
    work.append(W("disjoint", a2, 1, [0, 1]))
    bs.append((b2, [0, 1]))
    # empty A
    e = gen.CooTensor(idx=np.zeros((0, 3), np.uint32), vals=np.zeros(0), dims=np.array([5, 6, 7]))
    work.append(W("empty", e, 1, [0, 1, 2]))
    bs.append(None)
    return work, bs


def _out_order(w, b):
    oa = len(w.tensor.dims) - w.c
    ob = (len(b[0].dims) if b is not None else len(w.tensor.dims)) - w.c
    return oa + ob


def _expected(oracle_mod, work, bs):
    exp = []
    for w, b in zip(work, bs):
        empty = (np.zeros((0, _out_order(w, b)), np.uint32), np.zeros(0))
        if w.tensor.idx.shape[0] == 0:
            exp.append(empty)
            continue
        B, bm = (None, None) if b is None else b
        try:
            o = oracle_mod.contract(w.tensor, B, w.c, w.modes, bm)
            exp.append((o["idx"], o["vals"]))
        except ValueError:  # no matching fiber
            exp.append(empty)
    return exp


@pytest.fixture(scope="module")
def case(oracle_mod):
    work, bs = _items()
    return work, bs, _expected(oracle_mod, work, bs)


def _check(res, exp):
    assert len(res) == len(exp)
    for (idx, vals), (ei, ev) in zip(res, exp):
        assert idx.shape[1] == ei.shape[1]
        assert_same_output(idx, vals, ei, ev, bit_exact=True)


@pytest.mark.parametrize("wave_mib", [0, 1])
def test_batch_matches_oracle_per_item(engine, case, wave_mib):
    work, bs, exp = case
    keep = []
    items = _lib.batch_items(work, keep, bs)
    res, st = _lib.batch_contract(items, batch_wave_mib=wave_mib)
    _check(res, exp)
    assert st["out_nnz"] == sum(e[0].shape[0] for e in exp)
    if wave_mib == 1:
        assert st["batch_waves"] >= 2


def test_batch_sink_views(engine, case):
    work, bs, exp = case
    keep = []
    items = _lib.batch_items(work, keep, bs)
    got = {}

    def sink(i, t):
        n, d = t.nnz, t.order
        if n == 0:
            got[i] = (np.zeros((0, d), np.uint32), np.zeros(0))
            return
        idx = np.ctypeslib.as_array(t.idx, shape=(n * d,)).reshape(n, d).copy()
        vals = np.ctypeslib.as_array(t.vals, shape=(n,)).copy()
        got[i] = (idx, vals)

    _lib.batch_contract(items, outputs="sink", sink=sink, batch_wave_mib=1)
    assert sorted(got) == list(range(len(work)))
    _check([got[i] for i in range(len(work))], exp)


def test_batch_device_outputs(engine, case):
    import torch
    torch.cuda.init()
    rt = C.CDLL("libcudart.so.12")  # already loaded by torch
    rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    work, bs, exp = case
    keep = []
    items = _lib.batch_items(work, keep, bs)
    outs, st = _lib.batch_contract(items, outputs="device")
    res = []
    for t in outs:
        n, d = t.nnz, t.order
        idx = np.zeros((n, d), np.uint32)
        vals = np.zeros(n, np.float64)
        if n:
            assert t.location == _lib.PTC_DEVICE
            assert rt.cudaMemcpy(idx.ctypes.data, C.addressof(t.idx.contents), n * d * 4, 2) == 0
            assert rt.cudaMemcpy(vals.ctypes.data, C.addressof(t.vals.contents), n * 8, 2) == 0
        res.append((idx, vals))
        _lib.free(t)
    _check(res, exp)


def test_batch_learned_is_exact(engine, case):
    work, bs, exp = case
    keep = []
    items = _lib.batch_items(work, keep, bs)
    res, st = _lib.batch_contract(items, path="learned")
    _check(res, exp)


def test_batch_learned_with_a_sizer_that_predicts_one_entry(engine, case):
    work, bs, exp = case
    s = _lib.Sizer.create(seed=3)
    p = np.zeros(sizer_ref.NPARAM, np.float32)
    p[-1] = 1.0  # log2(1 + nnz) = 1 for every row
    s.set_params(p)
    keep = []
    items = _lib.batch_items(work, keep, bs)
    res, st = _lib.batch_contract(items, path="learned", sizer=s.h.value, batch_wave_mib=1)
    _check(res, exp)
    assert st["rerun_items"] > 0


def test_batch_of_generated_members(engine, oracle_mod):
    """Members of the 4096-member uneven batch workload whose products the oracle finishes fast."""
    work = []
    seed = 0
    while len(work) < 24:
        w = gen.batch_member(seed)
        seed += 1
        key = np.zeros(w.tensor.nnz, np.int64)
        for j in range(w.c):
            key = key * int(w.tensor.dims[w.modes[j]]) + w.tensor.idx[:, w.modes[j]].astype(np.int64)
        _, cnt = np.unique(key, return_counts=True)
        if int((cnt.astype(np.int64) ** 2).sum()) <= 3_000_000:
            work.append(w)
    exp = _expected(oracle_mod, work, [None] * len(work))
    keep = []
    items = _lib.batch_items(work, keep)
    for path in ("two_phase", "learned"):
        res, st = _lib.batch_contract(items, path=path)
        _check(res, exp)


def test_batch_rejects_bad_items(engine):
    t = gen.random_coo([10, 10, 10], 100, [None] * 3, 1, "uniform01")
    keep = []
    items = _lib.batch_items([gen.Workload("a", t, 1, [0, 1, 2])], keep)
    items[0].c = 5
    with pytest.raises(_lib.PtcError) as e:
        _lib.batch_contract(items)
    assert e.value.name == "PTC_ERR_INVALID_ARGUMENT"
    assert "item 0" in str(e.value)
