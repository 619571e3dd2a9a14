"""Parity at the full workload sizes (marked gpu).

* skew3d_20m (12000x9000x28000, 20M nonzeros, Zipf(1.3) on mode 1, contracted over {0,2}): the
  whole output, bit for bit, against the C restatement and against the digest of the reference's
  own output (tests/golden/full_size/, made by tests/golden/make_full_size.py).
* zipf4d_3m (2482x2862x14036x17, 3.1M nonzeros, Zipf(1.1), contracted over {0,1}; 2.87e9
  mult-adds, 1.70e9 output entries, left on the device): mult-adds and entry count, the entry
  count of every one of the 170k rows against the restatement's exact counts, and every entry of
  a seeded sample of 1010 whole rows bit for bit against the restatement and against the digest
  of the reference's own output on those rows.

Both numeric paths (two-phase and learned) are checked.
"""
import json
import os

import numpy as np
import pytest

from helpers import assert_same_output, digest, free_keys, input_digest, sample_rows
from partc_b200 import gen

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "full_size", "pins.json")) as _f:
    PIN = json.load(_f)

pytestmark = pytest.mark.gpu


class _DeviceArray:
    """A device buffer of the library's output as seen by torch (__cuda_array_interface__)."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def _device_views(out):
    import ctypes as C
    import torch
    n, d = int(out.nnz), int(out.order)
    ip = C.cast(out.idx, C.c_void_p).value
    vp = C.cast(out.vals, C.c_void_p).value
    idx = torch.as_tensor(_DeviceArray(ip, (n, d), "<i4"), device="cuda")
    vals = torch.as_tensor(_DeviceArray(vp, (n,), "<f8"), device="cuda")
    return idx, vals


@pytest.fixture(scope="module")
def skew3d():
    w = gen.skew3d_20m()
    assert input_digest(w.tensor) == PIN["skew3d_20m"]["input_sha256"], "the generator gave a different tensor"
    return w


@pytest.fixture(scope="module")
def skew3d_oracle(skew3d, oracle_mod):
    w = skew3d
    return oracle_mod.contract(w.tensor, None, w.c, w.modes)


@pytest.mark.parametrize("path", ["two_phase", "learned"])
def test_skew3d_20m_whole_output(engine, skew3d, skew3d_oracle, path):
    w, o = skew3d, skew3d_oracle
    pin = PIN["skew3d_20m"]
    idx, vals, st = engine.contract(w.tensor, None, w.c, w.modes, path=path)
    assert st["mult_adds"] == pin["mult_adds"] == o["flops"]
    assert st["out_nnz"] == pin["out_nnz"] == o["nnz"]
    assert_same_output(idx, vals, o["idx"], o["vals"], bit_exact=True)
    assert digest(idx, vals) == pin["out_sha256"], "differs from the reference's own output"


@pytest.fixture(scope="module")
def zipf4d():
    w = gen.zipf4d_3m()
    assert input_digest(w.tensor) == PIN["zipf4d_3m"]["input_sha256"], "the generator gave a different tensor"
    fk = free_keys(w.tensor, w.modes[w.c:])
    row_keys = np.unique(fk)
    row_nnz = np.load(os.path.join(HERE, "golden", "full_size", "zipf4d_3m_row_nnz.npz"))["row_nnz"]
    assert row_keys.size == row_nnz.size == PIN["zipf4d_3m"]["nrows"]
    return w, fk, row_keys, row_nnz


@pytest.fixture(scope="module")
def zipf4d_sample(zipf4d, oracle_mod):
    """The sampled rows' keys and the restatement's output on them (those rows of A times B)."""
    w, fk, row_keys, row_nnz = zipf4d
    keys = sample_rows(row_keys, row_nnz)
    keep = np.isin(fk, keys)
    t = w.tensor
    sub = gen.CooTensor(idx=t.idx[keep], vals=t.vals[keep], dims=t.dims)
    return keys, oracle_mod.contract(sub, t, w.c, w.modes, w.modes)


@pytest.mark.parametrize("path", ["two_phase", "learned"])
def test_zipf4d_3m_rows_and_sample(engine, zipf4d, zipf4d_sample, path):
    import torch
    w, _, row_keys, row_nnz = zipf4d
    keys, o = zipf4d_sample
    pin = PIN["zipf4d_3m"]
    t = w.tensor
    di = torch.from_numpy(t.idx.view(np.int32)).cuda()
    dv = torch.from_numpy(t.vals).cuda()
    keep = []
    coo = engine.device_coo(di.data_ptr(), dv.data_ptr(), t.nnz, t.dims, keep)
    out, st = engine.contract_coo(coo, None, w.c, w.modes, output_location="device", path=path)
    try:
        assert st["mult_adds"] == pin["mult_adds"]
        assert st["out_nnz"] == pin["out_nnz"]
        idx, vals = _device_views(out)
        fa = t.order - w.c
        free = w.modes[w.c:]
        nkeys = 1
        for m in free:
            nkeys *= int(t.dims[m])
        counts = torch.zeros(nkeys, dtype=torch.int64, device="cuda")
        keys_d = torch.from_numpy(keys.astype(np.int64)).cuda()
        got_i, got_v = [], []
        chunk = 1 << 27
        for s in range(0, idx.shape[0], chunk):
            ii = idx[s:s + chunk]
            key = torch.zeros(ii.shape[0], dtype=torch.int64, device="cuda")
            for j, m in enumerate(free):  # the row's tuple: A's free modes, in output order
                key = key * int(t.dims[m]) + ii[:, j].to(torch.int64)
            counts += torch.bincount(key, minlength=nkeys)
            sel = torch.isin(key, keys_d)
            got_i.append(ii[sel].cpu().numpy().view(np.uint32))
            got_v.append(vals[s:s + chunk][sel].cpu().numpy())
            del key, sel
        counts = counts.cpu().numpy()
        assert fa == len(free)
        # every row's entry count equals the exact count, and no entry lies outside A's rows
        assert int(counts.sum()) == pin["out_nnz"]
        assert np.array_equal(counts[row_keys.astype(np.int64)], row_nnz.astype(np.int64)), "row counts differ"
        gi, gv = np.concatenate(got_i), np.concatenate(got_v)
        assert gi.shape[0] == pin["sample_out_nnz"]
        assert_same_output(gi, gv, o["idx"], o["vals"], bit_exact=True)
        assert digest(gi, gv) == pin["sample_sha256"], "differs from the reference's own output on the sample"
    finally:
        engine.free(out)
        torch.cuda.empty_cache()
