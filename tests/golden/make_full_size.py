"""Fixtures that pin the full-size workloads to the reference (run where the reference is present).

    python tests/golden/make_full_size.py

* zipf4d_3m (2482x2862x14036x17, 3.1M nonzeros, contracted modes {0,1}).  The reference cannot
  hold this output in a 62 GB host (it allocates one entry per mult-add, fksCuckooTC.hpp:156), so
  the fixture keeps (1) the exact output count of every row, from the C restatement (oracle/),
  (2) the reference's own output on a seeded sample of whole rows (the 10 rows with the most
  entries and 1000 others), as its entry count and a digest of it in canonical order, and (3) the
  input's digest, so a different generator result is caught before anything is compared.
* skew3d_20m (12000x9000x28000, 20M nonzeros, contracted modes {0,2}): the reference's whole
  output (entry count and digest), and the input's digest.

The restatement's output on the same inputs must give the same digests (checked here).
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from partc_b200 import gen  # noqa: E402
import oracle  # noqa: E402
from helpers import digest, free_keys, input_digest, sample_rows  # noqa: E402

OUT_NPZ = os.path.join(HERE, "full_size", "zipf4d_3m_row_nnz.npz")
OUT_JSON = os.path.join(HERE, "full_size", "pins.json")


def zipf4d():
    w = gen.zipf4d_3m()
    t = w.tensor
    t0 = time.time()
    o = oracle.contract(t, None, w.c, w.modes, mode=oracle.COUNTS)
    row_keys = np.unique(free_keys(t, w.modes[w.c:]))
    assert np.array_equal(row_keys, o["row_key"]), "the restatement's rows are the distinct free keys"
    row_nnz = o["row_nnz"].astype(np.uint32)
    print(f"zipf4d_3m counts: {o['nnz']} entries, {o['flops']} mult-adds ({time.time() - t0:.0f} s)")
    keys = sample_rows(row_keys, row_nnz)
    keep = np.isin(free_keys(t, w.modes[w.c:]), keys)
    r = oracle.ref_self_contract(t, w.c, w.modes, keep_mask=keep)
    sub = gen.CooTensor(idx=t.idx[keep], vals=t.vals[keep], dims=t.dims)
    s = oracle.contract(sub, t, w.c, w.modes, w.modes)
    d_ref, d_or = digest(r["idx"], r["vals"]), digest(s["idx"], s["vals"])
    assert d_ref == d_or, "the restatement differs from the reference on the row sample"
    assert int(r["nnz"]) == int(row_nnz[np.isin(row_keys, keys)].sum())
    print(f"zipf4d_3m sample: {keys.size} rows, {r['nnz']} entries, reference {r['t_wall']:.1f} s")
    return row_nnz, {"input_sha256": input_digest(t), "mult_adds": int(o["flops"]), "out_nnz": int(o["nnz"]),
                     "nrows": int(o["nrows"]), "sample_rows": int(keys.size), "sample_out_nnz": int(r["nnz"]),
                     "sample_sha256": d_ref}


def skew3d():
    w = gen.skew3d_20m()
    t = w.tensor
    r = oracle.ref_self_contract(t, w.c, w.modes)
    o = oracle.contract(t, None, w.c, w.modes)
    d_ref, d_or = digest(r["idx"], r["vals"]), digest(o["idx"], o["vals"])
    assert d_ref == d_or, "the restatement differs from the reference on skew3d_20m"
    print(f"skew3d_20m: {r['nnz']} entries, {o['flops']} mult-adds, reference {r['t_wall']:.1f} s")
    return {"input_sha256": input_digest(t), "mult_adds": int(o["flops"]), "out_nnz": int(r["nnz"]),
            "out_sha256": d_ref}


if __name__ == "__main__":
    if not oracle.ref_available():
        oracle.build()
    row_nnz, z = zipf4d()
    s = skew3d()
    np.savez_compressed(OUT_NPZ, row_nnz=row_nnz)
    with open(OUT_JSON, "w") as f:
        json.dump({"zipf4d_3m": z, "skew3d_20m": s}, f, indent=1)
        f.write("\n")
    print(f"wrote {OUT_JSON} and {OUT_NPZ} ({os.path.getsize(OUT_NPZ) // 1024} KiB)")
