"""Generate the golden fixtures from the reference itself (run where the reference is present).

    python tests/golden/make_golden.py

For each small case below, the reference's own fksCuckooTC path (oracle/_ref, compiled from the
reference's unmodified sources) contracts a seeded synthetic tensor with itself, exactly as its
main.cpp does; the inputs and the output tensor (sorted lexicographically by index tuple, since
the reference emits rows in hash order) are stored in tests/golden/<name>.npz.  The tests check
both the C restatement (oracle/) and the CUDA engine against these files, bit for bit.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from partc_b200 import gen  # noqa: E402
import oracle  # noqa: E402

# name: (dims, nnz, alphas, seed, values, c, modes)
CASES = {
    "uniform3d_5k": ([500, 400, 300], 5_000, [None, None, None], 10, "uniform01", 2, [0, 1, 2]),
    "zipf4d_3k": ([60, 70, 80, 9], 3_000, [1.1, 1.1, 1.1, 1.1], 11, "uniform01", 2, [0, 1, 2, 3]),
    "zipf4d_3k_meta4d": ([60, 70, 80, 9], 3_000, [1.1, 1.1, 1.1, 1.1], 11, "uniform01", 2, [1, 2, 0, 3]),
    "uniform3d_c1": ([400, 300, 200], 1_500, [None, None, None], 12, "uniform01", 1, [1, 0, 2]),
    "skew3d_normal": ([300, 200, 400], 20_000, [None, 1.3, None], 13, "normal", 2, [0, 2, 1]),
    "zipf5d_c3": ([12, 14, 10, 30, 25], 4_000, [0.9, 0.9, 0.9, 0.9, 0.9], 14, "uniform11", 3, [4, 0, 2, 1, 3]),
}


def make(name: str):
    dims, nnz, alphas, seed, values, c, modes = CASES[name]
    t = gen.random_coo(dims, nnz, alphas, seed, values)
    r = oracle.ref_self_contract(t, c, modes)
    idx, vals = oracle.canonical(r["idx"], r["vals"])
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, idx=t.idx, vals=t.vals, dims=t.dims, c=np.uint32(c), modes=np.asarray(modes, np.uint32),
                        out_idx=idx, out_vals=vals)
    print(f"{name}: nnz {nnz} -> out {r['nnz']} ({os.path.getsize(path) // 1024} KiB)")


if __name__ == "__main__":
    if not oracle.ref_available():
        oracle.build()
    for n in CASES:
        make(n)
