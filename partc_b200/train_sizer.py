"""Train the learned sizer and evaluate it (runs on a B200).

    python -m partc_b200.train_sizer [--members 200] [--nnz-scale 1.0] [--epochs 30]

1. Training data: the exact symbolic pass (per-row output nnz) and the per-row features of 200
   seeded synthetic contractions (``gen.sizer_member``: 3-D/4-D, dims 1k-20k, nnz 100k-5M
   log-uniform, Zipf alpha in [0.8, 1.5], 1-2 contracted modes), collected through the C ABI,
   plus 200 contractions shaped like the uneven batch's members (seeds 100000+, never in the
   4096-member batch).
2. Training: the library's own CUDA forward/backward kernels with Adam (``ptc_sizer_train``).
3. Evaluation on held-out seeds of the 3-D 50k uniform workload and of the 4-D 3.1M Zipf
   workload: mean |log2(prediction / actual)| per row, the share of rows that needed an exact
   rerun on the learned path, and the learned path's time against the two-phase path's.
4. Writes the weights to partc_b200/sizer_default.bin (the library's built-in sizer) and a JSON
   report (path given by --report).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from partc_b200 import _lib, gen

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "sizer_default.bin")


# seeds of the batch-shaped training members: far from the 4096-member batch's seeds 0..4095
BATCH_TRAIN_SEED0 = 100_000


def collect(members: int, nnz_scale: float, first_seed: int = 0, batch_members: int = 0):
    """Sizer training rows: `members` contractions of gen.sizer_member, plus `batch_members`
    contractions shaped like the uneven batch's members (gen.batch_member, seeds from
    BATCH_TRAIN_SEED0), so the sizer also knows small tensors with long fibers."""
    xs, ts, info = [], [], []
    work = [("sizer", s, gen.sizer_member(s, nnz_scale=nnz_scale)) for s in range(first_seed, first_seed + members)]
    work += [("batch", s, None) for s in range(BATCH_TRAIN_SEED0, BATCH_TRAIN_SEED0 + batch_members)]
    for kind, seed, w in work:
        if w is None:
            w = gen.batch_member(seed)
        if w.tensor.nnz < 2:
            continue
        x, t = _lib.sizer_collect(w.tensor, None, w.c, w.modes)
        xs.append(x)
        ts.append(t)
        info.append({"kind": kind, "seed": seed, "nnz": w.tensor.nnz, "rows": int(len(t))})
    return np.concatenate(xs), np.concatenate(ts), info


def evaluate(sizer: _lib.Sizer, name: str, w, reps: int = 3) -> dict:
    """Prediction error and the learned path against the two-phase path on one workload."""
    x, t = _lib.sizer_collect(w.tensor, None, w.c, w.modes)
    pred = sizer.predict(x) if len(t) else np.zeros(0, np.float32)
    err = float(np.mean(np.abs(pred - t))) if len(t) else 0.0
    times = {}
    stats = {}
    for path in ("two_phase", "learned"):
        best = None
        for _ in range(reps):
            out, _, st = _lib.contract(w.tensor, None, w.c, w.modes, keep_device=True, path=path,
                                       sizer=sizer.h.value)
            _lib.free(out)
            best = st if best is None or st["t_total_ms"] < best["t_total_ms"] else best
        times[path] = best["t_total_ms"]
        stats[path] = best
    lp = stats["learned"]
    return {
        "workload": name, "rows_sized": int(len(t)),
        "mean_abs_log2_err": err,
        "median_abs_log2_err": float(np.median(np.abs(pred - t))) if len(t) else 0.0,
        "rerun_rows": int(lp["rerun_rows"]), "rerun_share": lp["rerun_rows"] / max(1, lp["rows_hash"]),
        "two_phase_ms": times["two_phase"], "learned_ms": times["learned"],
        "two_phase_symbolic_ms": stats["two_phase"]["t_symbolic_ms"],
        "learned_symbolic_ms": lp["t_symbolic_ms"],
        "speedup": times["two_phase"] / times["learned"],
    }


def evaluate_batch(sizer: _lib.Sizer, n: int) -> dict:
    """The first n members of the uneven batch (held out: never trained on) through the batched
    path, learned against two-phase."""
    work = [gen.batch_member(s) for s in range(n)]
    keep: list = []
    items = _lib.batch_items(work, keep)
    out = {"workload": f"batch members 0..{n - 1}"}
    for path in ("two_phase", "learned"):
        best = None
        for _ in range(2):
            _, st = _lib.batch_contract(items, outputs="none", path=path, sizer=sizer.h.value)
            best = st if best is None or st["t_total_ms"] < best["t_total_ms"] else best
        out[f"{path}_ms"] = best["t_total_ms"]
        if path == "learned":
            out["rerun_items"] = int(best["rerun_items"])
            out["rerun_rows"] = int(best["rerun_rows"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--members", type=int, default=200)
    ap.add_argument("--batch-members", type=int, default=200)
    ap.add_argument("--nnz-scale", type=float, default=1.0)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--report", default=None)
    args = ap.parse_args()

    t0 = time.time()
    x, t, info = collect(args.members, args.nnz_scale, batch_members=args.batch_members)
    t1 = time.time()
    s = _lib.Sizer.create(seed=2024)
    tr = s.train(x, t, epochs=args.epochs, batch=args.batch, lr=args.lr)
    t2 = time.time()
    s.save(args.out)
    # held-out seeds (the training members use other seeds and shapes)
    evals = [
        evaluate(s, "uniform3d_500x400x300_50k seed 1000", gen.uniform3d_50k(seed=1000)),
        evaluate(s, "zipf4d_2482x2862x14036x17_3.1m seed 1001", gen.zipf4d_3m(seed=1001)),
        evaluate(s, "zipf4d_2482x2862x14036x17_3.1m seed 1", gen.zipf4d_3m(seed=1)),
    ]
    evals.append(evaluate_batch(s, 64))
    report = {
        "members": args.members, "batch_members": args.batch_members, "nnz_scale": args.nnz_scale,
        "samples": int(len(t)),
        "collect_s": t1 - t0, "train": tr, "train_s": t2 - t1, "weights": os.path.basename(args.out),
        "train_mean_abs_log2_err": float(np.mean(np.abs(s.predict(x) - t))),
        "eval": evals,
    }
    text = json.dumps(report, indent=1)
    print(text)
    if args.report:
        with open(args.report, "w") as f:
            f.write(text + "\n")


if __name__ == "__main__":
    main()
