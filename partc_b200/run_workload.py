"""Run one named workload through ptc_contract a few times and print each call's statistics.

    python -m partc_b200.run_workload --workload zipf4d_3m --path learned --reps 3

The tensor (``partc_b200/gen.py``) goes to the device first; the output stays on the device and is
released after each call.  Meant for profiler captures and quick timings of one configuration
(``bench.py`` is the benchmark proper).
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="zipf4d_500k")
    ap.add_argument("--path", default="two_phase", choices=["two_phase", "learned"])
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--large-rows", default="auto", choices=["auto", "bitmap", "panels"])
    ap.add_argument("--bitmap-max-len", type=int, default=0)
    ap.add_argument("--panel-width", type=int, default=0)
    ap.add_argument("--warp-task-max-len", type=int, default=0)
    ap.add_argument("--hash-load-pct", type=int, default=0)
    a = ap.parse_args(argv)
    import torch
    from partc_b200 import _lib, gen
    w = gen.WORKLOADS[a.workload]()
    t = w.tensor
    di = torch.from_numpy(t.idx.view(np.int32)).cuda()
    dv = torch.from_numpy(t.vals).cuda()
    keep = []
    coo = _lib.device_coo(di.data_ptr(), dv.data_ptr(), t.nnz, t.dims, keep)
    s = torch.cuda.Stream()
    opts = dict(output_location="device", device=torch.cuda.current_device(), stream=s.cuda_stream, path=a.path,
                large_rows=a.large_rows, bitmap_max_len=a.bitmap_max_len, panel_width=a.panel_width,
                warp_task_max_len=a.warp_task_max_len, hash_load_pct=a.hash_load_pct)
    keys = ("t_build_ms", "t_symbolic_ms", "t_numeric_ms", "t_total_ms", "out_nnz", "mult_adds", "rerun_rows",
            "sizer_mean_abs_log2_err", "rows_hash", "hash_parts", "panel_width", "kernel_launches")
    for _ in range(a.reps):
        out, st = _lib.contract_coo(coo, None, w.c, w.modes, **opts)
        print(json.dumps({k: (round(st[k], 3) if isinstance(st[k], float) else st[k]) for k in keys}), flush=True)
        _lib.free(out)
    torch.cuda.synchronize()


if __name__ == "__main__":
    main()
