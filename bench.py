"""Benchmark of the B200 contraction engine on the 4-D 3.1M-nnz workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--path two_phase|learned]

One step = one full contraction (keys, sorts, cuckoo table, symbolic or sizer pass, numeric pass,
output in HBM) of the seeded synthetic tensor 2482x2862x14036x17 with 3.1M nonzeros, per-mode
Zipf(1.1) indices, U(0,1) values, contracted over modes {0,1} (2.87e9 mult-adds, 1.70e9 output
nonzeros).  Under torchrun every rank contracts its own replica on its own GPU (the path has no
exchange step), so the job scales weakly; rank 0 prints one JSON line.

``value``  = mult-adds of all ranks / max-over-ranks device time (CUDA events on the stream the
             library runs on), inputs already resident in HBM.
``e2e``    = the same metric through the C ABI with host buffers: pinned host inputs copied in and
             the 1.7e9-entry output copied back into host memory inside the timed region.
``roofline``: the numeric pass (hash accumulators + output writes), algorithmic bytes
             12*nnz_A + 12*mult_adds + (4*order_out + 8)*nnz_out per step over its event time.
``cpu_baseline`` / ``--impl reference``: the reference's own fksCuckooTC path (compiled from its
             sources into oracle/_ref) on the host cores, on a bounded sample of A's rows against
             the whole B; with no compiled reference, the oracle's C restatement.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "zipf4d_3m"
FALLBACK_HBM_GBS = 6650.0
TUNE_SEED = 1001    # the autotuner's held-out tensor: the timed workload drawn with this seed
L2_BYTES = 126 << 20     # B200 L2
L2_FLUSH_BYTES = 512 << 20  # written before a step whose data would otherwise stay in L2
CPU_WARMUP = 1      # reference runs before the timed ones (both CPU legs)
CPU_STEPS = 3       # timed reference runs of the cpu_baseline leg (median)


class ClockSampler:
    """nvidia-smi SM clock / throttle-reason samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for n, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def host_info():
    """The host's core count, CPU model and memory (for the CPU baselines)."""
    info = {"nproc": os.cpu_count(), "cpu_model": None, "ram_gb": None}
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    info["cpu_model"] = line.split(":", 1)[1].strip()
                    break
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemTotal"):
                    info["ram_gb"] = round(int(line.split()[1]) / 1024 ** 2, 1)
                    break
    except OSError:
        pass
    return info


def numeric_kernels(st):
    """The kernels of the numeric pass a call ran (large rows on the row bitmap kernel report
    panel width 0 and no parts)."""
    if st["rows_hash"] > 0 and st["panel_width"] == 0 and st["hash_parts"] == 0:
        large = "rowmap_kernel (one block per large row, column bitmap in shared memory)"
    else:
        large = "warp_task_kernel + hash_part_kernel (panel parts)"
    return f"numeric pass: {large} + small_rows_kernel + copy_rows_kernel + esc_fold_kernel"


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_from_profile(workload: str):
    """Per-launch DRAM bytes of the numeric pass from the committed ncu summary of this workload,
    if there is one (profiles/numeric_traffic.json names the workload it was scaled to)."""
    p = os.path.join(ROOT, "profiles", "numeric_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
    except Exception:
        return None
    return d if d.get("workload") == workload else None


# ---------------------------------------------------------------------------------------------
# reference arm (CPU)
# ---------------------------------------------------------------------------------------------

def _row_sample(w, target_flops: int, seed: int = 0):
    """Keep mask over A's nonzeros selecting whole rows whose mult-adds sum to about target."""
    import oracle
    t = w.tensor
    stats = oracle.contract(t, None, w.c, w.modes, mode=oracle.FLOPS_ONLY)
    rng = np.random.default_rng(seed)
    order = rng.permutation(stats["nrows"])
    flops = stats["row_flops"][order].astype(np.int64)
    take = order[: max(1, int(np.searchsorted(np.cumsum(flops), target_flops)) + 1)]
    keys = np.sort(stats["row_key"][take])
    free = w.modes[w.c:]
    dims = t.dims.astype(np.uint64)
    fkey = np.zeros(t.nnz, dtype=np.uint64)
    for m in free:
        fkey = fkey * dims[m] + t.idx[:, m].astype(np.uint64)
    keep = np.isin(fkey, keys)
    sample_flops = int(stats["row_flops"][take].astype(np.int64).sum())
    return keep, sample_flops, len(take)


def run_reference_once(w, keep, tmpdir):
    """One run of the reference path on the sample; returns its timing dict."""
    import oracle
    inp = os.path.join(tmpdir, "in.bin")
    kp = os.path.join(tmpdir, "keep.bin")
    if not os.path.exists(inp):
        oracle.write_ref_input(inp, w.tensor, w.c, w.modes)
        keep.astype(np.uint8).tofile(kp)
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
    r = subprocess.run([oracle.REF_BIN, inp, kp], capture_output=True, text=True, env=env, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"reference run failed: {r.stderr[-400:]}")
    return json.loads(r.stdout.strip().splitlines()[-1])


def run_port_once(w, keep):
    import oracle
    sub = type(w.tensor)(idx=w.tensor.idx[keep], vals=w.tensor.vals[keep], dims=w.tensor.dims)
    t0 = time.perf_counter()
    o = oracle.contract(sub, w.tensor, w.c, w.modes, w.modes, mode=oracle.VALUES)
    t1 = time.perf_counter()
    return {"t_wall": t1 - t0, "out_nnz": o["nnz"]}


def cpu_arm(w, target_flops, steps, warmup):
    """Times the reference (or the port) on a row sample; returns (value, cpu_baseline dict).

    The sample is seeded (the same rows for the reference arm and the cpu_baseline leg of the GPU
    arm).  value = the sample's mult-adds over the median time of the reference's whole path
    (HT_B and HT_A builds over the whole B and the sampled rows, preprocessing, numeric pass);
    numeric_only = the same mult-adds over the median of the reference's own "Total time for
    tensor contraction" line (fksCuckooTC.hpp:362-365), which excludes the builds that do not
    shrink with the sample."""
    import oracle
    keep, sflops, nrows = _row_sample(w, target_flops)
    kind = "reference" if os.path.exists(oracle.REF_BIN) else "port"
    times, numeric = [], []
    with tempfile.TemporaryDirectory() as td:
        for i in range(warmup + steps):
            if kind == "reference":
                r = run_reference_once(w, keep, td)
            else:
                r = run_port_once(w, keep)
            if i >= warmup:
                times.append(r["t_wall"])
                if r.get("t_contract"):
                    numeric.append(r["t_contract"])
    t = statistics.median(times)
    value = sflops / t
    # the reference is offered every host core (OMP_NUM_THREADS), but its hash builds are serial
    # loops and its numeric loop runs a team of one (fksCuckooTC.hpp:171-173): one core works
    cores = 1
    sample = (f"{nrows} of A's rows (whole rows, seeded) against the whole B: {sflops} mult-adds "
              f"({100.0 * sflops / max(1, w_flops(w)):.2f}% of the workload's); time = the reference's HT_B + "
              f"HT_A builds, preprocessing and numeric pass; median of {len(times)} after {warmup} warm-up; "
              f"OMP_NUM_THREADS={os.cpu_count()} offered, the reference's loops use one thread "
              f"(fksCuckooTC.hpp:171-173)")
    out = {"value": value, "unit": "mult-adds/s", "cores": cores, "kind": kind, "sample": sample,
           "sample_mult_adds": sflops, "seconds": t, "host": host_info()}
    if numeric:
        out["numeric_only"] = {"value": sflops / statistics.median(numeric), "unit": "mult-adds/s",
                               "seconds": statistics.median(numeric)}
    return value, out


_FLOPS_CACHE = {}


def w_flops(w):
    """Mult-adds of the whole workload (the oracle's flop count, cached)."""
    import oracle
    if w.name not in _FLOPS_CACHE:
        _FLOPS_CACHE[w.name] = int(oracle.contract(w.tensor, None, w.c, w.modes, mode=oracle.FLOPS_ONLY)["flops"])
    return _FLOPS_CACHE[w.name]


def cpu_arm_batch(n_items, target_seconds, steps, warmup):
    """The reference path on whole members of the uneven batch (seed order, every member whose
    products the reference finishes quickly), until about target_seconds of work per step."""
    import oracle
    from partc_b200 import gen
    kind = "reference" if os.path.exists(oracle.REF_BIN) else "port"
    members = []
    for seed in range(n_items):
        w = gen.batch_member(seed)
        if w.tensor.nnz > 1:
            members.append(w)
        if len(members) >= 64:
            break
    rates = []
    used = 0
    with tempfile.TemporaryDirectory() as td:
        for rep in range(warmup + steps):
            fl, sec = 0, 0.0
            for i, w in enumerate(members):
                st = oracle.contract(w.tensor, None, w.c, w.modes, mode=oracle.FLOPS_ONLY)
                if st["flops"] == 0 or st["flops"] > 2e8:
                    continue
                sub = os.path.join(td, f"m{i}")
                os.makedirs(sub, exist_ok=True)
                keep = np.ones(w.tensor.nnz, dtype=bool)
                r = run_reference_once(w, keep, sub) if kind == "reference" else run_port_once(w, keep)
                fl += st["flops"]
                sec += r["t_wall"]
                used = i + 1
                if sec > target_seconds:
                    break
            if rep >= warmup:
                rates.append(fl / sec)
    value = statistics.median(rates)
    sample = (f"whole members of the uneven batch in seed order (the first {used} seeds, members above 2e8 "
              f"mult-adds skipped), about {target_seconds:.0f} s of reference time per step; the reference's "
              f"loops use one thread (fksCuckooTC.hpp:171-173)")
    return value, {"value": value, "unit": "mult-adds/s", "cores": 1, "kind": kind, "sample": sample,
                   "seconds": target_seconds}


# ---------------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------------

def matricized_cusparse(w, dev, M):
    """The reference's other baseline, matricize then SpGEMM (matricizedspGEMM.hpp:172-603), on
    the GPU: A as a CSR matrix (rows = A's free keys, columns = contracted keys) times its
    transpose-shaped B, through torch's CSR x CSR product (cuSPARSE SpGEMM), float64.  Timed with
    CUDA events around the product only; a comparison point, not this library's path."""
    import torch
    t = w.tensor
    dims = t.dims.astype(np.int64)
    con, free = w.modes[:w.c], w.modes[w.c:]
    ck = np.zeros(t.nnz, np.int64)
    fk = np.zeros(t.nnz, np.int64)
    for m in con:
        ck = ck * dims[m] + t.idx[:, m]
    for m in free:
        fk = fk * dims[m] + t.idx[:, m]
    _, ci = np.unique(ck, return_inverse=True)
    _, fi = np.unique(fk, return_inverse=True)
    nr, nc = int(fi.max()) + 1, int(ci.max()) + 1
    try:
        a = torch.sparse_coo_tensor(torch.from_numpy(np.stack([fi, ci])), torch.from_numpy(t.vals), (nr, nc),
                                    device=dev).coalesce().to_sparse_csr()
        b = torch.sparse_coo_tensor(torch.from_numpy(np.stack([ci, fi])), torch.from_numpy(t.vals), (nc, nr),
                                    device=dev).coalesce().to_sparse_csr()
        c = torch.sparse.mm(a, b)  # warm-up
        nnz = int(c._nnz())
        del c
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        c = torch.sparse.mm(a, b)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        del a, b, c
        torch.cuda.empty_cache()
        return {"value": M / (ms * 1e-3), "unit": "mult-adds/s", "ms": ms, "out_nnz": nnz,
                "what": "torch CSR x CSR (cuSPARSE SpGEMM), f64, product only"}
    except Exception as ex:  # e.g. the product's workspace does not fit the device
        torch.cuda.empty_cache()
        return {"value": None, "error": str(ex)[:200]}


def run_batch(args, rank, world, local):
    """One step = ptc_batch_contract over the uneven batch (members 0..n-1 of gen.batch_member),
    inputs resident in HBM, outputs produced wave by wave and discarded; beside it the same members
    contracted one ptc_contract call each (two-phase, outputs freed)."""
    import torch
    from partc_b200 import _lib, gen
    from partc_b200 import dist as pdist
    n = args.batch_items
    work = gen.batch_members(n, procs=min(16, os.cpu_count() or 1))
    dev = f"cuda:{local}"
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    idx_cat = np.concatenate([w.tensor.idx.reshape(-1) for w in work]).view(np.int32)
    val_cat = np.concatenate([w.tensor.vals for w in work])
    di = torch.from_numpy(idx_cat).to(dev)
    dv = torch.from_numpy(val_cat).to(dev)
    keep = []

    def make_items(ibase, vbase, loc):
        items = (_lib.BatchItem * n)()
        io = vo = 0
        for i, w in enumerate(work):
            t = w.tensor
            d = np.ascontiguousarray(t.dims, dtype=np.uint32)
            keep.append(d)
            items[i].A = _lib.Coo(t.order, loc, t.nnz, ibase + 4 * io, vbase + 8 * vo, d.ctypes.data)
            items[i].c = w.c
            for j, m in enumerate(w.modes):
                items[i].a_modes[j] = m
            io += t.nnz * t.order
            vo += t.nnz
        return items

    items = make_items(di.data_ptr(), dv.data_ptr(), _lib.PTC_DEVICE)
    path = args.batch_path
    opts = dict(device=local, stream=stream.cuda_stream, path=path)
    sizes = {}

    def sink(i, t):
        sizes[i] = (t.nnz, t.order)

    _, st0 = _lib.batch_contract(items, outputs="sink", sink=sink, output_location="device", **opts)
    M, R = st0["mult_adds"], st0["out_nnz"]
    out_bytes = sum(k * (4 * o + 8) for k, o in sizes.values())
    for _ in range(max(0, args.warmup - 1)):
        _lib.batch_contract(items, outputs="none", **opts)
    torch.cuda.synchronize()
    pdist.barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    stats = []
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            stats.append(_lib.batch_contract(items, outputs="none", **opts)[1])
        ev1.record(stream)
        torch.cuda.synchronize()
    pdist.barrier()
    ms = pdist.max_over_ranks(ev0.elapsed_time(ev1), device=dev)
    value = pdist.job_throughput(M, args.steps, world, ms * 1e-3)
    na = int(sum(w.tensor.nnz for w in work))
    # the other path on the same batch, timed the same way
    paths = {path: {"value": value, "ms_per_step": ms / args.steps, "rerun_items": int(stats[0]["rerun_items"])}}
    if args.compare_paths:
        other = "learned" if path == "two_phase" else "two_phase"
        oo = dict(opts, path=other)
        _lib.batch_contract(items, outputs="none", **oo)
        torch.cuda.synchronize()
        ost = []
        ev0.record(stream)
        for _ in range(args.steps):
            ost.append(_lib.batch_contract(items, outputs="none", **oo)[1])
        ev1.record(stream)
        torch.cuda.synchronize()
        oms = pdist.max_over_ranks(ev0.elapsed_time(ev1), device=dev)
        paths[other] = {"value": pdist.job_throughput(M, args.steps, world, oms * 1e-3),
                        "ms_per_step": oms / args.steps, "rerun_items": int(ost[0]["rerun_items"])}
    alg = 12 * na + 12 * M + out_bytes
    t_num = statistics.mean(s["t_numeric_ms"] for s in stats) * 1e-3
    peak, peak_kind = measured_hbm_peak()
    roofline = {"bound": "hbm", "achieved": alg / t_num / 1e9, "peak": peak, "unit": "GB/s",
                "frac": alg / t_num / 1e9 / peak, "peak_source": peak_kind,
                "kernel": "numeric pass of every wave (graph launches)", "algorithmic_bytes": alg,
                "numeric_ms": t_num * 1e3, "traffic": None}

    # the same members, one ptc_contract call each (two-phase path, device outputs freed)
    loop = None
    if args.per_contraction:
        ev2 = torch.cuda.Event(enable_timing=True)
        ev3 = torch.cuda.Event(enable_timing=True)
        popts = dict(output_location="device", device=local, stream=stream.cuda_stream, path="two_phase")
        ev2.record(stream)
        fl = 0
        for i in range(n):
            try:
                out, st = _lib.contract_coo(items[i].A, None, items[i].c, list(items[i].a_modes)[:items[i].A.order],
                                            **popts)
                _lib.free(out)
                fl += st["mult_adds"]
            except _lib.PtcError:
                pass  # an item with no matching fiber or at most one nonzero: an error for a single call
        ev3.record(stream)
        torch.cuda.synchronize()
        lms = ev2.elapsed_time(ev3)
        loop = {"value": fl / (lms * 1e-3), "unit": "mult-adds/s", "ms": lms, "mult_adds": fl,
                "calls": n, "path": "two_phase"}

    # end to end: host inputs through the C ABI, per-item output counts read back
    e2e = None
    if args.e2e_steps > 0:
        pi = torch.from_numpy(idx_cat).pin_memory()
        pv = torch.from_numpy(val_cat).pin_memory()
        hitems = make_items(pi.data_ptr(), pv.data_ptr(), _lib.PTC_HOST)
        pdist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            _lib.batch_contract(hitems, outputs="none", device=local, stream=stream.cuda_stream, path=path)
        el = pdist.max_over_ranks(time.perf_counter() - t0, device=dev)
        e2e = {"value": pdist.job_throughput(M, args.e2e_steps, world, el), "unit": "mult-adds/s",
               "h2d_bytes_per_step": int(idx_cat.nbytes + val_cat.nbytes), "d2h_bytes_per_step": 8 * n,
               "note": "outputs stay in device waves (the library's sink interface); per-item counts come back",
               "steps": args.e2e_steps, "ms_per_step": el / args.e2e_steps * 1e3}
    if rank == 0:
        line = {
            "metric": "contraction mult-adds/s", "value": value, "unit": "mult-adds/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator partc_b200/gen.py batch_member, seeds 0..n-1)",
            "config": {"workload": f"batch{n}", "items": n, "nnz": na, "path": path,
                       "parallelism": f"replicas x{world}", "mult_adds_per_step": M, "out_nnz_per_step": R,
                       "l2": "no flush needed: each step writes its outputs (>> 126 MB L2)"},
            "phase_ms": {k: statistics.mean(s[k] for s in stats) for k in
                         ("t_build_ms", "t_symbolic_ms", "t_numeric_ms", "t_d2h_ms", "t_total_ms")},
            "batch_waves": stats[0]["batch_waves"], "rerun_items": stats[0]["rerun_items"],
            "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
            "roofline": roofline, "per_contraction": loop, "paths": paths, "e2e": e2e, "cpu_baseline": None,
            "clocks": clk.summary(),
        }
        print(json.dumps(line))


def batch_record(n, local, stream, steps, warmup=1):
    """The first n members of the uneven batch (gen.batch_member seeds 0..n-1) through
    ptc_batch_contract on both paths, inputs resident in HBM, outputs produced wave by wave and
    discarded; CUDA events on the library's stream.  A record for the default bench line."""
    import torch
    from partc_b200 import _lib, gen
    work = gen.batch_members(n, procs=min(16, os.cpu_count() or 1))
    dev = f"cuda:{local}"
    idx_cat = np.concatenate([w.tensor.idx.reshape(-1) for w in work]).view(np.int32)
    val_cat = np.concatenate([w.tensor.vals for w in work])
    di = torch.from_numpy(idx_cat).to(dev)
    dv = torch.from_numpy(val_cat).to(dev)
    keep = []
    items = (_lib.BatchItem * n)()
    io = vo = 0
    for i, w in enumerate(work):
        t = w.tensor
        items[i].A = _lib.device_coo(di.data_ptr() + 4 * io, dv.data_ptr() + 8 * vo, t.nnz, t.dims, keep)
        items[i].c = w.c
        for j, m in enumerate(w.modes):
            items[i].a_modes[j] = m
        io += t.nnz * t.order
        vo += t.nnz
    rec = {"items": n, "nnz": int(vo), "seeds": f"0..{n - 1}"}
    for path in ("two_phase", "learned"):
        opts = dict(device=local, stream=stream.cuda_stream, path=path)
        for _ in range(warmup):
            _, st = _lib.batch_contract(items, outputs="none", **opts)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        sts = []
        e0.record(stream)
        for _ in range(steps):
            sts.append(_lib.batch_contract(items, outputs="none", **opts)[1])
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        M = sts[0]["mult_adds"]
        rec[path] = {"value": M / (ms * 1e-3), "unit": "mult-adds/s", "ms_per_step": ms, "mult_adds": M,
                     "out_nnz": sts[0]["out_nnz"], "rerun_items": int(sts[0]["rerun_items"]),
                     "t_symbolic_ms": statistics.mean(x["t_symbolic_ms"] for x in sts),
                     "t_numeric_ms": statistics.mean(x["t_numeric_ms"] for x in sts),
                     "launches_per_step": int(sts[0]["kernel_launches"])}
    rec["learned_over_two_phase"] = rec["learned"]["value"] / rec["two_phase"]["value"]
    del di, dv
    torch.cuda.empty_cache()
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--path", default="learned", choices=["two_phase", "learned"])
    ap.add_argument("--no-compare-paths", dest="compare_paths", action="store_false")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false")
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-target-flops", type=float, default=6e7)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-items", type=int, default=4096)
    ap.add_argument("--batch-path", default="two_phase", choices=["two_phase", "learned"])
    ap.add_argument("--no-cusparse", dest="cusparse", action="store_false")
    ap.add_argument("--no-per-contraction", dest="per_contraction", action="store_false")
    ap.add_argument("--batch-record", type=int, default=256,
                    help="members of the uneven batch timed on both paths for the default line (0: none)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    from partc_b200 import dist as pdist
    if pdist.needs_launcher(args.gpus):
        # one replica rank per GPU: start this script again under the launcher
        sys.exit(subprocess.call(pdist.launcher_command(os.path.abspath(__file__), sys.argv[1:], args.gpus)))
    rank, world, local = pdist.rank_env()

    if args.workload.startswith("batch") and args.impl == "ours":
        if world > 1:
            pdist.init("nccl", local)
        run_batch(args, rank, world, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    from partc_b200 import gen
    w = None if args.workload.startswith("batch") else gen.WORKLOADS[args.workload]()
    t = w.tensor if w is not None else None

    if args.impl == "reference" and args.workload.startswith("batch"):
        if not pdist.runs_reference_arm(rank):
            return
        steps = max(1, args.steps)
        value, cb = cpu_arm_batch(args.batch_items, 10.0, steps, min(args.warmup, 1))
        line = {"impl": "reference", "metric": "contraction mult-adds/s", "value": value, "unit": "mult-adds/s",
                "n_gpus": args.gpus, "steps": steps, "warmup": min(args.warmup, 1), "ms_per_step": None,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generator partc_b200/gen.py batch_member)",
                "config": {"workload": f"batch{args.batch_items}", "parallelism": "host cores"},
                "cpu_baseline": {k: cb[k] for k in ("kind", "cores", "sample", "value")},
                "e2e": {"value": value, "unit": "mult-adds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if args.impl == "reference":
        if not pdist.runs_reference_arm(rank):
            return
        steps = max(1, args.steps)
        value, cb = cpu_arm(w, int(args.cpu_target_flops), steps, CPU_WARMUP)
        line = {"impl": "reference", "metric": "contraction mult-adds/s", "value": value, "unit": "mult-adds/s",
                "n_gpus": args.gpus, "steps": steps, "warmup": CPU_WARMUP, "ms_per_step": cb["seconds"] * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generator, partc_b200/gen.py)",
                "config": {"workload": w.name, "nnz": t.nnz, "dims": [int(x) for x in t.dims], "contracted_modes":
                           w.modes[:w.c], "parallelism": "host cores"},
                "cpu_baseline": {k: cb[k] for k in ("kind", "cores", "sample", "value", "numeric_only", "host")
                                 if k in cb},
                "e2e": {"value": value, "unit": "mult-adds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    import torch.distributed as dist
    from partc_b200 import _lib

    torch.cuda.set_device(local)
    if world > 1:
        pdist.init("nccl", local)

    stream = torch.cuda.Stream()
    di = torch.from_numpy(t.idx.view(np.int32)).to(f"cuda:{local}")
    dv = torch.from_numpy(t.vals).to(f"cuda:{local}")
    keep = []
    coo = _lib.device_coo(di.data_ptr(), dv.data_ptr(), t.nnz, t.dims, keep)
    opts = dict(output_location="device", device=local, stream=stream.cuda_stream, path=args.path)
    tuned = {args.path: {}}
    other = "two_phase" if args.path == "learned" else "learned"
    if args.autotune:
        # the library's autotuner picks each path's knobs (untimed) on a held-out tensor: the same
        # workload drawn with another seed, never the tensor that is timed
        wt = gen.WORKLOADS[args.workload](seed=TUNE_SEED)
        ti = torch.from_numpy(wt.tensor.idx.view(np.int32)).to(f"cuda:{local}")
        tv = torch.from_numpy(wt.tensor.vals).to(f"cuda:{local}")
        items = (_lib.BatchItem * 1)()
        items[0].A = _lib.device_coo(ti.data_ptr(), tv.data_ptr(), wt.tensor.nnz, wt.tensor.dims, keep)
        items[0].c = wt.c
        for j, m in enumerate(wt.modes):
            items[0].a_modes[j] = m
        for p in ([args.path, other] if args.compare_paths else [args.path]):
            kn, _ = _lib.autotune(items, repeats=1, device=local, stream=stream.cuda_stream, path=p)
            tuned[p] = {k: v for k, v in kn.items() if v}
        del ti, tv, items
        torch.cuda.empty_cache()
    knobs = tuned[args.path]
    opts.update(knobs)

    def step():
        out, st = _lib.contract_coo(coo, None, w.c, w.modes, **opts)
        _lib.free(out)
        return st

    for _ in range(args.warmup):
        st0 = step()
    torch.cuda.synchronize()
    pdist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    # a step that touches less than 4x the L2 (inputs + output) gets the L2 flushed before it,
    # outside its timed span: each step is timed on its own and the spans are summed
    touched = t.nnz * (4 * t.order + 8) + st0["out_nnz"] * (4 * 2 * (t.order - w.c) + 8)
    flush = touched < 4 * L2_BYTES
    l2_note = (f"L2 flushed before every step ({L2_FLUSH_BYTES >> 20} MiB written, untimed): a step touches "
               f"{touched / 1e6:.0f} MB" if flush else
               f"no flush needed: a step touches {touched / 1e9:.2f} GB (inputs + output, >> 126 MB L2)")
    scrub = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{local}") if flush else None
    stats = []
    with ClockSampler(local) as clk:
        if not flush:
            ev0.record(stream)
            for _ in range(args.steps):
                stats.append(step())
            ev1.record(stream)
            torch.cuda.synchronize()
            span = ev0.elapsed_time(ev1)
        else:
            span = 0.0
            for _ in range(args.steps):
                with torch.cuda.stream(stream):
                    scrub.fill_(1)
                ev0.record(stream)
                stats.append(step())
                ev1.record(stream)
                torch.cuda.synchronize()
                span += ev0.elapsed_time(ev1)
    pdist.barrier()
    torch.cuda.synchronize()
    ms = pdist.max_over_ranks(span, device=f"cuda:{local}")
    M = stats[0]["mult_adds"]
    R = stats[0]["out_nnz"]
    value = pdist.job_throughput(M, args.steps, world, ms * 1e-3)
    ms_step = ms / args.steps

    # the other path, timed the same way (learned-sized against exact two-phase sizing), with the
    # knobs tuned for it
    paths = {args.path: {"value": value, "ms_per_step": ms_step,
                         "t_symbolic_ms": statistics.mean(s["t_symbolic_ms"] for s in stats),
                         "rerun_rows": int(stats[0]["rerun_rows"]),
                         "sizer_mean_abs_log2_err": stats[0]["sizer_mean_abs_log2_err"]}}
    if args.compare_paths:
        oopts = dict(output_location="device", device=local, stream=stream.cuda_stream, path=other,
                     **tuned.get(other, {}))
        for _ in range(2):
            out, _ = _lib.contract_coo(coo, None, w.c, w.modes, **oopts)
            _lib.free(out)
        torch.cuda.synchronize()
        pdist.barrier()
        ost = []
        ev0.record(stream)
        for _ in range(args.steps):
            out, st = _lib.contract_coo(coo, None, w.c, w.modes, **oopts)
            _lib.free(out)
            ost.append(st)
        ev1.record(stream)
        torch.cuda.synchronize()
        oms = pdist.max_over_ranks(ev0.elapsed_time(ev1), device=f"cuda:{local}")
        paths[other] = {"value": pdist.job_throughput(M, args.steps, world, oms * 1e-3),
                        "ms_per_step": oms / args.steps,
                        "t_symbolic_ms": statistics.mean(s["t_symbolic_ms"] for s in ost),
                        "rerun_rows": int(ost[0]["rerun_rows"]),
                        "sizer_mean_abs_log2_err": ost[0]["sizer_mean_abs_log2_err"],
                        "knobs": tuned.get(other) or "defaults"}

    # numeric pass roofline
    od = 2 * (t.order - w.c)
    alg_bytes = 12 * t.nnz + 12 * M + (4 * od + 8) * R
    t_num = statistics.mean(s["t_numeric_ms"] for s in stats) * 1e-3
    achieved = alg_bytes / t_num / 1e9
    peak, peak_kind = measured_hbm_peak()
    traffic = traffic_from_profile(args.workload)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind,
                "kernel": numeric_kernels(stats[0]),
                "algorithmic_bytes": alg_bytes, "numeric_ms": t_num * 1e3,
                "traffic": traffic.get("bytes_per_launch") if traffic else None}

    # end to end through the C ABI with host buffers
    e2e = None
    if args.e2e_steps > 0:
        from partc_b200.gen import CooTensor
        pi = torch.from_numpy(t.idx.view(np.int32)).pin_memory()
        pv = torch.from_numpy(t.vals).pin_memory()
        ht = CooTensor(idx=pi.numpy().view(np.uint32), vals=pv.numpy(), dims=t.dims)
        e2e_opts = dict(device=local, stream=stream.cuda_stream, path=args.path, **knobs)
        idx, vals, _ = _lib.contract(ht, None, w.c, w.modes, **e2e_opts)  # warm-up
        del idx, vals
        pdist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            idx, vals, _ = _lib.contract(ht, None, w.c, w.modes, **e2e_opts)
            del idx, vals
        el = pdist.max_over_ranks(time.perf_counter() - t0, device=f"cuda:{local}")
        e2e = {"value": pdist.job_throughput(M, args.e2e_steps, world, el), "unit": "mult-adds/s",
               "h2d_bytes_per_step": t.nnz * (4 * t.order + 8), "d2h_bytes_per_step": R * (4 * od + 8),
               "steps": args.e2e_steps, "ms_per_step": el / args.e2e_steps * 1e3}

    cusparse = matricized_cusparse(w, f"cuda:{local}", M) if (args.cusparse and rank == 0 and world == 1) else None
    batch = None
    if args.batch_record > 0 and rank == 0 and world == 1:
        batch = batch_record(args.batch_record, local, stream, steps=3)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            _, cpu = cpu_arm(w, int(args.cpu_target_flops), CPU_STEPS, CPU_WARMUP)
        except Exception as ex:  # reported, never fatal to the GPU number
            cpu = {"value": None, "error": str(ex)[:200]}

    if rank == 0:
        line = {
            "metric": "contraction mult-adds/s", "value": value, "unit": "mult-adds/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": f"synthetic (seeded generator partc_b200/gen.py, {args.workload}: {gen.describe(args.workload)})",
            "config": {"workload": w.name, "nnz": t.nnz, "dims": [int(x) for x in t.dims],
                       "contracted_modes": w.modes[:w.c], "path": args.path, "parallelism": f"replicas x{world}",
                       "knobs": knobs or "defaults",
                       "mult_adds_per_step": M, "out_nnz_per_step": R,
                       "l2": l2_note},
            "hbm_gbs_numeric": achieved,
            "phase_ms": {k: statistics.mean(s[k] for s in stats) for k in
                         ("t_build_ms", "t_symbolic_ms", "t_numeric_ms", "t_total_ms")},
            "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
            "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu, "clocks": clk.summary(),
            "matricized_cusparse": cusparse, "paths": paths, f"batch{args.batch_record}": batch,
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
