"""Host-side helpers for running the engine on several GPUs of one node.

The contraction path has no exchange step (output rows are independent), so multi-GPU runs are
replicas: every rank contracts its own tensor on its own GPU and the job's throughput is the sum
of the ranks' work over the slowest rank's time.  Only the timing needs a collective: the
maximum of the ranks' elapsed times (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import os
import socket
import sys
from typing import List, Optional


def rank_env():
    """(rank, world_size, local_rank) from the torchrun environment (single process: 0, 1, 0)."""
    def get(name, default):
        try:
            return int(os.environ.get(name, default))
        except ValueError:
            return default
    return get("RANK", 0), get("WORLD_SIZE", 1), get("LOCAL_RANK", 0)


def init(backend: str, local_rank: int, timeout_s: int = 120):
    import datetime

    import torch
    import torch.distributed as dist
    kw = {}
    if backend == "nccl":
        kw["device_id"] = torch.device("cuda", local_rank)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)


def max_over_ranks(value: float, device: Optional[str] = None) -> float:
    """Maximum of a float over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def job_throughput(units_per_rank_step: float, steps: int, world: int, max_seconds: float) -> float:
    """Whole-job throughput of replicated work: all ranks' units over the slowest rank's time."""
    if max_seconds <= 0:
        raise ValueError("elapsed time must be positive")
    return world * steps * units_per_rank_step / max_seconds


def runs_reference_arm(rank: int) -> bool:
    """The CPU reference arm runs on rank 0 only; the other ranks exit without work."""
    return rank == 0


def needs_launcher(gpus: int) -> bool:
    """True when N > 1 GPUs were asked for but this process was not started by a launcher."""
    return gpus > 1 and "WORLD_SIZE" not in os.environ


def free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def launcher_command(script: str, argv: List[str], gpus: int, port: Optional[int] = None) -> List[str]:
    """torchrun command that starts `script argv` as `gpus` ranks on this node (one per GPU),
    rendezvous on 127.0.0.1."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
            "--master-addr=127.0.0.1", f"--master-port={port or free_port()}", script, *argv]
