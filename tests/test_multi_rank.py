"""The multi-GPU host logic on CPU: two gloo ranks, max-over-ranks timing, replica throughput."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from partc_b200 import dist as pdist


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    r, w, lr = pdist.rank_env()
    pdist.init("gloo", lr, timeout_s=60)
    elapsed = 1.0 + rank  # rank 1 is the slow one
    pdist.barrier()
    m = pdist.max_over_ranks(elapsed)
    value = pdist.job_throughput(100.0, 5, w, m)
    q.put((r, w, m, value, pdist.runs_reference_arm(r)))
    dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=10) for _ in range(2))
    for r, w, m, value, ref in res:
        assert w == 2 and m == 2.0
        assert value == pytest.approx(2 * 5 * 100.0 / 2.0)
        assert ref == (r == 0)


def test_single_process_defaults(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert pdist.rank_env() == (0, 1, 0)
    assert pdist.max_over_ranks(3.5) == 3.5
    with pytest.raises(ValueError):
        pdist.job_throughput(1, 1, 1, 0.0)


def test_launcher_command(monkeypatch):
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    assert pdist.needs_launcher(4) and not pdist.needs_launcher(1)
    monkeypatch.setenv("WORLD_SIZE", "4")
    assert not pdist.needs_launcher(4)
    cmd = pdist.launcher_command("bench.py", ["--gpus", "4", "--steps", "2"], 4, port=29511)
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and "--master-addr=127.0.0.1" in cmd and "--master-port=29511" in cmd
    assert cmd[-5:] == ["bench.py", "--gpus", "4", "--steps", "2"]
