"""The multi-GPU reporting of bench.py (one replica of the single-rank problem
per rank; the job's time is the slowest rank's, its work the sum over ranks),
run as two gloo ranks on the CPU."""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = 10.0 + 5.0 * rank  # rank 1 is slower
    m = bench.max_over_ranks(torch, ms, "cpu")
    value = bench.whole_job_tflops(bench.FLOPS, world, m)
    out.put((rank, m, value))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_report_slowest_rank_and_summed_work():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sys.path.insert(0, str(ROOT))
    import bench
    for rank, m, value in res:
        assert m == 15.0
        assert value == pytest.approx(bench.FLOPS * 2 / 0.015 / 1e12)
