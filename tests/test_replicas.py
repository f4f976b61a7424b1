"""Multi-rank bookkeeping of bench.py on CPU: two gloo ranks (world size 2)
take the same barrier/all-reduce steps and agree on the whole-job rate."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    sys.path.insert(0, os.path.join(ROOT, "topopt-slp-3d_b200"))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from tosp import replicas
    replicas.barrier()
    # rank r processed 5 solves in (r + 1) seconds; the job rate uses the slowest
    rate, t = replicas.job_rate(5, float(rank + 1))
    out.put((rank, rate, t))
    replicas.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[0] for r in res] == [0, 1]
    for _, rate, t in res:
        assert t == pytest.approx(2.0)
        assert rate == pytest.approx(2 * 5 / 2.0)


def test_single_process_is_identity():
    sys.path.insert(0, os.path.join(ROOT, "topopt-slp-3d_b200"))
    from tosp import replicas
    assert replicas.world() == (1, 0)
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.job_rate(4, 2.0) == (2.0, 2.0)
