"""The N > 1 path of the bench: independent replicas with one timing
reduction, run as two gloo ranks on the CPU (the reduction code is the same
one the bench runs over NCCL)."""
import datetime
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                           timeout=datetime.timedelta(seconds=60))
    from internship_b200 import replicas
    ms = 10.0 * (rank + 1)  # rank 1 is the slow one
    slow = replicas.slowest_ms(ms, dist, "cpu")
    fps = replicas.throughput(50, world, slow)
    q.put((rank, slow, fps, replicas.frame_seed(rank)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    # both ranks agree on the slowest time and on the whole-job throughput
    assert [o[1] for o in out] == [20.0, 20.0]
    assert out[0][2] == pytest.approx(2 * 50 / 0.020)
    assert out[0][2] == out[1][2]
    # every replica renders its own frames
    assert out[0][3] != out[1][3]


def test_single_process_needs_no_group():
    from internship_b200 import replicas
    assert replicas.slowest_ms(12.5) == 12.5
    assert replicas.throughput(50, 1, 250.0) == pytest.approx(200.0)
