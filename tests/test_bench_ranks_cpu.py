"""bench.py's multi-rank host logic on CPU, two gloo ranks on 127.0.0.1.
The ranks are replicas that share no data: the only cross-rank step is the
max over ranks of the timed region's device time, and in the reference arm
only rank 0 works and prints."""
import argparse
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    from datetime import timedelta

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    got = [bench.slowest_rank_ms(10.0 + 5.0 * rank, world, "cpu"),
           bench.slowest_rank_ms(3.0 - rank, world, "cpu")]
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, got))


def test_slowest_rank_time_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(out.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: [15.0, 3.0], 1: [15.0, 3.0]}


def test_single_rank_time_is_its_own():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.slowest_rank_ms(12.5, 1, "cpu") == 12.5


def test_reference_arm_other_ranks_do_no_work(capsys):
    sys.path.insert(0, ROOT)
    import bench

    args = argparse.Namespace(workload="c2_1M_4x800", steps=2, warmup=1, gpus=2, ref_budget=1.0)
    assert bench.reference_arm(args, rank=1) is None
    assert capsys.readouterr().out == ""
