"""The N > 1 path of the benchmark on CPU with two gloo ranks (one process
per rank, as torchrun launches them): the job's time is the max over the
ranks, and in the reference arm only rank 0 does work.  The data path has
no cross-rank exchange (replicas), so this is the whole multi-rank logic."""
import datetime
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    try:
        sys.path.insert(0, ROOT)
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
        import torch.distributed as dist
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        import bench
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 0.5 * rank], "cpu")
        # the reference arm under torchrun: ranks other than 0 return at once
        ran = None
        if rank != 0:
            class A:
                steps, warmup = 1, 1
            bench.run_reference(A(), rank, world)
            ran = "returned"
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, got, ran))
    except Exception as e:  # reported to the parent, which fails the test
        q.put((rank, repr(e), None))


def test_two_gloo_ranks_reduce_to_the_slowest():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict()
    for _ in procs:
        rank, got, ran = q.get(timeout=120)
        out[rank] = (got, ran)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in (0, 1):
        assert out[rank][0] == [2.0, 10.0, 0.5], out
    assert out[1][1] == "returned"
