"""Multi-process path of the benchmark on CPU: two gloo ranks, max-over-ranks timing (CPU)."""
import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, queue):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    elapsed = [12.5, 20.0][rank]
    slowest = bench.max_over_ranks(elapsed, world)
    value = bench.replica_throughput(64, world, slowest)
    bench.barrier(world)
    queue.put((rank, slowest, value))
    dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, value in res:
        assert slowest == 20.0
        assert abs(value - 2 * 64 / 0.020) < 1e-6
