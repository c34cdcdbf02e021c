"""The multi-process side of bench.py on CPU (gloo, world size 2): replicas
are timed as the maximum over ranks, and the reference arm runs on rank 0
only while the other ranks leave without work or output."""
import io
import os
import socket
from contextlib import redirect_stdout

import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, results) -> None:
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        got = bench.max_over_ranks([1.0 + rank, 10.0 * (world - rank)], dist, "cpu")
        out = io.StringIO()

        class Args:
            warmup, steps = 0, 0

        if rank != 0:
            with redirect_stdout(out):
                bench.reference_arm(Args, rank, world)
        dist.barrier()
        results[rank] = (got, out.getvalue())
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rank0_only_reference():
    world = 2
    manager = mp.get_context("spawn").Manager()
    results = manager.dict()
    mp.start_processes(_rank_main, args=(world, _free_port(), results), nprocs=world, join=True, start_method="spawn")
    for rank in range(world):
        got, printed = results[rank]
        assert got == [2.0, 20.0]
        assert printed == ""


def test_max_over_ranks_single_process():
    import bench
    assert bench.max_over_ranks([3.0, 4.0], None, "cpu") == [3.0, 4.0]
