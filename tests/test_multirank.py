"""The N > 1 path of bench.py on CPU: two gloo ranks (one process per rank, as torchrun starts
them).  Pixels are independent, so ranks share no data; they meet only for barriers and for the
max-over-ranks step time from which rank 0 reports the whole-job throughput."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import sys

    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    w, r, local = bench.dist_setup(backend="gloo")
    assert (w, r, local) == (world, rank, rank)
    # rank r's step took 10 + 5 r ms; the slowest rank sets the job time
    value, ms = bench.job_throughput(4096, 10.0 + 5.0 * rank, w, torch.device("cpu"))
    bench.barrier(w)
    # the reference arm runs on rank 0 only; the others return nothing and exit 0
    class A:
        steps, warmup = 1, 0
    ref = bench.run_reference(A) if rank != 0 else "rank0"
    out.put((rank, value, ms, ref))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_report_max_over_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, ms, ref in res:
        assert ms == pytest.approx(15.0)                    # max over ranks
        assert value == pytest.approx(2 * 4096 / 0.015)     # both ranks' pixels over that time
    assert res[1][3] is None                                # rank 1 runs no reference arm
