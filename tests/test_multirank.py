"""The bench's multi-GPU plumbing on CPU: two gloo ranks (one process each, as torchrun
starts them) agree on the max-over-ranks time and draw different inputs.  The GPU work of
each rank is independent (no data-path collective), so this is all the ranks share."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        m = bench.max_over_ranks(10.0 + 3.5 * rank, dist, torch, device="cpu")
        seeds = bench.rank_seeds(8192, 2048, rank)
        out.put((rank, m, seeds))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_time_and_differ_in_inputs():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [13.5, 13.5]
    s0, s1 = res[0][2], res[1][2]
    assert all(s0[k] != s1[k] for k in s0)


def test_single_rank_needs_no_process_group():
    import torch
    import bench
    assert bench.max_over_ranks(4.25, None, torch) == 4.25
