"""The multi-rank bookkeeping of bench.py on CPU: two gloo ranks, each with
its own device times, agree on the element-wise maximum (a multi-GPU run is
timed as the slowest rank), and a single process passes its times through."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        r, w, local = bench._dist_env()
        times = [10.0 + rank, 20.0 - 5.0 * rank, 7.5]
        out.put((rank, (r, w, local), bench._max_over_ranks(times, torch.device("cpu"))))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, env, mx in res:
        assert env == (rank, 2, rank)
        assert mx == [11.0, 20.0, 7.5]


def test_max_over_ranks_single_process():
    if dist.is_available() and dist.is_initialized():
        pytest.skip("a process group is already active")
    assert bench._max_over_ranks([3, 1.5], torch.device("cpu")) == [3.0, 1.5]
