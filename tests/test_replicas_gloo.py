"""The replica path of bench.py (one process per GPU, no data-path collective)
on CPU: two gloo ranks read their rank from the launcher's environment and take
the max of their timings, as the NCCL ranks do on GPUs."""
import os
import socket

import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    r, w, local = bench.dist_env()
    assert (r, w, local) == (rank, world, rank)
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank          # this rank's timed region
        out[rank] = bench.max_over_ranks(ms, "cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_world_2():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        assert dict(out) == {0: 15.0, 1: 15.0}
