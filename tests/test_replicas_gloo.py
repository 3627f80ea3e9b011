"""Multi-process (replicas) logic of bench.py on CPU ranks with the gloo backend.

`bench.py --gpus N` runs one process per GPU, each rendering its own cameras of
the same scene (the path has no collective); the reported time is the maximum
over ranks.  Two gloo ranks check both on the CPU.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sc = bench.make_scene(rank, world, 1000, 4)
        t_max = bench.max_over_ranks(10.0 + rank, world)
        bench.barrier(world)
        out.put((rank, sc["viewmats"], t_max))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_render_distinct_cameras_and_agree_on_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, vm, t = q.get(timeout=120)
        res[r] = (vm, t)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == res[1][1] == 11.0
    assert not np.allclose(res[0][0], res[1][0])  # each replica renders its own cameras
