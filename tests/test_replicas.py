"""The multi-GPU layout of bench.py, on CPU: one process per rank (gloo,
world size 2), each solving its own seeded replica of the workload, timings
combined as the maximum over ranks, and the reference arm run by rank 0 only.
(There is no data-path collective: the replicas are independent.)"""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import argparse
    import torch
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # every rank's time enters the job's time as a maximum
        t = bench.max_over_ranks(10.0 + rank, world, torch.device("cpu"))
        # each rank builds its own seeded replica
        _, _, m = bench.build_case("dc2d_small", seed=rank)
        # the reference arm: ranks other than 0 leave without work
        args = argparse.Namespace(workload="dc2d_small", warmup=3, steps=1, gpus=world)
        rc = bench.run_reference(args) if rank != 0 else None
        out[rank] = (t, float(np.asarray(m).sum()), rc)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_max_over_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world,
                           start_method="spawn", join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 11.0
    assert res[0][1] != res[1][1]          # different seeded replicas
    assert res[1][2] == 0                  # rank 1: no reference run
