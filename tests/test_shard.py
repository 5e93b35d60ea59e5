"""The multi-rank path of the batched solve on CPU: two gloo ranks take disjoint seeded cells, reduce the step
time by max and gather C in rank order (the same helpers bench.py uses under torchrun with nccl)."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as tmp

from nlfiber_b200 import shard
from oracle import density_ref as OD
from oracle import linear_ref as OL


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seeds = shard.cell_seeds(rank, 2)
        lh = OL.LinearHomogenization((4, 4, 4), tol=1e-10, maxit=500)
        C = np.stack([lh.C_full(OD.random_cell(i, n_o=2, beta=4.0)[0])[0] for i in seeds])
        t = shard.max_over_ranks(1.0 + rank, dist)  # rank 1 is the slower one
        allC = shard.gather_C(C, dist)
        out[rank] = (seeds, t, allC, shard.whole_job_rate(2, world, t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_cells_and_reduce_timing():
    world, port = 2, _free_port()
    with tmp.get_context("spawn").Manager() as mgr:  # no fork of this (threaded) test process
        out = mgr.dict()
        tmp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert res[0][0] == [0, 1] and res[1][0] == [2, 3]  # disjoint seeds, weak scaling
    assert res[0][1] == res[1][1] == 2.0  # max over ranks on every rank
    assert res[0][3] == 2.0  # 4 cells over the slowest rank's 2 s
    lh = OL.LinearHomogenization((4, 4, 4), tol=1e-10, maxit=500)
    ref = np.stack([lh.C_full(OD.random_cell(i, n_o=2, beta=4.0)[0])[0] for i in range(4)])
    for r in (0, 1):
        np.testing.assert_allclose(res[r][2], ref, rtol=1e-12, atol=1e-15)  # gathered in rank order
