"""The multi-GPU path's host logic on CPU: two gloo ranks (world size 2) shard the points (each
rank its own seeded points of the same family split, no data-path exchange) and meet once, in
bench.reduce_over_ranks: the slowest rank's step time and the families' summed totals."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, path):
    import datetime

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sums = torch.tensor([1.0 + rank, 10.0 * rank], dtype=torch.float64)
        squares = torch.tensor([2.0, 3.0 + rank], dtype=torch.float64)
        peak = torch.tensor([5.0 - rank, 1.0 + rank], dtype=torch.float64)
        ms, total, sq, mx = bench.reduce_over_ranks(dist, 3.0 + 2.0 * rank, sums, squares, peak)
        bench.POINTS = 4096
        fams = bench.workload(rank)
        first = np.concatenate([p[:4].reshape(-1) for _, _, p in fams])
        np.savez(f"{path}_{rank}.npz", ms=ms, total=total.numpy(), sq=sq.numpy(), mx=mx.numpy(),
                 counts=[p.shape[0] for _, _, p in fams], first=first)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_points_and_reduce_once(tmp_path):
    world, port = 2, _free_port()
    path = str(tmp_path / "rank")
    mp.start_processes(_rank, args=(world, port, path), nprocs=world, join=True, start_method="spawn")
    r = [np.load(f"{path}_{k}.npz") for k in range(world)]
    for x in r:
        assert float(x["ms"]) == 5.0                       # the slowest rank's time
        assert np.array_equal(x["total"], [3.0, 10.0])     # summed over the ranks
        assert np.array_equal(x["sq"], [4.0, 7.0]) and np.array_equal(x["mx"], [5.0, 2.0])
    assert np.array_equal(r[0]["counts"], r[1]["counts"])  # the same family split per rank
    assert sum(r[0]["counts"]) == 4096
    assert not np.array_equal(r[0]["first"], r[1]["first"])  # each rank its own points
