"""Shot sharding across ranks: two gloo processes on CPU."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from tspeed_b200.shard import gather_seismograms, max_over_ranks, shots_for_rank


def test_slices_partition_the_shots():
    for total in (0, 1, 7, 64, 130):
        for world in (1, 2, 3, 8):
            got = [i for r in range(world) for i in shots_for_rank(total, r, world)]
            assert got == list(range(total))
            sizes = [len(shots_for_rank(total, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shots_for_rank(4, 2, 2)


def _fake_seismogram(shot, nk=5, nr=3):
    k = np.arange(nk)[:, None, None]
    r = np.arange(nr)[None, :, None]
    c = np.arange(2)[None, None, :]
    return np.sin(0.1 * shot + k) * (r + 1) + c


def _worker(rank, world, port, total, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shots_for_rank(total, rank, world)
        local = np.stack([_fake_seismogram(s) for s in mine]) if len(mine) else np.zeros((0, 5, 3, 2))
        t = max_over_ranks(10.0 + rank, dist)
        g = gather_seismograms(local, total, dist)
        if rank == 0:
            np.save(out, g)
            np.save(out + ".t.npy", np.array([t]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("total", [7, 8])
def test_gather_in_global_shot_order(tmp_path, total):
    out = str(tmp_path / "g.npy")
    mp.spawn(_worker, args=(2, _free_port(), total, out), nprocs=2, join=True)
    g = np.load(out)
    ref = np.stack([_fake_seismogram(s) for s in range(total)])
    assert np.array_equal(g, ref)
    assert float(np.load(out + ".t.npy")[0]) == 11.0
