"""Sharding across ranks on the CPU: the reference's contiguous split (NumericalHelpers.hpp:76-82)
and the concentration all-reduce of per-shard counts, run as two `gloo` ranks on 127.0.0.1."""
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import bindings as ob
from wacommplusplus_b200 import sharding
from wacommplusplus_b200 import synthetic as syn


@pytest.mark.parametrize("total,workers", [(0, 1), (7, 1), (7, 3), (10, 4), (1000003, 8), (3, 5)])
def test_partition_covers_every_particle_once(total, workers):
    counts = [sharding.partition_count(total, workers, w) for w in range(workers)]
    offsets = [sharding.partition_offset(total, workers, w) for w in range(workers)]
    assert sum(counts) == total
    assert offsets[0] == 0
    for w in range(1, workers):
        assert offsets[w] == offsets[w - 1] + counts[w - 1]
        assert counts[w] == total // workers          # only rank 0 takes the remainder
    assert counts[0] == total // workers + total % workers


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, records, win_shape, out):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        n_times, s_rho, eta, xi = win_shape
        Grid = type("Grid", (), {"sRho": s_rho, "eta": eta, "xi": xi})
        mine = sharding.shard(records, rank, world)
        conc = ob.oracle_concentration(np.ascontiguousarray(mine), 1, n_times, Grid)
        view = torch.from_numpy(conc.view(np.int32))
        sharding.reduce_counts(view[1])
        # counts past 2^31 keep their uint32 meaning through the signed view
        big = torch.tensor([np.uint32(3_000_000_000).view(np.int32), 5], dtype=torch.int32)
        sharding.reduce_counts(big)
        out[rank] = (conc.copy(), big.numpy().view(np.uint32).copy())
    finally:
        dist.destroy_process_group()


def test_two_rank_concentration_equals_the_whole_set():
    win = syn.config1_window(n_frames=3, eta=32, xi=24, s_rho=4)
    records = syn.uniform_particles(20001, win.eta, win.xi, seed=6)
    records["k"] = -np.random.default_rng(2).uniform(0, 3, len(records))
    records["health"][::17] = -1.0
    shape = (win.T, win.sRho, win.eta, win.xi)
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_rank_main, args=(2, _free_port(), records, shape, out), nprocs=2,
                       join=True, start_method="spawn")
    want = ob.oracle_concentration(records, 1, win.T, win)
    for rank in (0, 1):
        conc, big = out[rank]
        assert np.array_equal(conc[1], want[1]), rank
        assert not conc[0].any() and not conc[2].any()
        assert big[0] == np.uint32((2 * 3_000_000_000) % 2**32) and big[1] == 10
