"""Particle shards on the GPU: the device view of the concentration grid, its all-reduce through
NCCL (a one-rank group here: one GPU per call on this pool), and the shard decomposition itself,
emulated as two contexts on one GPU with no kernel waiting on another -- records and summed
concentration must equal the single-context run bit for bit, since each particle's update depends
only on its own state and id."""
import socket

import numpy as np
import pytest

from wacommplusplus_b200 import sharding
from wacommplusplus_b200 import synthetic as syn
from wacommplusplus_b200.engine import Engine
from wacommplusplus_b200.types import default_config

pytestmark = pytest.mark.gpu


def engine_for(win, cfg, records):
    e = Engine(0, arithmetic="fp32", storage="fp32")
    e.set_config(cfg)
    e.load_window(win)
    e.concentration_reset(win.T)
    e.set_particles(records)
    return e


def test_device_view_and_one_rank_nccl_allreduce(cuda_device):
    import torch
    import torch.distributed as dist
    win = syn.config1_window(n_frames=3)
    cfg = default_config(random=True, randomSeed=9)
    e = engine_for(win, cfg, syn.uniform_particles(50000, win.eta, win.xi, seed=2))
    e.move_interval(0)
    host = e.concentration()
    view = e.concentration_view(1)
    torch.cuda.synchronize()
    assert view.dtype == torch.int32 and tuple(view.shape) == host.shape[1:]
    assert np.array_equal(view.cpu().numpy().view(np.uint32), host[1])
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            device_id=torch.device("cuda", cuda_device))
    try:
        sharding.allreduce_concentration(e, 1)
        e.synchronize()
        assert np.array_equal(e.concentration(), host)
    finally:
        dist.destroy_process_group()
    e.close()


@pytest.mark.parametrize("world", [2, 3])
def test_shards_sum_to_the_whole(cuda_device, world):
    win = syn.config1_window(n_frames=4)
    cfg = default_config(random=True, randomSeed=21)
    records = syn.uniform_particles(90001, win.eta, win.xi, seed=5)
    whole = engine_for(win, cfg, records)
    parts = [engine_for(win, cfg, sharding.shard(records, r, world)) for r in range(world)]
    for t in range(3):
        whole.move_interval(t)
        for p in parts:
            p.move_interval(t)
    want = whole.get_particles()
    got = np.concatenate([p.get_particles() for p in parts])
    for f in want.dtype.names:
        assert want[f].tobytes() == got[f].tobytes(), f
    total = sum(p.concentration().astype(np.uint64) for p in parts)
    assert np.array_equal(total, whole.concentration())
    for e in parts + [whole]:
        e.close()
