"""Asynchronous record upload (wacomm_b200_upload_frame_async): a run that uploads each record one
interval ahead, from page-locked memory while the kernels run, must equal the run with every
record resident from the start, bit for bit; and re-uploading a record that an enqueued interval
still reads must not change that interval (the copy waits for the kernels enqueued before it)."""
import numpy as np
import pytest

from wacommplusplus_b200 import synthetic as syn
from wacommplusplus_b200.engine import Engine
from wacommplusplus_b200.types import default_config

pytestmark = pytest.mark.gpu


def pinned_frame(win, t, scale=1.0):
    """Record t of `win` copied into page-locked host arrays (numpy views of pinned tensors)."""
    import torch
    out = {}
    for name, arr in win.frame(t).items():
        if arr is None:
            out[name] = None
            continue
        buf = torch.empty(arr.shape, dtype=torch.float32, pin_memory=True)
        view = buf.numpy()
        view[...] = arr * (scale if name in ("u", "v") else 1.0)
        out[name] = view
    return out


def upload(e, t, f, async_=True):
    (e.upload_frame_async if async_ else e.upload_frame)(
        t, f["zeta"], f["u"], f["v"], f["w"], f["akt"], f["windU10"], f["windV10"], f["stokesU"],
        f["stokesV"])


def fresh(win, cfg, records, frames=None):
    e = Engine(0)
    e.set_config(cfg)
    e.load_window(win, frames=frames)
    e.concentration_reset(win.T)
    e.set_particles(records)
    return e


def test_prefetch_one_interval_ahead_equals_resident(cuda_device):
    forcing = syn.RealisticForcing(eta=128, xi=112, s_rho=10, n_frames=6, seed=8)
    win = forcing.window()
    cfg = default_config(random=True, randomSeed=4)
    records = forcing.release(400000, n_sources=32, seed=5)
    records["time"] = win.times[0]
    resident = fresh(win, cfg, records)
    ahead = fresh(win, cfg, records, frames=[0, 1])
    for t in range(win.T - 1):
        if t + 2 < win.T:
            upload(ahead, t + 2, pinned_frame(win, t + 2))
        ahead.move_interval(t)
        resident.move_interval(t)
    ahead.synchronize()
    a, b = ahead.get_particles(), resident.get_particles()
    for f in a.dtype.names:
        assert a[f].tobytes() == b[f].tobytes(), f
    assert np.array_equal(ahead.concentration(), resident.concentration())
    ahead.close()
    resident.close()


def test_reupload_waits_for_the_interval_that_reads_the_record(cuda_device):
    win = syn.config1_window(n_frames=3)
    cfg = default_config(random=False)
    records = syn.uniform_particles(2_000_000, win.eta, win.xi, seed=3, time=win.times[0])
    # reference: interval 0 with the original record 1, interval 1 with record 1 doubled
    changed = pinned_frame(win, 1, scale=2.0)
    ref = fresh(win, cfg, records)
    ref.move_interval(0)
    after0 = ref.get_particles()
    upload(ref, 1, changed, async_=False)
    ref.move_interval(1)
    after1 = ref.get_particles()
    ref.close()
    # the re-upload is enqueued while interval 0's kernels may still run
    e = fresh(win, cfg, records)
    e.move_interval(0)
    upload(e, 1, changed)
    got0 = e.get_particles()
    e.move_interval(1)
    got1 = e.get_particles()
    e.close()
    for f in after0.dtype.names:
        assert got0[f].tobytes() == after0[f].tobytes(), f
        assert got1[f].tobytes() == after1[f].tobytes(), f
