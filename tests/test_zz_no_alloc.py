"""The allocation-free launcher against the drop-in launcher, through the C ABI.

wacomm_b200_cuda_move_particle_noalloc serves callers that may not allocate device memory while
they drive the particle step (cudaFree synchronizes the device and stalls their other streams;
some frameworks own all device memory). Its working memory is a fixed array inside the library,
shared by every call on a device, so two calls in a row are checked: the second runs on a
smaller grid with fewer records, on top of what the first left in the array. Each call must
give the drop-in launcher's records within the parity tolerance (1e-9 degrees; the two run the
same step code with the same flags, so they are in fact identical).

This file is collected last on purpose.
"""
import numpy as np
import pytest

from test_gpu_dropin import call_dropin, torch  # noqa: F401  (torch: skip when absent)
from wacommplusplus_b200 import _native, synthetic as syn
from wacommplusplus_b200.types import default_config

pytestmark = pytest.mark.gpu


def _scene(eta, n, seed):
    rf = syn.RealisticForcing(eta=eta, xi=eta - 8, s_rho=6, n_frames=3, seed=seed,
                              dlon=0.002, dlat=0.002)
    win = rf.window()
    rng = np.random.default_rng(seed)
    T = win.T
    win.windU10 = (7 + 2 * rng.standard_normal((T, win.eta, win.xi))).astype(np.float32)
    win.windV10 = (2 * rng.standard_normal((T, win.eta, win.xi))).astype(np.float32)
    p = rf.release(n, n_sources=16, seed=seed + 1)
    p["time"] = win.times[0] + rng.uniform(0, 3600, len(p))
    p["driftObjectType"] = rng.integers(0, 23, len(p))
    p["driftSide"] = rng.choice([-1, 1], len(p))
    cfg = default_config(random=True, driftModel=1, windErrorStdDev=0.5, windU10=5.0,
                         leewayJibeProbabilityHourly=0.2)
    return win, p, cfg


def _noalloc(*args):
    return _native.lib().wacomm_b200_cuda_move_particle_noalloc(*args)


def _within(got, want, win):
    deg = max(float(np.abs(np.diff(win.lon, axis=1)).max()),
              float(np.abs(np.diff(win.lat, axis=0)).max()))
    assert np.array_equal(got["id"], want["id"])
    assert np.array_equal(got["health"] > 0, want["health"] > 0)
    assert np.array_equal(got["driftSide"], want["driftSide"])
    for f in ("i", "j"):
        assert np.nanmax(np.abs(got[f] - want[f])) * deg <= 1e-9
    assert np.nanmax(np.abs(got["k"] - want["k"])) <= 1e-9 / deg
    assert np.nanmax(np.abs(got["age"] - want["age"])) <= 1e-9


def test_noalloc_matches_the_dropin_launcher_on_two_calls(cuda_device):
    for eta, n, seed in ((96, 150000, 41), (40, 20000, 42)):
        win, p, cfg = _scene(eta, n, seed)
        for t in (0, 1):
            want = call_dropin(cfg, p, win, t)
            got = call_dropin(cfg, p, win, t, launcher=_noalloc)
            _within(got, want, win)
            # every field identical (padding bytes of the 64-byte records are not compared)
            for f in got.dtype.names:
                assert np.array_equal(got[f], want[f], equal_nan=True), f
            p = got


def test_noalloc_refuses_sizes_beyond_its_limit(cuda_device):
    win, p, cfg = _scene(40, 64, 43)
    big = 1 << 22  # claims more records than the fixed working memory holds; nothing is read
    status = _native.lib().wacomm_b200_cuda_move_particle_noalloc(
        None, None, 0, win.T, win.sW, win.sRho, win.eta, win.xi, *([None] * 15), big, 1, 1, None)
    assert status == -_native.ERR_CAPACITY
    status = _native.lib().wacomm_b200_cuda_move_particle_noalloc(
        None, None, 0, win.T, win.sW, win.sRho, 2048, 1024, *([None] * 15), 10, 1, 1, None)
    assert status == -_native.ERR_CAPACITY


def test_noalloc_moves_records_of_a_grid_without_cells(cuda_device):
    """A grid one node wide has no interpolation cell: the allocation-free launcher moves its
    records in caller order without the cell sort, as the drop-in launcher does (both kill every
    record on its first substep, before any forcing read)."""
    T, eta, xi = 2, 1, 5
    lon = np.linspace(14.0, 14.1, xi)[None, :]
    lat = np.full((eta, xi), 40.8)
    win = syn.Window(times=np.array([0.0, 3600.0]), mask=np.ones((eta, xi)), lon=lon, lat=lat,
                     lonRad=lon * syn.ADAPTER_DEG2RAD, latRad=lat * syn.ADAPTER_DEG2RAD,
                     h=np.full((eta, xi), 50.0), sWValues=np.array([-1.0, -.5, 0.0]),
                     depthIntervals=np.array([.5, .5]), zeta=np.zeros((T, eta, xi), np.float32),
                     u=np.full((T, 2, eta, xi), .2, np.float32),
                     v=np.zeros((T, 2, eta, xi), np.float32),
                     w=np.zeros((T, 3, eta, xi), np.float32),
                     akt=np.full((T, 3, eta, xi), 1e-4, np.float32))
    p = syn.uniform_particles(300, 2, xi, seed=44)
    p["j"] = 0.0
    cfg = default_config(random=True)
    want = call_dropin(cfg, p, win, 0)
    got = call_dropin(cfg, p, win, 0, launcher=_noalloc)
    for f in got.dtype.names:
        assert np.array_equal(got[f], want[f], equal_nan=True), f
    assert not np.any(got["health"] > 0)
