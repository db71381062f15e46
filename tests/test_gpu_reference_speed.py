"""The reference's own GPU path timed beside this library on the same B200 (the GPU comparator).

The reference kernel (cuda/kernel.cu, launched through its unmodified cudaMoveParticle) is built
for sm_100a from its sources into oracle/_ref by oracle/Makefile. On the precision workload's
grid (128x128x10, uniform current, deterministic midpoint, dt = 30 s) and 2,097,152 particles
resident on the device, one forcing interval is timed kernel-only with CUDA events for:

* the reference cudaMoveParticle (FP64, one thread per particle, particles in caller order);
* this library's drop-in with the identical signature and the same device buffers (reference
  arithmetic, device rules: the same results to round-off; the work ordered by cell through
  stream-ordered scratch);
* the allocation-free drop-in (the same update, the same ordering, a fixed scratch array);
* the engine's FP32 step on the same particles (resident, cell-sorted, cell-column layout).

Both drop-ins must be clearly faster than the kernel they replace, and the FP32 step far faster;
the rates are printed for the design notes.
"""
import ctypes
import os
import time

import numpy as np
import pytest

from oracle import bindings as ob
from wacommplusplus_b200 import _native, synthetic as syn
from wacommplusplus_b200.engine import Engine
from wacommplusplus_b200.types import default_config

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

N = 1 << 21
SUBSTEPS = 120
INTERVAL = 3


def _reference_kernel():
    if not os.path.exists(ob.REF_CUDA_SO):
        return None
    lib = ctypes.CDLL(ob.REF_CUDA_SO)
    fn = lib.ref_cuda_move
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 6 + \
                  [ctypes.c_void_p] * 15 + [ctypes.c_int, ctypes.c_void_p]
    return fn


def _dev(array):
    a = np.ascontiguousarray(array)
    return torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).cuda()


def _timed(call, repeats=3):
    """Mean device milliseconds of call() over `repeats` after one warm-up."""
    stream = torch.cuda.current_stream()
    call()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(repeats):
        call()
    end.record(stream)
    torch.cuda.synchronize()
    return start.elapsed_time(end) / repeats


def test_reference_kernel_against_this_library(cuda_device):
    fn = _reference_kernel()
    if fn is None:
        pytest.skip("reference kernel build absent")
    win = syn.config1_window(n_frames=25)
    cfg = default_config(random=False)
    parts = syn.uniform_particles(N, win.eta, win.xi, seed=3)
    d_cfg = torch.frombuffer(bytearray(bytes(cfg)), dtype=torch.uint8).cuda()
    f64 = lambda a: _dev(np.asarray(a, np.float64))
    f32 = lambda a: _dev(np.asarray(a, np.float32))
    fields = [f64(win.times), f64(win.mask), f64(win.lonRad), f64(win.latRad),
              f64(win.depthIntervals), f64(win.h), f32(win.zeta), f32(win.u), f32(win.v),
              f32(win.w), f32(win.akt)]
    ptrs = [x.data_ptr() for x in fields] + [None] * 4
    stream = torch.cuda.current_stream().cuda_stream
    head = [win.T, win.sW, win.sRho, win.eta, win.xi]
    # every timed call starts from the same records: each moves a fresh copy over one interval
    theirs = _dev(parts)
    ours = _dev(parts)
    start = _dev(parts)

    def reference():
        theirs.copy_(start)
        assert fn(d_cfg.data_ptr(), theirs.data_ptr(), INTERVAL, *head, *ptrs, N, stream) == 0

    def dropin():
        ours.copy_(start)
        assert _native.lib().wacomm_b200_cuda_move_particle(
            d_cfg.data_ptr(), ours.data_ptr(), INTERVAL, *head, *ptrs, N, 1, 1, stream) == 0

    def noalloc():
        ours.copy_(start)
        assert _native.lib().wacomm_b200_cuda_move_particle_noalloc(
            d_cfg.data_ptr(), ours.data_ptr(), INTERVAL, *head, *ptrs, N, 1, 1, stream) == 0

    # three interleaved rounds, the fastest of each: another tenant of a shared GPU slows single
    # rounds, not all of them
    copy_ms = min(_timed(lambda: theirs.copy_(start)) for _ in range(3))
    rounds = [(_timed(reference), _timed(noalloc), _timed(dropin)) for _ in range(3)]
    ref_ms, noalloc_ms, dropin_ms = (min(r[c] for r in rounds) - copy_ms for c in range(3))
    got = ours.cpu().numpy().view(parts.dtype)
    want = theirs.cpu().numpy().view(parts.dtype)
    assert np.array_equal(got["health"] > 0, want["health"] > 0)
    assert max(np.abs(got[f] - want[f]).max() for f in ("i", "j", "k")) <= 1e-7

    with Engine(cuda_device, arithmetic="fp32") as e:
        e.set_config(cfg)
        e.load_window(win)
        e.set_particles(parts)
        fp32 = []
        for _ in range(4):
            e.set_particles(parts)
            e.move_interval(INTERVAL)
            fp32.append(e.stats()["move_ms"])
        fp32_ms = float(np.mean(fp32[1:]))

    steps = N * SUBSTEPS
    rate = lambda ms: steps / (ms / 1000.0)
    print(f"\nreference cudaMoveParticle: {ref_ms:.2f} ms ({rate(ref_ms):.3g} particle-steps/s); "
          f"drop-in (cell-ordered work, pool scratch): {dropin_ms:.2f} ms ({rate(dropin_ms):.3g}, {ref_ms / dropin_ms:.1f}x); "
          f"allocation-free drop-in (cell-ordered work, fixed scratch): {noalloc_ms:.2f} ms "
          f"({rate(noalloc_ms):.3g}, {ref_ms / noalloc_ms:.1f}x); "
          f"FP32 step: {fp32_ms:.2f} ms ({rate(fp32_ms):.3g}, {ref_ms / fp32_ms:.1f}x)")
    # ordering the work by cell makes both launchers faster than the kernel they replace (all
    # three run the FP64 arithmetic; measured about 1.7x, asserted with margin for box-to-box
    # variation), the FP32 step is far ahead
    assert dropin_ms * 1.3 < ref_ms and noalloc_ms * 1.3 < ref_ms
    assert fp32_ms * 4 < ref_ms


def _reference_staged():
    if not os.path.exists(ob.REF_CUDA_SO):
        return None
    fn = ctypes.CDLL(ob.REF_CUDA_SO).ref_cuda_interval_staged
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 6 + \
                  [ctypes.c_void_p] * 11 + [ctypes.c_int]
    return fn


def test_reference_staged_interval_against_the_host_buffer_entry(cuda_device):
    """One interval end to end from host records, on the same window and particles: the reference's
    own per-interval GPU staging around its kernel (Wacomm.cpp:386-660: allocate and upload the
    whole forcing window, upload the records, move, download, free; restated in the oracle's
    shim) against this library's host-buffer entry (window resident, one new forcing record
    uploaded per interval, records streamed in slabs), with pageable host records on both sides.
    The reference-arithmetic run must reproduce the reference's records."""
    fn = _reference_staged()
    if fn is None:
        pytest.skip("reference kernel build absent")
    win = syn.config1_window(n_frames=25)
    cfg = default_config(random=False)
    parts = syn.uniform_particles(N, win.eta, win.xi, seed=3)
    f64 = lambda a: np.ascontiguousarray(a, np.float64)
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    fields = [f64(win.times), f64(win.mask), f64(win.lonRad), f64(win.latRad),
              f64(win.depthIntervals), f64(win.h), f32(win.zeta), f32(win.u), f32(win.v),
              f32(win.w), f32(win.akt)]
    cfg_bytes = np.frombuffer(bytearray(bytes(cfg)), np.uint8)
    head = [win.T, win.sW, win.sRho, win.eta, win.xi]

    def reference():
        host = parts.copy()
        t0 = time.perf_counter()
        assert fn(cfg_bytes.ctypes.data, host.ctypes.data, INTERVAL, *head,
                  *[a.ctypes.data for a in fields], N) == 0
        return time.perf_counter() - t0, host

    ref_s, want = min((reference() for _ in range(3)), key=lambda r: r[0])
    frame = {k: np.ascontiguousarray(v) for k, v in win.frame(INTERVAL + 2).items()
             if k in ("zeta", "u", "v", "w", "akt")}
    ours = {}
    for arithmetic in ("reference", "fp32"):
        with Engine(cuda_device, semantics="device", arithmetic=arithmetic) as e:
            e.set_config(cfg)
            e.load_window(win)
            best = None
            for _ in range(4):
                host = parts.copy()
                t0 = time.perf_counter()
                e.upload_frame(INTERVAL + 2, **frame)
                e.move_interval_host(INTERVAL, host)
                dt = time.perf_counter() - t0
                best = dt if best is None else min(best, dt)
            ours[arithmetic] = (best, host)
    d = max(float(np.abs(ours["reference"][1][f] - want[f]).max()) for f in ("i", "j", "k"))
    assert d <= 1e-7, d
    steps = N * SUBSTEPS
    rate = lambda s: steps / s
    print(f"\nreference staged interval (window + records up, move, records down): "
          f"{ref_s * 1e3:.1f} ms ({rate(ref_s):.3g} particle-steps/s); host-buffer entry, "
          f"reference arithmetic: {ours['reference'][0] * 1e3:.1f} ms "
          f"({ref_s / ours['reference'][0]:.1f}x); FP32 step: {ours['fp32'][0] * 1e3:.1f} ms "
          f"({rate(ours['fp32'][0]):.3g}, {ref_s / ours['fp32'][0]:.1f}x)")
    assert ours["fp32"][0] * 4 < ref_s
