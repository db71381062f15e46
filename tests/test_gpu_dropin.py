"""The drop-in launcher (cudaMoveParticle's C twin) on caller-owned device buffers.

Restates the reference's CPU/GPU parity test (tests/CudaParticleParityTest.cu:30-158: 11 modes x
2 integrators, particle id 2^53+1, tolerance 1e-12 deterministic / 1e-9 stochastic against the
CPU Particle::move), runs the fixture cases against the oracle's device rules, and compares with
the reference kernel itself where oracle/_ref holds its sm_100a build.
"""
import ctypes
import os

import numpy as np
import pytest

from helpers import DEG, load_move_cases, max_abs_diff
from oracle import bindings as ob
from wacommplusplus_b200 import _native, synthetic as syn
from wacommplusplus_b200.types import PARTICLE_DTYPE, default_config, make_particles

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev(array):
    a = np.ascontiguousarray(array)
    return torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).cuda()


def dev_cfg(cfg):
    return torch.frombuffer(bytearray(bytes(cfg)), dtype=torch.uint8).cuda()


def call_dropin(cfg, records, win, time_index, launcher=None):
    """Runs the launcher on device copies and returns the moved records."""
    d_cfg = dev_cfg(cfg)
    d_p = dev(records)
    f64 = lambda a: dev(np.asarray(a, np.float64))
    f32 = lambda a: None if a is None else dev(np.asarray(a, np.float32))
    t = [f64(win.times), f64(win.mask), f64(win.lonRad), f64(win.latRad), f64(win.depthIntervals),
         f64(win.h), f32(win.zeta), f32(win.u), f32(win.v), f32(win.w), f32(win.akt),
         f32(win.windU10), f32(win.windV10), f32(win.stokesU), f32(win.stokesV)]
    ptr = lambda x: None if x is None else x.data_ptr()
    stream = torch.cuda.current_stream().cuda_stream
    args = [d_cfg.data_ptr(), d_p.data_ptr(), time_index, win.T, win.sW, win.sRho, win.eta,
            win.xi] + [ptr(x) for x in t] + [len(records), 1, 1, stream]
    if launcher is None:
        status = _native.lib().wacomm_b200_cuda_move_particle(*args)
    else:
        status = launcher(*args)
    assert status == 0
    torch.cuda.synchronize()
    return d_p.cpu().numpy().view(PARTICLE_DTYPE).copy()


def parity_window():
    """kernel parity grid (CudaParticleParityTest.cu:35-70)."""
    T = 2
    win = syn.Window(times=np.array([0.0, 65.0]), mask=np.ones((2, 2)),
                     lon=np.array([[0, 1], [0, 1]], np.float64), lat=np.array([[0, 0], [1, 1]], np.float64),
                     lonRad=np.array([[0, DEG], [0, DEG]]), latRad=np.array([[0, 0], [DEG, DEG]]),
                     h=np.full((2, 2), 100.0), sWValues=np.array([-1.0, -.5, 0.0]),
                     depthIntervals=np.array([.5, .5]), zeta=np.zeros((T, 2, 2), np.float32),
                     u=np.zeros((T, 2, 2, 2), np.float32), v=np.zeros((T, 2, 2, 2), np.float32),
                     w=np.zeros((T, 3, 2, 2), np.float32), akt=np.full((T, 3, 2, 2), .01, np.float32))
    win.u[1] = .25
    wind_u = np.arange(8, 16, dtype=np.float32).reshape(T, 2, 2)
    wind_v = np.arange(-2, 6, dtype=np.float32).reshape(T, 2, 2)
    stokes_u = np.array([.05, .06, .07, .08, .09, .10, .11, .12], np.float32).reshape(T, 2, 2)
    stokes_v = np.array([-.04, -.03, -.02, -.01, 0, .01, .02, .03], np.float32).reshape(T, 2, 2)
    return win, (wind_u, wind_v), (stokes_u, stokes_v)


@pytest.mark.parametrize("run", range(22))
def test_reference_parity_modes(cuda_device, run):
    win, wind, stokes = parity_window()
    mode = run % 11
    integrator = 1 if run < 11 else 2
    stochastic = mode == 1
    leeway = mode >= 2
    obj = 7 if mode == 6 else (1 if leeway else 0)
    side = -1 if mode == 6 else (1 if leeway else 0)
    cfg = default_config(random=stochastic, randomSeed=5489, deltat=3600, dti=30, survprob=0,
                         tau0=86400, crid=1, sigma=.1, shoreLimit=.25, upperClosure=1,
                         lowerClosure=1, horizontalClosure=1, integrator=integrator,
                         leewayCoefficientEnsemble=mode == 3,
                         leewayJibeProbabilityHourly=1 if mode == 4 else 0,
                         leewayResidualCorrelation=-.35 if mode == 3 else 0,
                         windErrorStdDev=1.5 if mode == 5 else 0, driftModel=1 if leeway else 0,
                         driftObjectType=obj, driftSide=side, hasWind=leeway, windU10=10,
                         windV10=0, leewayRightSideProbability=0)
    time_index = 1 if mode >= 9 else 0
    cfg.trackingDirection = -1 if mode >= 9 else 1
    cfg.restartCheckpoint = 35 if mode == 10 else float("nan")
    dynamic_wind = mode >= 7
    dynamic_wave = mode == 8 or mode >= 9
    win.windU10, win.windV10 = wind if dynamic_wind else (None, None)
    win.stokesU, win.stokesV = stokes if dynamic_wave else (None, None)
    p = make_particles(1, ids=np.array([9007199254740993], np.uint64), k=-.5, j=.25, i=.25,
                       drift_type=obj, drift_side=side)
    cpu = ob.oracle_move(cfg, p.copy(), win, time_index, ob.SEMANTICS_HOST, 1)
    gpu = call_dropin(cfg, p, win, time_index)
    tol = 1e-9 if stochastic else 1e-12
    assert gpu["id"][0] == cpu["id"][0]
    for f in ("i", "j", "k", "health", "age", "time"):
        assert abs(gpu[f][0] - cpu[f][0]) <= tol, (f, gpu[f][0], cpu[f][0])
    assert gpu["driftSide"][0] == cpu["driftSide"][0]


@pytest.mark.parametrize("case", load_move_cases(), ids=lambda c: c["name"])
def test_fixture_cases_against_device_rules(cuda_device, case):
    cfg = default_config(**case["overrides"])
    win = case["window"]
    got = case["start"].copy()
    want = case["start"].copy()
    for t in (0, 1):
        got = call_dropin(cfg, got, win, t)
        ob.oracle_move(cfg, want, win, t, ob.SEMANTICS_DEVICE, threads=1)
    assert np.array_equal(got["health"] > 0, want["health"] > 0)
    assert np.array_equal(got["driftSide"], want["driftSide"])
    d = max_abs_diff(got, want)
    # 1e-9 degrees (positions), see test_gpu_parity for why not bit-exact
    deg = max(float(np.abs(np.diff(win.lon, axis=1)).max()), float(np.abs(np.diff(win.lat, axis=0)).max()))
    assert max(d["i"], d["j"]) * deg <= 1e-9 and d["k"] <= 1e-9 / deg, d


def _reference_kernel():
    if not os.path.exists(ob.REF_CUDA_SO):
        return None
    lib = ctypes.CDLL(ob.REF_CUDA_SO)
    fn = lib.ref_cuda_move
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 6 + [ctypes.c_void_p] * 15 + \
                  [ctypes.c_int, ctypes.c_void_p]
    return fn


@pytest.mark.parametrize("case", load_move_cases(), ids=lambda c: c["name"])
def test_against_the_reference_kernel(cuda_device, case):
    """The reference kernel is compiled with multiply-add contraction, so it drifts from its own
    CPU path by a few 1e-9 index units over hundreds of substeps (its snapshot tolerance is 1e-8,
    tools/performance_evidence.py:10-11). The drop-in must stay at least as close to the CPU
    rules (the oracle's device rules) as the reference kernel does, and agree with it on
    alive/dead status and drift sides."""
    fn = _reference_kernel()
    if fn is None:
        pytest.skip("reference kernel build absent")
    launcher = lambda *a: fn(*a[:23], a[23], a[26])  # (.., count, numThread, numGPU, stream)
    cfg = default_config(**case["overrides"])
    win = case["window"]
    ours = case["start"].copy()
    theirs = case["start"].copy()
    cpu = case["start"].copy()
    for t in (0, 1):
        ours = call_dropin(cfg, ours, win, t)
        theirs = call_dropin(cfg, theirs, win, t, launcher=launcher)
        ob.oracle_move(cfg, cpu, win, t, ob.SEMANTICS_DEVICE, threads=1)
    assert np.array_equal(ours["health"] > 0, theirs["health"] > 0)
    assert np.array_equal(ours["driftSide"], theirs["driftSide"])
    d_ours = max(max_abs_diff(ours, cpu)[f] for f in ("i", "j", "k"))
    d_theirs = max(max_abs_diff(theirs, cpu)[f] for f in ("i", "j", "k"))
    assert d_ours <= max(1e-9, d_theirs), (d_ours, d_theirs)
    assert max(max_abs_diff(ours, theirs)[f] for f in ("i", "j", "k")) <= 1e-7


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "wacommplusplus_b200")
REF_PROGRAM = os.path.join(ROOT, "oracle", "_ref", "cuda_particle_parity_test")


def test_reference_parity_program_links_against_the_library(cuda_device):
    """The reference's own GPU parity program (tests/CudaParticleParityTest.cu), compiled
    unmodified with its asserts on by oracle/Makefile and linked against libwacomm_b200.so instead
    of cuda/kernel.cu: its 22 cudaMoveParticle calls (Euler and midpoint, every drift mode,
    backward, restart clip) go to the drop-in and must pass the program's own checks against
    Particle::move (1e-12 deterministic, 1e-9 stochastic)."""
    import subprocess
    if not os.path.exists(REF_PROGRAM):
        pytest.skip("the reference program is built only where the reference tree was present")
    ldd = subprocess.run(["ldd", REF_PROGRAM], capture_output=True, text=True).stdout
    line = [x for x in ldd.splitlines() if "libwacomm_b200.so" in x]
    assert line and os.path.realpath(LIB_DIR) in os.path.realpath(line[0].split("=>")[1].split()[0])
    assert "libwacomm_ref_cuda" not in ldd
    run = subprocess.run([REF_PROGRAM], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, (run.returncode, run.stdout[-2000:], run.stderr[-2000:])


def test_engine_abi_from_a_cpp_program(cuda_device, tmp_path):
    """A C++ host program (tests/abi_caller.cpp) drives a whole interval through the extern "C"
    engine ABI only, compiled here against include/wacomm_b200.h and linked to the library."""
    import subprocess
    exe = str(tmp_path / "abi_caller")
    build = subprocess.run(
        ["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "abi_caller.cpp"),
         "-I", os.path.join(ROOT, "include"), "-L", LIB_DIR, "-lwacomm_b200",
         f"-Wl,-rpath,{LIB_DIR}", "-o", exe], capture_output=True, text=True)
    assert build.returncode == 0, build.stderr[-2000:]
    run = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, (run.returncode, run.stdout[-2000:], run.stderr[-2000:])
    assert "2000 records, 0 off" in run.stdout
