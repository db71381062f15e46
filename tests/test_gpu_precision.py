"""FP32 interpolation and FP16/BF16 forcing storage against the FP64 oracle, and the Philox
diffusion streams by ensemble moments.

Bounds (positions as great-circle metres after the stated simulated time):
  * FP32 forcing, FP32 interpolation: mean <= 0.05 m, p99 <= 0.5 m;
  * FP16 / BF16 forcing:              mean <= 50 m, p99 <= 200 m (the precision targets).
Closure decisions (a landing test or a reflection taken by one side and not the other) move a
particle onto another trajectory; they dominate the maximum error, so they are counted
separately (errors above 1 m in FP32) and must stay rare.
"""
import numpy as np
import pytest

from helpers import great_circle_m, max_abs_diff
from oracle import bindings as ob
from wacommplusplus_b200 import synthetic as syn
from wacommplusplus_b200.engine import Engine
from wacommplusplus_b200.types import default_config

pytestmark = pytest.mark.gpu


def _run(engine, win, cfg, particles, intervals):
    engine.load_window(win)
    engine.set_config(cfg)
    engine.set_particles(particles)
    for t in intervals:
        engine.move_interval(t)
    return engine.get_particles()


def _oracle(win, cfg, particles, intervals):
    out = particles.copy()
    for t in intervals:
        ob.oracle_move(cfg, out, win, t, threads=0)
    return out


@pytest.fixture(scope="module")
def analytic_day():
    win = syn.config1_window(n_frames=25)
    p = syn.uniform_particles(8192, win.eta, win.xi, seed=7)
    cfg = default_config(random=False, horizontalClosure=1)
    return win, cfg, p, _oracle(win, cfg, p, range(24))


@pytest.fixture(scope="module")
def realistic_six_hours():
    rf = syn.RealisticForcing(eta=160, xi=144, s_rho=12, n_frames=7, seed=31)
    win = rf.window()
    p = rf.release(8192, n_sources=32, seed=32)
    p["time"] = win.times[0]
    cfg = default_config(random=False, dti=15.0)
    return win, cfg, p, _oracle(win, cfg, p, range(6))


@pytest.mark.parametrize("storage,mean_max,p99_max,flip_m", [
    ("fp32", 0.05, 0.5, 1.0), ("fp16", 50.0, 200.0, None), ("bf16", 50.0, 200.0, None)])
@pytest.mark.parametrize("scene", ["analytic_day", "realistic_six_hours"])
def test_position_error_against_fp64_oracle(cuda_device, request, scene, storage, mean_max,
                                            p99_max, flip_m):
    win, cfg, p, want = request.getfixturevalue(scene)
    intervals = range(win.T - 1)
    with Engine(cuda_device, arithmetic="fp32", storage=storage) as e:
        got = _run(e, win, cfg, p, intervals)
    both = (got["health"] > 0) & (want["health"] > 0)
    flips = int(np.sum((got["health"] > 0) != (want["health"] > 0)))
    assert flips <= max(1, len(p) // 200), f"{flips} alive/dead decisions differ"
    err = great_circle_m(win.lon, win.lat, got[both], want[both])
    mean, p99, mx = float(err.mean()), float(np.percentile(err, 99)), float(err.max())
    decision = int(np.sum(err > flip_m)) if flip_m is not None else 0
    print(f"{scene} {storage}: mean {mean:.4g} m p99 {p99:.4g} m max {mx:.4g} m, "
          f"alive/dead flips {flips}, closure-decision divergences {decision}")
    assert mean <= mean_max and p99 <= p99_max, (mean, p99, mx)
    assert decision <= len(p) // 500, (decision, mx)


def test_reference_draws_in_fp32_mode_track_the_oracle(cuda_device):
    """With the reference random keys the FP32 step takes the same draws as the FP64 oracle, so
    a stochastic trajectory stays within FP32 rounding of it."""
    win = syn.config1_window(n_frames=3)
    p = syn.uniform_particles(4096, win.eta, win.xi, seed=9)
    cfg = default_config(random=True, horizontalClosure=1)
    want = _oracle(win, cfg, p, range(2))
    with Engine(cuda_device, arithmetic="fp32", rng="reference") as e:
        got = _run(e, win, cfg, p, range(2))
    d = max_abs_diff(got, want)
    assert d["i"] < 1e-4 and d["j"] < 1e-4 and d["k"] < 1e-4, d


@pytest.mark.parametrize("rng", ["reference", "philox"])
def test_diffusion_ensemble_moments(cuda_device, rng):
    """No current, constant diffusivity: after n substeps of dt=dti the horizontal displacement
    of each particle is sigma_k * sqrt(n) * N(0, 1) metres per axis (Particle.cpp:518-533), with
    sigma_k = sigma (1 - k/kLower) at the release depth (k stays put: w=0, AKT=0)."""
    win = syn.config1_window(n_frames=2, u=0.0, v=0.0, akt=0.0)
    n = 200000
    p = syn.uniform_particles(n, win.eta, win.xi, seed=4)
    p["i"], p["j"], p["k"] = 60.5, 60.5, 0.0
    cfg = default_config(random=True, horizontalClosure=1)
    with Engine(cuda_device, arithmetic="fp32", rng=rng) as e:
        got = _run(e, win, cfg, p, [0])
    steps = 120
    sigma_m = cfg.sigma * np.sqrt(steps)
    lat0 = np.radians(win.lat[60, 0])
    dx = 6371000.0 * np.radians(win.lon[0, 1] - win.lon[0, 0]) * np.cos(lat0)
    dy = 6371000.0 * np.radians(win.lat[1, 0] - win.lat[0, 0])
    x = (got["i"] - 60.5) * dx / sigma_m
    y = (got["j"] - 60.5) * dy / sigma_m
    for z in (x, y):
        assert abs(z.mean()) < 5 / np.sqrt(n)
        assert abs(z.var() - 1.0) < 0.02
        assert abs(np.mean(z ** 4) - 3.0) < 0.1
    assert abs(np.corrcoef(x, y)[0, 1]) < 0.01


@pytest.mark.parametrize("case_name", ["drift_i1", "drift_i2", "realistic_i2_c123"])
def test_fp32_step_on_reference_fixture_cases(cuda_device, case_name):
    """The FP32 step (drift model, diffusion with the reference draws, land and closures) over
    the fixture cases, two intervals, against the FP64 oracle."""
    from helpers import load_move_cases
    case = {c["name"]: c for c in load_move_cases()}[case_name]
    cfg = default_config(**case["overrides"])
    win = case["window"]
    want = _oracle(win, cfg, case["start"], range(2))
    with Engine(cuda_device, arithmetic="fp32") as e:
        got = _run(e, win, cfg, case["start"], range(2))
    assert np.array_equal(got["driftSide"], want["driftSide"])
    both = (got["health"] > 0) & (want["health"] > 0)
    flips = int(np.sum((got["health"] > 0) != (want["health"] > 0)))
    err = great_circle_m(win.lon, win.lat, got[both], want[both])
    print(f"{case_name}: mean {err.mean():.3g} m p99 {np.percentile(err, 99):.3g} m "
          f"max {err.max():.3g} m flips {flips}")
    assert flips <= max(2, len(got) // 100)
    assert err.mean() <= 0.1 and np.percentile(err, 99) <= 1.0


@pytest.mark.parametrize("random", [False, True])
def test_plain_drift_form_against_fp64_oracle(cuda_device, random):
    """The plain-drift form of the FP32 step (leeway regression in FP32, wind and Stokes from
    the environment pair, with and without the random walk under the reference draws) against
    the FP64 oracle: every catalogue object on both sides, six hours over the analytic grid with
    wind and Stokes fields on the rho nodes."""
    win = syn.config1_window(n_frames=7)
    env = syn.environment(win.times[0], 6, wind_n=60)
    with Engine(cuda_device, arithmetic="fp32") as e:
        e.load_window(win)
        e.set_geo_grid(win.lon, win.lat, win.sWValues)
        e.regrid_environment("wind", "curvilinear", *env["wind"])
        e.regrid_environment("stokes", "geographic", *env["stokes"])
        wind = [e.environment("wind", t) for t in range(win.T)]
        stokes = [e.environment("stokes", t) for t in range(win.T)]
    win.windU10 = np.ascontiguousarray([w[0] for w in wind])
    win.windV10 = np.ascontiguousarray([w[1] for w in wind])
    win.stokesU = np.ascontiguousarray([s[0] for s in stokes])
    win.stokesV = np.ascontiguousarray([s[1] for s in stokes])
    p = syn.uniform_particles(8192, win.eta, win.xi, seed=12)
    p["driftObjectType"] = 1 + np.arange(len(p)) % 22
    p["driftSide"] = np.where(np.arange(len(p)) % 3 == 0, 1, -1)
    cfg = default_config(random=random, driftModel=1, horizontalClosure=1, randomSeed=77)
    want = _oracle(win, cfg, p, range(6))
    with Engine(cuda_device, arithmetic="fp32") as e:
        got = _run(e, win, cfg, p, range(6))
    both = (got["health"] > 0) & (want["health"] > 0)
    err = great_circle_m(win.lon, win.lat, got[both], want[both])
    print(f"plain drift random={random}: mean {err.mean():.3g} m p99 "
          f"{np.percentile(err, 99):.3g} m max {err.max():.3g} m")
    assert np.array_equal(got["health"] > 0, want["health"] > 0)
    assert err.mean() <= 0.05 and np.percentile(err, 99) <= 0.5
