"""Captured runs (wacomm_b200_graph_capture / graph_launch) and the launch autotuner.

A run of intervals recorded as one CUDA graph must give the records, the concentration grid and
the particle-step count of the same intervals run one call at a time, bit for bit, and a relaunch
on a new batch of the same size must equal an eager run of that batch. A launch after a change the
graph cannot see (particle count, config) is refused. The autotuner leaves records and
concentration as they were and only changes the launch configuration.
"""
import numpy as np
import pytest

from wacommplusplus_b200 import synthetic as syn
from wacommplusplus_b200._native import WacommError
from wacommplusplus_b200.engine import Engine
from wacommplusplus_b200.types import default_config

pytestmark = pytest.mark.gpu

INTERVALS = 4


@pytest.fixture(scope="module")
def setting():
    win = syn.config1_window(n_frames=INTERVALS + 2)
    env = syn.environment(win.times[0], INTERVALS + 1, wind_n=80)
    cfg = default_config(random=True, randomSeed=17, driftModel=1)
    return win, env, cfg


def batch(n, seed, win):
    p = syn.uniform_particles(n, win.eta, win.xi, seed=seed)
    rng = np.random.default_rng(seed)
    p["driftObjectType"] = rng.integers(0, 23, n)
    p["driftSide"] = rng.choice([-1, 1], n)
    p["time"] = win.times[0] + rng.uniform(0, 2 * 3600.0, n)  # staggered releases
    return p


def engine(win, env, cfg, particles):
    e = Engine(0, arithmetic="fp32", storage="fp32")
    e.set_config(cfg)
    e.load_window(win)
    e.set_geo_grid(win.lon, win.lat, win.sWValues)
    e.regrid_environment("wind", "curvilinear", *env["wind"])
    e.regrid_environment("stokes", "geographic", *env["stokes"])
    e.concentration_reset(win.T)
    e.set_particles(particles)
    return e


def eager(e):
    steps = 0.0
    for t in range(INTERVALS):
        e.move_interval(t)
        steps += e.stats()["particle_steps"]
    return steps


def same(a, b):
    pa, pb = a.get_particles(), b.get_particles()
    for f in pa.dtype.names:
        assert pa[f].tobytes() == pb[f].tobytes(), f
    assert np.array_equal(a.concentration(), b.concentration())


def test_graph_equals_eager_and_relaunches_on_a_new_batch(cuda_device, setting):
    win, env, cfg = setting
    first, second = batch(30000, 1, win), batch(30000, 2, win)
    ref = engine(win, env, cfg, first)
    ref_steps = eager(ref)
    g = engine(win, env, cfg, first)
    g.graph_capture(0, INTERVALS)
    g.graph_launch()
    g.synchronize()
    assert g.stats()["particle_steps"] == ref_steps > 0
    # the device-side running totals agree with the per-interval counts
    assert g.steps_total() == ref_steps and ref.steps_total(reset=True) == ref_steps
    assert ref.steps_total() == 0
    same(g, ref)
    # a new batch of the same size through the same graph
    ref.set_particles(second)
    ref.concentration_reset(win.T)
    eager(ref)
    g.set_particles(second)
    g.concentration_reset(win.T)
    g.graph_launch()
    g.synchronize()
    same(g, ref)
    ref.close()
    g.close()


def test_graph_launch_refused_after_changes(cuda_device, setting):
    win, env, cfg = setting
    g = engine(win, env, cfg, batch(5000, 3, win))
    g.graph_capture(0, INTERVALS)
    g.set_particles(batch(4000, 4, win))
    with pytest.raises(WacommError):
        g.graph_launch()
    g.set_particles(batch(5000, 4, win))
    g.graph_launch()
    g.synchronize()
    g.set_config(default_config(random=True, randomSeed=18, driftModel=1))
    with pytest.raises(WacommError):
        g.graph_launch()
    g.graph_release()
    with pytest.raises(WacommError):
        g.graph_launch()
    g.set_options(surrogate=1)
    with pytest.raises(WacommError):
        g.graph_capture(0, 2)   # the surrogate option without weights
    g.close()


@pytest.mark.parametrize("random", [False, True])
def test_graph_of_surrogate_intervals_equals_eager(cuda_device, random):
    """The learned form needs no host round trip inside an interval (the fallback step reads
    its list length on the device), so its intervals are captured too: deterministic (closed-form
    displacement) and diffusive (the plain stochastic operator per substep), with fallback
    particles (drifting objects) in the same run; captured equals eager bit for bit."""
    win = syn.config1_window(n_frames=INTERVALS + 2)
    cfg = default_config(random=random, randomSeed=23, driftModel=1, windU10=6.0, windV10=-2.0,
                         hasWind=True)
    parts = batch(30000, 8, win)
    parts["driftObjectType"][parts["driftObjectType"] % 3 != 0] = 0  # two thirds passive

    def build():
        e = Engine(0, arithmetic="fp32", storage="fp16", surrogate=1, rng="philox")
        e.set_config(cfg)
        e.load_window(win)
        e.set_surrogate()
        e.concentration_reset(win.T)
        e.set_particles(parts)
        return e

    ref = build()
    ref_steps = eager(ref)
    sst = ref.surrogate_stats()
    assert sst["fallback"] > 0 and sst["run"] > 0
    g = build()
    g.graph_capture(0, INTERVALS)
    g.graph_launch()
    g.synchronize()
    assert g.stats()["particle_steps"] == ref_steps > 0
    assert g.surrogate_stats()["run"] == sst["run"]
    same(g, ref)
    ref.close()
    g.close()


def test_autotune_changes_only_the_launch_shape(cuda_device, setting):
    win, env, cfg = setting
    e = engine(win, env, cfg, batch(40000, 5, win))
    e.move_interval(0)
    before, conc = e.get_particles(), e.concentration()
    shape, ms = e.autotune(1)
    assert shape in (0, 1, 2, 3) and ms > 0
    assert e.options().launch_shape == shape
    assert e.options().particles_per_thread in (1, 2, 4)  # chosen after the shape
    assert e.options().sort_by_cell in (1, 2, 4)  # the sort cadence chosen after the shape
    after = e.get_particles()
    for f in before.dtype.names:
        assert before[f].tobytes() == after[f].tobytes(), f
    assert np.array_equal(conc, e.concentration())
    e.close()


def test_graph_of_chunked_launches_and_full_drift_form(cuda_device, setting):
    """Intervals split into launches of 40 substeps, with the wind-error field and the leeway
    coefficient ensemble on (the full form of the FP32 step): captured equals eager."""
    win, env, _ = setting
    cfg = default_config(random=True, randomSeed=5, driftModel=1, windErrorStdDev=1.0,
                         windErrorComponentCorrelation=0.3, leewayCoefficientEnsemble=True,
                         leewayResidualCorrelation=-0.35)
    parts = batch(20000, 6, win)
    ref = engine(win, env, cfg, parts)
    ref.set_options(substeps_per_launch=40)
    ref_steps = eager(ref)
    g = engine(win, env, cfg, parts)
    g.set_options(substeps_per_launch=40)
    g.graph_capture(0, INTERVALS)
    g.graph_launch()
    g.synchronize()
    assert g.stats()["particle_steps"] == ref_steps > 0
    same(g, ref)
    ref.close()
    g.close()


def test_autotune_block_size_under_reference_arithmetic(cuda_device, setting):
    win, env, cfg = setting
    e = Engine(0, arithmetic="reference")
    e.set_config(cfg)
    e.load_window(win)
    e.concentration_reset(win.T)
    e.set_particles(batch(20000, 7, win))
    before, conc = e.get_particles(), e.concentration()
    size, ms = e.autotune(1)
    assert size in (64, 128, 192, 256) and ms > 0
    assert e.options().block_size == size
    after = e.get_particles()
    for f in before.dtype.names:
        assert before[f].tobytes() == after[f].tobytes(), f
    assert np.array_equal(conc, e.concentration())
    e.close()


@pytest.mark.parametrize("surrogate", [False, True])
def test_sort_cadence_changes_only_the_work_order(cuda_device, setting, surrogate):
    """Sorting every N-th interval (options.sort_by_cell = N) only changes the order the work is
    taken in: every particle is moved on its own, so the records, the concentration and the
    particle-step count equal those of sorting every interval, bit for bit, for the plain step
    (leeway drift, random walk) and for the learned form's walk kernel."""
    win, env, cfg = setting
    parts = batch(30000, 9, win)
    if surrogate:
        parts["driftObjectType"][:] = 0
    results = []
    for cadence in (1, 3, 0):
        if surrogate:
            e = Engine(0, arithmetic="fp32", storage="fp16", surrogate=1, rng="philox",
                       sort_by_cell=cadence)
            e.set_config(default_config(random=True, randomSeed=31))
            e.load_window(win)
            e.set_surrogate()
            e.concentration_reset(win.T)
            e.set_particles(parts)
        else:
            e = engine(win, env, cfg, parts)
            e.set_options(sort_by_cell=cadence)
        steps = eager(e)
        results.append((e.get_particles(), e.concentration(), steps))
        e.close()
    for got, conc, steps in results[1:]:
        for f in got.dtype.names:
            assert got[f].tobytes() == results[0][0][f].tobytes(), f
        assert np.array_equal(conc, results[0][1]) and steps == results[0][2]


def test_particles_per_thread_changes_only_the_grid(cuda_device, setting):
    """Several work items per thread (options.particles_per_thread) shrink the grid of the FP32
    step and stride each block over it: every particle is moved on its own, so the records, the
    concentration and the particle-step count equal one item per thread's, bit for bit, eager and
    captured; values outside 1..16 are refused."""
    win, env, cfg = setting
    parts = batch(30001, 12, win)   # not a multiple of any block
    results = []
    for per in (1, 2, 4, 16):
        e = engine(win, env, cfg, parts)
        e.set_options(particles_per_thread=per)
        steps = eager(e)
        results.append((e.get_particles(), e.concentration(), steps))
        e.close()
    for got, conc, steps in results[1:]:
        for f in got.dtype.names:
            assert got[f].tobytes() == results[0][0][f].tobytes(), f
        assert np.array_equal(conc, results[0][1]) and steps == results[0][2]
    g = engine(win, env, cfg, parts)
    g.set_options(particles_per_thread=4)
    g.graph_capture(0, INTERVALS)
    g.graph_launch()
    g.synchronize()
    assert g.stats()["particle_steps"] == results[0][2]
    pg = g.get_particles()
    for f in pg.dtype.names:
        assert pg[f].tobytes() == results[0][0][f].tobytes(), f
    for bad in (0, 17):
        with pytest.raises(WacommError):
            g.set_options(particles_per_thread=bad)
    g.close()
