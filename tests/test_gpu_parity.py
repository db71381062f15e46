"""Parity of the B200 kernels with the oracle, through the C ABI.

Reference arithmetic (ARITH_REFERENCE) must reproduce the oracle to round-off: positions within
1e-9 degrees (the FP64-mode bound of the precision targets) and, for 99% of the particles, within
1e-12 grid-index units; health within a few ulp; drift sides and alive/dead status exactly;
concentration counts bit-exactly given the positions.

Why not bit-exact everywhere: CUDA's and glibc's sin/cos/atan2/exp differ in the last bit, so
the cell metric (and with it a position) can differ by ~1e-16; the reference rounds each bilinear
corner term to float (Particle.cpp:356-377), and once in a few million terms that tiny input
difference moves a product across a float rounding boundary: a one-ulp float velocity change,
a few 1e-9 grid units after the step. The reference's own CPU/GPU snapshot tolerance for the
same effect is 1e-8 index units (tools/performance_evidence.py:10-11).
"""
import ctypes

import numpy as np
import pytest

from helpers import load_move_cases, max_abs_diff, records_equal
from kats import concentration_kat, particle_move_kats
from oracle import bindings as ob
from wacommplusplus_b200 import synthetic as syn
from wacommplusplus_b200.engine import Engine
from wacommplusplus_b200.types import default_config

pytestmark = pytest.mark.gpu

HEALTH_TOL = 1e-15


class EngineMover:
    """Runs one interval through the engine the way the reference calls Particle::move."""

    def __init__(self, engine):
        self.engine = engine
        self.loaded = None

    def __call__(self, cfg, records, window, time_index):
        e = self.engine
        if self.loaded is not window:
            e.load_window(window)
            self.loaded = window
        e.set_config(cfg)
        e.set_particles(records)
        e.move_interval(time_index)
        out = e.get_particles()
        records[:] = out
        return records


@pytest.fixture(scope="module")
def engine_host(cuda_device):
    with Engine(cuda_device, semantics="host", arithmetic="reference") as e:
        yield e


@pytest.fixture(scope="module")
def engine_device(cuda_device):
    with Engine(cuda_device, semantics="device", arithmetic="reference") as e:
        yield e


def degrees_per_index(win):
    return max(float(np.abs(np.diff(win.lon, axis=1)).max()),
               float(np.abs(np.diff(win.lat, axis=0)).max()))


def assert_close(got, want, win, what="", max_deg=1e-9, p99_index=1e-12):
    assert len(got) == len(want)
    assert np.array_equal(got["id"], want["id"])
    assert np.array_equal(got["health"] > 0, want["health"] > 0), what
    assert np.array_equal(got["driftSide"], want["driftSide"]), what
    d = max_abs_diff(got, want)
    deg = degrees_per_index(win)
    assert max(d["i"], d["j"]) * deg <= max_deg and d["k"] <= max_deg / deg, (what, d)
    err = np.maximum(np.abs(got["i"] - want["i"]), np.abs(got["j"] - want["j"]))
    err = np.nan_to_num(err, nan=0.0)
    assert np.percentile(err, 99) <= p99_index, (what, float(np.percentile(err, 99)))
    assert d["age"] <= 1e-9, (what, d)
    rel = np.abs(got["health"] - want["health"]) / np.maximum(1.0, np.abs(want["health"]))
    assert np.nanmax(rel) <= HEALTH_TOL * 8, (what, d)


def test_known_answers_host_rules(engine_host):
    assert particle_move_kats(EngineMover(engine_host)) > 40


def test_known_answers_device_rules(engine_device):
    assert particle_move_kats(EngineMover(engine_device)) > 40


def test_concentration_known_answer(engine_host):
    def count(records, t, n_times, s_rho, eta, xi):
        e = engine_host
        win = syn.config1_window(n_frames=1, eta=eta, xi=xi, s_rho=s_rho)
        e.load_window(win)
        e.set_config(default_config())
        e.set_particles(records)
        e.concentration_reset(n_times)
        e.concentration_count(t)
        return e.concentration()
    assert concentration_kat(count) == 2


@pytest.mark.parametrize("case", load_move_cases(), ids=lambda c: c["name"])
@pytest.mark.parametrize("rules", ["host", "device"])
def test_fixture_cases_reference_arithmetic(case, rules, engine_host, engine_device):
    engine = engine_host if rules == "host" else engine_device
    sem = ob.SEMANTICS_HOST if rules == "host" else ob.SEMANTICS_DEVICE
    cfg = default_config(**case["overrides"])
    win = case["window"]
    engine.load_window(win)
    engine.set_config(cfg)
    engine.set_particles(case["start"])
    want = case["start"].copy()
    for t in (0, 1):
        engine.move_interval(t)
        ob.oracle_move(cfg, want, win, t, sem, threads=1)
        assert_close(engine.get_particles(), want, win, what=f"{case['name']} t={t}")
    if rules == "host":
        assert_close(engine.get_particles(), case["after2"], win, what="vs reference fixture")
    cfg.trackingDirection = -1
    engine.set_config(cfg)
    engine.move_interval(win.T - 1)
    ob.oracle_move(cfg, want, win, win.T - 1, sem, threads=1)
    assert_close(engine.get_particles(), want, win, what=f"{case['name']} backward")


def test_concentration_float_land_mask(engine_host):
    """The float concentration grid with the land mask (Wacomm.cpp:188-196,724-737): counts as
    float in water, 1e37 in every level of each land cell of the concentration times evaluated,
    times never evaluated left at 0; equal, value for value, to the oracle's restatement applied
    to the oracle's count of the kernel's own positions."""
    win = syn.config1_window(n_frames=6, eta=64, xi=64, s_rho=10)
    land = np.zeros((win.eta, win.xi), dtype=bool)
    land[20:30, 40:52] = True
    land[50:, :6] = True
    win.mask = np.where(land, 0.0, 1.0)
    win.h = np.where(land, 0.0, win.h)
    p0 = syn.uniform_particles(8192, win.eta, win.xi, seed=7)
    wet = ~land[np.floor(p0["j"]).astype(int), np.floor(p0["i"]).astype(int)]
    wet &= ~land[np.floor(p0["j"]).astype(int) + 1, np.floor(p0["i"]).astype(int) + 1]
    p0 = p0[wet]
    e = engine_host
    e.load_window(win)
    e.set_config(default_config(random=True))
    e.set_particles(p0)
    e.concentration_reset(win.T)
    e.move_interval(0)
    e.move_interval(1)
    got = e.get_particles()
    counts = e.concentration()
    assert np.array_equal(counts[2], ob.oracle_concentration(got, 2, win.T, win)[2])
    plain = e.concentration_float(mask_land=False)
    assert np.array_equal(plain, counts.astype(np.float32))
    masked = e.concentration_float(mask_land=True)
    want = ob.oracle_concentration_float(counts, [1, 2], win)
    assert np.array_equal(masked, want)
    assert np.all(masked[1:3][:, :, land] == np.float32(1e37))
    assert np.all(masked[[0, 3, 4, 5]] == 0)
    assert masked[1:3][:, :, ~land].sum() > 0


def _config1(n_particles=16384, frames=6):
    win = syn.config1_window(n_frames=frames)
    return win, syn.uniform_particles(n_particles, win.eta, win.xi, seed=1)


@pytest.mark.parametrize("arithmetic", ["reference", "fp32"])
def test_config1_forward_backward(cuda_device, arithmetic):
    """Plain analytic case: 16,384 particles, 5 intervals forward then back, midpoint, no
    diffusion; concentration counted in the move kernel equals the oracle's count of the
    kernel's own positions."""
    win, p0 = _config1()
    cfg = default_config(random=False)
    with Engine(cuda_device, arithmetic=arithmetic) as e:
        e.load_window(win)
        e.set_config(cfg)
        e.set_particles(p0)
        e.concentration_reset(win.T)
        want = p0.copy()
        for t in range(win.T - 1):
            e.move_interval(t)
            ob.oracle_move(cfg, want, win, t, threads=0)
        got = e.get_particles()
        if arithmetic == "reference":
            assert_close(got, want, win, what="config 1 forward")
        else:
            assert np.array_equal(got["health"] > 0, want["health"] > 0)
            d = max_abs_diff(got, want)
            assert max(d["i"], d["j"], d["k"]) <= 1e-5, d
        conc = e.concentration()
        assert np.array_equal(conc[win.T - 1], ob.oracle_concentration(got, win.T - 1, win.T, win)[win.T - 1])
        # backward from the end state returns to the release points of the survivors
        cfg.trackingDirection = -1
        e.set_config(cfg)
        back_want = want.copy()
        for t in range(win.T - 1, 0, -1):
            e.move_interval(t)
            ob.oracle_move(cfg, back_want, win, t, threads=0)
        back = e.get_particles()
        if arithmetic == "reference":
            assert_close(back, back_want, win, what="config 1 backward")
        else:
            d = max_abs_diff(back, back_want)
            assert max(d["i"], d["j"]) <= 1e-5, d
        # 0.2 m/s east and 0.1 m/s north move a particle ~27 and ~14 cells in 5 h; those released
        # far enough from the east and north edges never meet a closure
        inside = (back_want["health"] > 0) & (p0["i"] < win.xi - 36) & (p0["j"] < win.eta - 20)
        assert inside.sum() > 5000
        assert np.abs(back["i"][inside] - p0["i"][inside]).max() < 1e-6
        assert np.abs(back["j"][inside] - p0["j"][inside]).max() < 1e-6


def test_chunked_and_unsorted_launches_are_identical(cuda_device):
    cases = {c["name"]: c for c in load_move_cases()}
    case = cases["drift_i2"]
    cfg = default_config(**case["overrides"])
    outs = []
    for opts in (dict(), dict(substeps_per_launch=7), dict(sort_by_cell=0),
                 dict(block_size=64, substeps_per_launch=50)):
        with Engine(cuda_device, arithmetic="reference", **opts) as e:
            e.load_window(case["window"])
            e.set_config(cfg)
            e.set_particles(case["start"])
            e.move_interval(0)
            e.move_interval(1)
            outs.append(e.get_particles())
    for o in outs[1:]:
        assert records_equal(o, outs[0])


def test_host_buffer_entry_matches_resident_path(cuda_device):
    win, p0 = _config1(n_particles=50000, frames=3)
    cfg = default_config(random=True)
    with Engine(cuda_device, arithmetic="reference") as e:
        e.load_window(win)
        e.set_config(cfg)
        e.set_particles(p0)
        e.move_interval(0)
        resident = e.get_particles()
        host = p0.copy()
        e.move_interval_host(0, host)
        assert records_equal(host, resident)


@pytest.mark.parametrize("n", [2_200_000, 4_500_001, 9_000_000])
def test_host_buffer_slabs_match_resident_path(cuda_device, n):
    """Every slab layout of the host-buffer entry (two slabs; end slabs ramping up to one or
    several middle slabs) gives the resident path's records and concentration."""
    win = syn.config1_window(n_frames=3)
    p0 = syn.uniform_particles(n, win.eta, win.xi, seed=8)
    cfg = default_config(random=True, randomSeed=4)
    with Engine(cuda_device, arithmetic="fp32", rng="philox") as e:
        e.load_window(win)
        e.set_config(cfg)
        e.concentration_reset(win.T)
        e.set_particles(p0)
        e.move_interval(0)
        resident, conc = e.get_particles(), e.concentration()
        e.concentration_reset(win.T)
        host = p0.copy()
        e.move_interval_host(0, host)
        assert e.stats()["particle_steps"] == 120 * n
        assert records_equal(host, resident)
        assert np.array_equal(e.concentration(), conc)


def test_sort_sequences_across_host_and_resident_intervals(cuda_device):
    """Each sort walks the order the previous sort of the same records left (per slab on the host
    path, whole on the resident one); switching between the two paths, and a graph captured while
    the sequence held the other layout, still give the records of resident intervals alone."""
    n = 4_500_001
    win = syn.config1_window(n_frames=6)
    p0 = syn.uniform_particles(n, win.eta, win.xi, seed=9)
    with Engine(cuda_device, arithmetic="fp32") as e:
        e.load_window(win)
        e.set_config(default_config(random=False))
        e.set_particles(p0)
        for t in range(5):
            e.move_interval(t)
        want = e.get_particles()
        host = p0.copy()
        e.move_interval_host(0, host)
        e.move_interval_host(1, host)  # each slab walks its own order from interval 0
        e.set_particles(host)
        e.move_interval(2)  # the slab orders do not cover the whole population: slot order
        after2 = e.get_particles()
        e.graph_capture(3, 1)
        scratch = after2.copy()
        e.move_interval_host(3, scratch)  # the sequence holds slab orders again
        e.set_particles(after2)
        e.graph_launch()
        assert records_equal(e.get_particles(), scratch)
        e.move_interval(4)  # walks the order the graph's sort left
        assert records_equal(e.get_particles(), want)
        e.graph_release()


def test_remove_dead_keeps_order(cuda_device):
    win = syn.config1_window(n_frames=2)
    p = syn.uniform_particles(1000, win.eta, win.xi, seed=3)
    p["health"][::3] = -1.0
    with Engine(cuda_device) as e:
        e.load_window(win)
        e.set_config(default_config())
        e.set_particles(p)
        e.remove_dead()
        got = e.get_particles()
    assert np.array_equal(got, p[p["health"] > 0])


def test_unknown_drift_object_is_an_error_under_host_rules(cuda_device):
    win = syn.config1_window(n_frames=2)
    p = syn.uniform_particles(64, win.eta, win.xi, seed=3)
    p["driftObjectType"] = 40
    p["driftSide"] = 1
    cfg = default_config(driftModel=1, windU10=5.0)
    with Engine(cuda_device, arithmetic="reference") as e:
        e.load_window(win)
        e.set_config(cfg)
        e.set_particles(p)
        e.move_interval(0)
        with pytest.raises(RuntimeError, match="catalogue"):
            e.synchronize()


@pytest.mark.parametrize("form", ["fp32", "fp32_random_walk", "walk"])
def test_survival_threshold_crossed_inside_the_interval(cuda_device, form):
    """Particles whose age crosses the survival threshold (exp(-age/tau0) = survprob) at every
    substep of the interval: each dies at the substep the oracle's survival test kills it, so
    alive/dead status, age (which stops at death) and health agree. The FP32 step and the walk
    kernel skip the lazy survival tests while the outcome cannot change; this holds them to the
    oracle where it does."""
    win = syn.config1_window(n_frames=2)
    cfg = default_config(random=form != "fp32", randomSeed=7, tau0=86400.0, survprob=1e-4)
    kill = -86400.0 * np.log(1e-4)
    n = 8192
    p = syn.uniform_particles(n, win.eta, win.xi, time=win.times[0], seed=31)
    rng = np.random.default_rng(32)
    p["age"] = kill - rng.uniform(-60.0, 7200.0, n)   # dies before, during or after the hour
    p["age"][:64] = rng.uniform(0.0, 1000.0, 64)      # young ones too
    p["health"] = np.exp(-p["age"] / 86400.0)
    if form == "walk":
        e = Engine(0, arithmetic="fp32", storage="fp32", surrogate=1)
        e.set_config(cfg)
        e.load_window(win)
        e.set_surrogate()
    else:
        e = Engine(0, arithmetic="fp32", storage="fp32")
        e.set_config(cfg)
        e.load_window(win)
    e.set_particles(p)
    e.move_interval(0)
    got = e.get_particles()
    e.close()
    want = ob.oracle_move(cfg, p.copy(), win, 0, ob.SEMANTICS_HOST, threads=0)
    alive = want["health"] > 0
    assert 0.3 < alive.mean() < 0.7
    assert np.array_equal(got["health"] > 0, alive)
    assert np.allclose(got["age"], want["age"], rtol=0, atol=1e-9)
    assert np.allclose(got["health"][alive], want["health"][alive], rtol=1e-12, atol=0)
