"""Device-side emission and geographic positions through the C ABI, against the oracle.

Emission (wacomm_b200_emit) must give, record for record, what the oracle's Sources::emit
restatement gives: release times (SourceEmission.hpp:38-79), the stable merge by time across
sources (Sources.cpp:233-249), ids last+1 onwards, sides and every other field bit for bit
(Source.cpp:25-45). The seeded position offsets 0.25 N(0,1) go through log, sqrt and cos, whose
CUDA and glibc results may differ in the last bit; positions with offsets are therefore held to
2 ulp of the position, and to bit equality without them. Geographic positions (wacomm_b200_geo_positions) must equal the oracle's
kji2deplatlon (OceanModelAdapter.cpp:271-327) bit for bit, the off-grid marker included.
"""
import numpy as np
import pytest

from oracle import bindings as ob
from test_oracle_emission import mixed_sources
from wacommplusplus_b200 import synthetic as syn
from wacommplusplus_b200._native import ERR_ARGUMENT, WacommError
from wacommplusplus_b200.engine import Engine
from wacommplusplus_b200.types import default_config, make_particles, make_sources

pytestmark = pytest.mark.gpu

DAY = 86400.0


def same_records(a, b, position_ulps=0):
    """Bit equality of every field (record padding is not compared); with position_ulps > 0,
    k, j and i within that many ulp of max(|expected|, 1)."""
    if len(a) != len(b):
        return False
    for f in a.dtype.names:
        if position_ulps and f in ("k", "j", "i"):
            if np.any(np.abs(a[f] - b[f]) > position_ulps * np.spacing(np.maximum(np.abs(b[f]), 1.0))):
                return False
        elif a[f].tobytes() != b[f].tobytes():
            return False
    return True


@pytest.fixture(scope="module")
def engine(cuda_device):
    e = Engine(cuda_device)
    yield e
    e.close()


def emit_times(engine, mode, value, s0, s1, i0, i1):
    """The release times of one source through the engine (sourceEmissionTimes' arguments in
    seconds; the source record holds days)."""
    engine.set_config(default_config(randomSources=False))
    engine.set_particles(make_particles(0))
    src = make_sources([(0.0, 1.5, 1.5, s0 / DAY if s0 >= 0 else s0,
                         s1 / DAY if s1 >= 0 else s1, value, mode)])
    n = engine.emit(src, i0, i1)
    recs = engine.get_particles()
    assert len(recs) == n
    return recs["time"]


def test_release_times_known_answers(engine):
    # tests/SourceEmissionTest.cpp through the device path
    U, B, P = "uniform_rate", "forcing_interval_batch", "single_pulse"
    hourly = emit_times(engine, U, 1000, 0, -1, 0, 3600)
    assert len(hourly) == 1000
    assert abs(hourly[0] - 1.8) < 1e-12 and abs(hourly[-1] - 3598.2) < 1e-9
    gap = emit_times(engine, U, 1000, 0, -1, 3600, 10800)
    assert len(gap) == 2000
    assert abs(gap[0] - 3601.8) < 1e-9 and abs(gap[-1] - 10798.2) < 1e-9
    a, b = emit_times(engine, U, 7, 0, -1, 0, 450), emit_times(engine, U, 7, 0, -1, 450, 3600)
    assert len(a) + len(b) == 7
    assert list(np.concatenate([a, b])) == list(emit_times(engine, U, 7, 0, -1, 0, 3600))
    bounded = emit_times(engine, U, 10, 900, 2700, 0, 3600)
    assert len(bounded) == 5 and all(900 <= t < 2700 for t in bounded)
    legacy = emit_times(engine, B, 1000, 0, -1, 0, 7200)
    assert len(legacy) == 1000 and all(t == 0 for t in legacy)
    instant = emit_times(engine, B, 4, 3600, 3600, 3600, 7200)
    assert len(instant) == 4 and all(t == 3600 for t in instant)
    assert len(emit_times(engine, B, 4, 3600, 3600, 7200, 10800)) == 0
    assert len(emit_times(engine, B, 4, 3600, 3600, 0, 3600)) == 0
    assert len(emit_times(engine, B, 4, 0, 7200, 7200, 10800)) == 4
    assert len(emit_times(engine, B, 4, 0, 1800, 3600, 7200)) == 0
    assert len(emit_times(engine, B, 4, 3600.00001, 3600.00001, 3600, 7200)) == 4
    assert len(emit_times(engine, B, 4, 3599.99999, 3599.99999, 3600, 7200)) == 4
    pulse = emit_times(engine, P, 25, 1800, -1, 0, 3600)
    assert len(pulse) == 25 and all(t == 1800 for t in pulse)
    assert len(emit_times(engine, P, 25, 1800, -1, 1800, 3600)) == 25
    assert len(emit_times(engine, P, 25, 1800, -1, 0, 1800)) == 0


def test_release_times_match_the_fixture_schedules(engine):
    """Every schedule of the committed sourceEmissionTimes fixture, bit for bit."""
    import json
    import os
    from helpers import GOLDEN
    with open(os.path.join(GOLDEN, "emission.json")) as fh:
        cases = json.load(fh)
    engine.set_config(default_config(randomSources=False))
    checked = 0
    for c in cases:
        s0, s1 = c["source"]
        # the device record holds days; keep the cases whose seconds survive the round trip
        if (s0 >= 0 and (s0 / DAY) * DAY != s0) or (s1 >= 0 and (s1 / DAY) * DAY != s1):
            continue
        engine.set_particles(make_particles(0))
        src = make_sources([(0.0, 1.5, 1.5, s0 / DAY if s0 >= 0 else -1.0,
                             s1 / DAY if s1 >= 0 else -1.0, c["value"], c["mode"])])
        if c["times"] is None:
            with pytest.raises(WacommError) as err:
                engine.emit(src, *c["interval"])
            assert err.value.code == ERR_ARGUMENT
            assert engine.count() == 0
        else:
            engine.emit(src, *c["interval"])
            assert [t.hex() for t in engine.get_particles()["time"]] == c["times"], c
        checked += 1
    assert checked >= len(cases) // 2


@pytest.mark.parametrize("random_sources,random_side", [(False, False), (True, True)])
def test_merged_emission_matches_oracle(engine, random_sources, random_side):
    cfg = default_config(randomSources=random_sources, leewayRandomSide=random_side,
                         driftObjectType=3, driftSide=1, leewayRightSideProbability=0.3)
    engine.set_config(cfg)
    src = mixed_sources()
    # resident records whose last id (not the largest) decides the next id
    resident = make_particles(3, ids=np.array([5, 1000, 3], np.uint64))
    engine.set_particles(resident)
    expected = [resident]
    last = 3
    for t0, t1 in [(0.0, 3600.0), (3600.0, 7200.0), (7200.0, 9000.0), (1800.0, 5400.0)]:
        n = engine.emit(src, t0, t1)
        want = ob.sources_emit(cfg, src, 0.0, t0, t1, last + 1)
        assert n == len(want) > 0
        expected.append(want)
        last = int(want["id"][-1])
    got = engine.get_particles()
    want = np.concatenate(expected)
    assert same_records(got, want, position_ulps=2 if random_sources else 0)


def test_emission_with_the_run_start_and_empty_set(engine):
    cfg = default_config(randomSources=True)
    engine.set_config(cfg)
    engine.set_particles(make_particles(0))
    julian = 19000.25  # start < 0 takes the run start, in days
    src = make_sources([(-0.1, 4.5, 5.5, -1, -1, 360, "uniform_rate"),
                        (-0.2, 6.5, 7.5, julian + 0.5 / 24, -1, 9, "single_pulse")])
    t0 = julian * DAY
    n = engine.emit(src, t0, t0 + 3600.0, julian_start=julian)
    want = ob.sources_emit(cfg, src, julian, t0, t0 + 3600.0, 0)
    assert n == len(want) == 369
    assert same_records(engine.get_particles(), want, position_ulps=2)
    assert engine.get_particles()["id"][0] == 0


def test_invalid_schedule_appends_nothing(engine):
    engine.set_config(default_config())
    engine.set_particles(make_particles(4))
    bad = make_sources([(0, 1.5, 1.5, 0, -1, 10, "uniform_rate"),
                        (0, 1.5, 1.5, 0, -1, 2.5, "single_pulse")])
    with pytest.raises(WacommError) as err:
        engine.emit(bad, 0.0, 3600.0)
    assert err.value.code == ERR_ARGUMENT
    assert engine.count() == 4
    with pytest.raises(WacommError):
        engine.emit(bad[:1], 3600.0, 3600.0)  # empty interval
    assert engine.emit(bad[:0], 0.0, 3600.0) == 0


def test_large_emission_matches_oracle(engine):
    """64 sources at 2000 particles per hour each, with ties between equal schedules: 128,000
    records in one call, merged by the device in stable time order."""
    cfg = default_config(randomSources=True, leewayRandomSide=True)
    engine.set_config(cfg)
    engine.set_particles(make_particles(0))
    rng = np.random.default_rng(11)
    rows = []
    for s in range(64):
        start = 0.0 if s % 4 else 1800.0 / DAY   # groups share starts and rates: equal times
        rows.append((-rng.uniform(0, 1), rng.uniform(5, 50), rng.uniform(5, 50), start, -1,
                     2000.0 if s % 2 else 1000.0 * (1 + s % 3), "uniform_rate"))
    src = make_sources(rows)
    n = engine.emit(src, 0.0, 3600.0)
    want = ob.sources_emit(cfg, src, 0.0, 0.0, 3600.0, 0)
    assert n == len(want) > 100000
    got = engine.get_particles()
    assert same_records(got, want, position_ulps=2)


def test_geo_positions_match_oracle(engine):
    forcing = syn.RealisticForcing(eta=96, xi=80, s_rho=12, n_frames=2, seed=4)
    win = forcing.window()
    engine.load_window(win)
    engine.set_geo_grid(win.lon, win.lat, win.sWValues)
    rng = np.random.default_rng(5)
    n = 50000
    recs = make_particles(n, k=rng.uniform(-win.sW + 0.5, 0.2, n), j=rng.uniform(-2, win.eta + 1, n),
                          i=rng.uniform(-2, win.xi + 1, n))
    recs["k"][:100] = 0.0
    recs["k"][100:200] = -(win.sW - 2)
    recs["k"][200:210] = np.nan
    engine.set_particles(recs)
    dep, lat, lon = engine.geo_positions()
    grid = type("G", (), dict(eta=win.eta, xi=win.xi, sW=win.sW, lon=win.lon, lat=win.lat,
                             h=win.h, sWValues=win.sWValues))
    want = np.array([ob.kji2deplatlon(grid, r["k"], r["j"], r["i"]) for r in recs])
    assert np.array_equal(dep, want[:, 0]) and np.array_equal(lat, want[:, 1])
    assert np.array_equal(lon, want[:, 2])
    off = dep == 1e37
    assert 0 < off.sum() < n  # both branches exercised
    assert np.all(off[200:210])
