"""The oracle's emission (Sources::emit, Sources.cpp:233-249) on the CPU.

* sourceEmissionTimes restated against the assertions of the reference's
  tests/SourceEmissionTest.cpp;
* the merged multi-source emission (ids last+1 in stable time order, seeded offsets, sides)
  against the reference's own helpers compiled from its sources (oracle/_ref), composed the way
  Sources::emit composes them.
"""
import numpy as np
import pytest

from oracle import bindings as ob
from wacommplusplus_b200.types import SOURCE_DTYPE, default_config, make_sources

U, B, P = 0, 1, 2  # uniform_rate, forcing_interval_batch, single_pulse


def times(mode, value, s0, s1, i0, i1):
    return ob.emission_times("oracle", mode, value, s0, s1, i0, i1)


def test_source_emission_known_answers():
    # tests/SourceEmissionTest.cpp
    hourly = times(U, 1000, 0, -1, 0, 3600)
    assert len(hourly) == 1000
    assert abs(hourly[0] - 1.8) < 1e-12 and abs(hourly[-1] - 3598.2) < 1e-9
    gap = times(U, 1000, 0, -1, 3600, 10800)
    assert len(gap) == 2000
    assert abs(gap[0] - 3601.8) < 1e-9 and abs(gap[-1] - 10798.2) < 1e-9
    a, b = times(U, 7, 0, -1, 0, 450), times(U, 7, 0, -1, 450, 3600)
    assert len(a) + len(b) == 7
    assert list(np.concatenate([a, b])) == list(times(U, 7, 0, -1, 0, 3600))
    bounded = times(U, 10, 900, 2700, 0, 3600)
    assert len(bounded) == 5 and all(900 <= t < 2700 for t in bounded)
    legacy = times(B, 1000, 0, -1, 0, 7200)
    assert len(legacy) == 1000 and all(t == 0 for t in legacy)
    instant = times(B, 4, 3600, 3600, 3600, 7200)
    assert len(instant) == 4 and all(t == 3600 for t in instant)
    assert len(times(B, 4, 3600, 3600, 7200, 10800)) == 0
    assert len(times(B, 4, 3600, 3600, 0, 3600)) == 0
    assert len(times(B, 4, 0, 7200, 7200, 10800)) == 4
    assert len(times(B, 4, 0, 1800, 3600, 7200)) == 0
    assert len(times(B, 4, 3600.00001, 3600.00001, 3600, 7200)) == 4
    assert len(times(B, 4, 3599.99999, 3599.99999, 3600, 7200)) == 4
    pulse = times(P, 25, 1800, -1, 0, 3600)
    assert len(pulse) == 25 and all(t == 1800 for t in pulse)
    assert len(times(P, 25, 1800, -1, 1800, 3600)) == 25
    assert len(times(P, 25, 1800, -1, 0, 1800)) == 0
    assert times(B, 1.5, 0, -1, 0, 3600) is None
    lib = ob.oracle_lib()
    off = lib.wo_source_position_offset(5489, 42, 0)
    assert off == lib.wo_source_position_offset(5489, 42, 0)
    assert off != lib.wo_source_position_offset(5489, 43, 0)
    assert off != lib.wo_source_position_offset(5489, 42, 1)
    assert off != lib.wo_source_position_offset(5490, 42, 0)


def mixed_sources():
    """Sources whose releases interleave and tie: batch and pulse releases at the interval start,
    equal uniform rates with equal starts, a bounded window, an inactive source (mode 0) and a
    source that starts at the run start (start < 0)."""
    day = 86400.0
    return make_sources([
        (-0.2, 10.5, 11.5, 0.0, -1, 40, "uniform_rate"),
        (-0.1, 20.5, 21.5, 3600 / day, -1, 7, "forcing_interval_batch"),
        (-0.3, 12.5, 30.5, 3600 / day, -1, 5, "single_pulse"),
        (-0.4, 13.5, 31.5, 0.0, -1, 40, "uniform_rate"),
        (-0.5, 14.5, 32.5, 0.0, 5400 / day, 100, "uniform_rate"),
        (-0.6, 15.5, 33.5, 0.0, -1, 1000, "uniform_rate", 0),
        (-0.7, 16.5, 34.5, -1, -1, 13, "uniform_rate"),
        (-0.8, 17.5, 35.5, 3600 / day, 3600 / day, 3, "forcing_interval_batch"),
    ])


def composed_reference_emit(config, sources, julian_start, t0, t1, first_id):
    """Sources::emit composed from the reference's compiled helpers: sourceEmissionTimes per
    active source (Source.cpp:16-23), a stable sort by time (Sources.cpp:233-249), and
    Source::emit's id, offsets and side (Source.cpp:25-45)."""
    lib = ob.ref_lib()
    pairs = []
    for s, src in enumerate(sources):
        if src["mode"] != 1:
            continue
        start = julian_start * 86400.0 if src["start"] < 0 else src["start"] * 86400.0
        end = -1.0 if src["end"] < 0 else src["end"] * 86400.0
        ts = ob.emission_times("ref", int(src["emission_mode"]), float(src["emission_value"]),
                               start, end, t0, t1)
        assert ts is not None
        pairs += [(t, s) for t in ts]
    pairs.sort(key=lambda p: p[0])  # list.sort is stable
    out = np.zeros(len(pairs), dtype=ob.PARTICLE_DTYPE)
    for r, (t, s) in enumerate(pairs):
        src = sources[s]
        pid = first_id + r
        k, j, i = src["k"], src["j"], src["i"]
        if config.randomSources:
            k = k + lib.ref_source_position_offset(config.randomSeed, pid, 0)
            j = j + lib.ref_source_position_offset(config.randomSeed, pid, 1)
            i = i + lib.ref_source_position_offset(config.randomSeed, pid, 2)
        side = config.driftSide
        if config.leewayRandomSide:
            side = lib.ref_sample_drift_side(config.randomSeed, pid,
                                             config.leewayRightSideProbability)
        out[r] = (pid, k, j, i, 1.0, 0.0, t, config.driftObjectType, side)
    return out


@pytest.mark.parametrize("random_sources,random_side", [(False, False), (True, True)])
def test_sources_emit_matches_reference_helpers(random_sources, random_side):
    if not ob.ref_available():
        pytest.skip("reference library not built here")
    cfg = default_config(randomSources=random_sources, leewayRandomSide=random_side,
                         driftObjectType=3, driftSide=1, leewayRightSideProbability=0.3)
    src = mixed_sources()
    for (t0, t1), first in zip([(0.0, 3600.0), (3600.0, 7200.0), (1800.0, 5400.0)],
                               [7, 0, 123456]):
        got = ob.sources_emit(cfg, src, 0.0, t0, t1, first)
        want = composed_reference_emit(cfg, src, 0.0, t0, t1, first)
        assert len(got) == len(want) > 0
        assert all(got[f].tobytes() == want[f].tobytes() for f in got.dtype.names)


def test_sources_emit_properties():
    cfg = default_config(randomSources=False)
    src = mixed_sources()
    whole = ob.sources_emit(cfg, src, 0.0, 0.0, 7200.0, 0)
    first = ob.sources_emit(cfg, src, 0.0, 0.0, 3600.0, 0)
    second = ob.sources_emit(cfg, src, 0.0, 3600.0, 7200.0, len(first))
    assert np.all(np.diff(whole["time"]) >= 0)
    assert np.array_equal(whole["id"], np.arange(len(whole)))
    # uniform sources split across intervals release the same times; batch sources release one
    # batch per interval start, so the two halves hold one more interval start than the whole
    uni = lambda a: a[np.isin(a["k"], [-0.2, -0.4, -0.5, -0.7])]["time"]
    assert list(uni(np.concatenate([first, second]))) == list(uni(whole))
    assert not np.any(np.isclose(whole["k"], -0.6))  # mode 0 never emits
    bad = src.copy()
    bad[1]["emission_value"] = 2.5
    assert ob.sources_emit(cfg, bad, 0.0, 0.0, 3600.0, 0) is None
    assert SOURCE_DTYPE.itemsize == 56
