"""The oracle (our C restatement) pinned against the reference's own known answers:
pinned random-key values, helper identities, drift-model algebra, the particle-step and
concentration known-answer tests, and record-for-record fixtures produced by the reference's
Particle::move (tests/golden/)."""
import json
import math
import os
from types import SimpleNamespace

import numpy as np
import pytest

from helpers import GOLDEN, load_move_cases, records_equal
from kats import concentration_kat, particle_move_kats
from oracle import bindings as ob
from wacommplusplus_b200.types import default_config


@pytest.fixture(scope="module")
def lib():
    return ob.oracle_lib()


def test_pinned_random_keys(lib):
    # NumericalHelpersTest.cpp:86-89 (scheme ordered-splitmix64-v2)
    assert lib.wo_uniform(5489, 7, 3600, 2, 0) == float.fromhex("0x1.bd90c6590112ep-1")
    assert lib.wo_uniform(0, 0, 0, 0, 0) == float.fromhex("0x1.e2b96a69ad7f4p-2")


def test_random_key_properties(lib):
    # NumericalHelpersTest.cpp:63-83
    r0 = lib.wo_normal(5489, 7, 3600, 2, 0)
    assert r0 == lib.wo_normal(5489, 7, 3600, 2, 0)
    assert r0 != lib.wo_normal(5490, 7, 3600, 2, 0)
    assert r0 != lib.wo_normal(5489, 7, 3600, 3, 0)
    assert r0 != lib.wo_normal(5489, 7, 3600, 2, 1)
    u = lib.wo_uniform
    assert u(5489, 3, 3600, 7, 0) != u(5489, 7, 3600, 3, 0)
    assert u(5489, 5, 3600, 5, 0) != u(5489, 9, 3600, 9, 0)
    assert u(5489, 42, 3600, 2, 0) != u(42, 5489, 3600, 2, 0)
    assert u(5489, 42, 3600, 2, 0) != u(5489, 42, 3600, 0, 2)
    assert u(5489, 42, 3600, 5489, 0) != u(5489, 43, 3600, 5489, 0)
    draws = set()
    for particle in range(1000):
        for substep in range(120):
            for component in range(6):
                draws.add(u(5489, particle, 1675900800, substep, component))
    assert len(draws) == 1000 * 120 * 6


def test_random_fixture(lib):
    with open(os.path.join(GOLDEN, "rng.json")) as fh:
        data = json.load(fh)
    for row in data["uniform"]:
        key = [int(x) for x in row[:5]]
        assert lib.wo_uniform(*key) == float.fromhex(row[5]), row
    for row in data["normal"]:
        key = [int(x) for x in row[:5]]
        assert lib.wo_normal(*key) == float.fromhex(row[5]), row
    for row in data["forcing_error"]:
        args = [int(row[0]), int(row[1]), int(row[2]), int(row[3]), int(row[4])] + \
               [float(x) for x in row[5:10]]
        assert lib.wo_forcing_error_normal(*args) == float.fromhex(row[10]), row


def test_numerical_helpers(lib):
    # NumericalHelpersTest.cpp:25-55
    assert math.isnan(lib.wo_restart_elapsed(0, 900, 900))
    assert lib.wo_restart_elapsed(0, 900, 450) == 450
    assert math.isnan(lib.wo_restart_elapsed(900, 0, 0))
    assert lib.wo_restart_elapsed(900, 0, 450) == 450
    assert lib.wo_restart_elapsed(2700, 5400, 2700) == 0
    assert math.isnan(lib.wo_restart_elapsed(5400, 2700, 2700))
    assert abs(lib.wo_reflect_cell(1.2, 1, .7, 0) - 1.5) < 1e-12
    assert abs(lib.wo_reflect_cell(1.8, 1, 2.3, 2) - 1.7) < 1e-12
    assert lib.wo_reflect_cell(1.2, 1, 1.4, 1) == 1.4
    assert abs(lib.wo_reflect_domain(-.2, 2) - .2) < 1e-12
    assert abs(lib.wo_reflect_domain(2.3, 2) - 1.7) < 1e-12
    assert abs(lib.wo_reflect_domain(6.3, 2) - 1.7) < 1e-12
    assert lib.wo_reflect_domain(2, 2) < 2


def _leeway(lib, coeff, wu, wv, side, dn=0.0, cn=0.0):
    import ctypes
    c = (ctypes.c_double * 9)(*coeff)
    out = (ctypes.c_double * 2)()
    lib.wo_compute_leeway(c, wu, wv, side, dn, cn, out)
    return out[0], out[1]


def _catalogue(lib, t):
    import ctypes
    out = (ctypes.c_double * 9)()
    assert lib.wo_drift_coefficients(t, out) == 0
    return list(out)


def test_drift_model(lib):
    # DriftModelTest.cpp:11-81
    down = [.01, 0, 0, 0, 0, 0, 0, 0, 0]
    assert _leeway(lib, down, 0, 0, 1) == (0, 0)
    east = _leeway(lib, down, 10, 0, 1)
    assert abs(east[0] - .1) < 1e-12 and east[1] == 0
    cross = [0, 0, 0, .01, 0, 0, -.01, 0, 0]
    left, right = _leeway(lib, cross, 10, 0, -1), _leeway(lib, cross, 10, 0, 1)
    assert left[0] == 0 and right[0] == 0
    assert abs(left[1] + right[1]) < 1e-12 and abs(left[1]) == abs(right[1])
    unc = [.01, .02, .03, .04, .05, .06, -.04, -.05, .06]
    m = _leeway(lib, unc, 10, 0, 1, 2, -1)
    assert abs(m[0] - (.1 + .02 + 2 * .03)) < 1e-12 and abs(m[1] - (.4 + .05 - .06)) < 1e-12
    assert lib.wo_correlated_normal(2, -1, 0) == -1
    assert lib.wo_correlated_normal(2, -1, 1) == 2
    assert lib.wo_correlated_normal(2, -1, -1) == -2
    assert lib.wo_sample_drift_side(5489, 42, .5) == lib.wo_sample_drift_side(5489, 42, .5)
    assert lib.wo_sample_drift_side(5489, 42, 0) == -1
    assert lib.wo_sample_drift_side(5489, 42, 1) == 1
    e = lib.wo_forcing_error_normal
    s0 = e(5489, 42, 0, 0, 0x57494e4455, .1, .5, 1200, 10000, 3600)
    s1 = e(5489, 99, 9, 7, 0x57494e4455, .100001, .500001, 1250, 10000, 3600)
    assert s0 == s1
    assert s0 != e(5489, 99, 9, 7, 0x57494e4455, .100001, .500001, 4800, 10000, 3600)
    cell = lambda lo, la: e(5489, 0, 0, 0, 0x57494e4455, lo, la, 1200, 10000, 3600)
    assert cell(.0008, .0008) != cell(.0024, .0024)
    assert cell(.0024, .0035) != cell(.0035, .0024)
    assert lib.wo_jibe_step_probability(0, 3600) == 0
    assert lib.wo_jibe_step_probability(1, 1) == 1
    assert abs(lib.wo_jibe_step_probability(.04, 3600) - .04) < 1e-12
    half = lib.wo_jibe_step_probability(.04, 1800)
    assert abs((1 - half) * (1 - half) - .96) < 1e-12
    person = _catalogue(lib, 1)
    assert person[0] == .0096
    suit = _catalogue(lib, 7)
    sr, sl = _leeway(lib, suit, 10, 0, 1), _leeway(lib, suit, 10, 0, -1)
    assert abs(sr[1] - (.0136 * 10 - .033)) < 1e-12
    assert abs(sl[1] - (-.0013 * 10 - .0265)) < 1e-12
    assert abs(_leeway(lib, person, 10, 0, -1, 0, 1)[1] - (-.0054 * 10 - .094)) < 1e-12
    assert _catalogue(lib, 19)[1] == .0266


def oracle_mover(cfg, records, window, time_index):
    return ob.oracle_move(cfg, records, window, time_index, ob.SEMANTICS_HOST, threads=1)


def test_particle_move_known_answers():
    assert particle_move_kats(oracle_mover) > 40


def test_particle_move_known_answers_device_rules():
    mover = lambda cfg, rec, win, t: ob.oracle_move(cfg, rec, win, t, ob.SEMANTICS_DEVICE, 1)
    assert particle_move_kats(mover) > 40


def test_concentration_known_answer():
    def count(records, t, n_times, s_rho, eta, xi):
        return ob.oracle_concentration(records, t, n_times,
                                       SimpleNamespace(sRho=s_rho, eta=eta, xi=xi))
    assert concentration_kat(count) == 2


@pytest.mark.parametrize("case", load_move_cases(), ids=lambda c: c["name"])
def test_reference_fixtures(case):
    """Bit-exact against the reference Particle::move over two forward intervals and one
    backward interval (tests/golden/move_cases.npz)."""
    cfg = default_config(**case["overrides"])
    win = case["window"]
    a = case["start"].copy()
    ob.oracle_move(cfg, a, win, 0, threads=1)
    assert records_equal(a, case["after1"])
    ob.oracle_move(cfg, a, win, 1, threads=1)
    assert records_equal(a, case["after2"])
    cfg.trackingDirection = -1
    b = case["after2"].copy()
    ob.oracle_move(cfg, b, win, win.T - 1, threads=1)
    assert records_equal(b, case["back"])


def test_concentration_fixture():
    data = np.load(os.path.join(GOLDEN, "concentration.npz"))
    case = [c for c in load_move_cases() if c["name"] == str(data["case"])][0]
    grid = ob.oracle_concentration(case["after2"], 2, 3, case["window"])
    assert np.array_equal(grid.astype(np.float32), data["conc"])


def test_emission_fixture():
    with open(os.path.join(GOLDEN, "emission.json")) as fh:
        cases = json.load(fh)
    for c in cases:
        got = ob.emission_times("oracle", c["mode"], c["value"], c["source"][0], c["source"][1],
                                c["interval"][0], c["interval"][1])
        if c["times"] is None:
            assert got is None, c
        else:
            assert [t.hex() for t in got] == c["times"], c
