"""The reference's own known-answer tests of the particle step and the concentration grid,
restated against an abstract mover so that the same assertions pin the oracle (CPU) and the B200
kernels (GPU).

`move(cfg, records, window, time_index)` must move the record array in place over one interval.
Each block cites the reference assertion it restates (tests/ParticleMoveTest.cpp,
tests/ConcentrationTest.cpp).
"""
import math

import numpy as np

from helpers import DEG, kat_config, one, tiny_window
from wacommplusplus_b200.types import make_particles

PIW, RIGHT, LEFT = 1, 1, -1


def _xdist():
    d = math.sin(0.5 * DEG) ** 2
    return 2.0 * math.atan2(math.sqrt(d), math.sqrt(1.0 - d)) * 6371000.0


def _u_frame1(value):
    def fill(u):
        u[1, :, :, :] = value
    return fill


def particle_move_kats(move):
    """ParticleMoveTest.cpp:9-299. Returns the number of assertions checked."""
    checks = 0
    xdist = _xdist()
    win = tiny_window((0.0, 65.0), u_fn=_u_frame1(2.0))
    zero = tiny_window((0.0, 65.0))
    cfg = kat_config()

    # exact time-linear integration (:33-38)
    full = move(cfg, one(1, -.5, .25, .25, 0), win, 0)
    assert abs(full["age"][0] - 65) < 1e-12
    assert abs(full["i"][0] - (.25 + 65.0 / xdist)) < 1e-10
    # particle emitted part-way through the interval (:40-44)
    emitted = move(cfg, one(2, -.5, .25, .25, 40), win, 0)
    assert abs(emitted["age"][0] - 25) < 1e-12
    assert abs(emitted["i"][0] - (.25 + (65.0 * 65.0 - 40.0 * 40.0) / 65.0 / xdist)) < 1e-10
    # deterministic backward return (:46-50)
    cfg.trackingDirection = -1
    back = move(cfg, one(3, -.5, full["j"][0], full["i"][0], 65), win, 1)
    assert abs(back["age"][0] - 65) < 1e-12 and abs(back["i"][0] - .25) < 1e-10
    checks += 6

    # seeded repeatability and seed sensitivity (:52-64)
    cfg.trackingDirection = 1
    cfg.random = True
    cfg.randomSeed = 5489
    s0 = move(cfg, one(4, -.5, .25, .25, 0), win, 0)
    s1 = move(cfg, one(4, -.5, .25, .25, 0), win, 0)
    assert s0["i"][0] == s1["i"][0] and s0["j"][0] == s1["j"][0] and s0["k"][0] == s1["k"][0]
    cfg.randomSeed = 5490
    s2 = move(cfg, one(4, -.5, .25, .25, 0), win, 0)
    assert s0["i"][0] != s2["i"][0] or s0["j"][0] != s2["j"][0] or s0["k"][0] != s2["k"][0]
    checks += 2

    # stochastic restart equality (:66-81)
    cfg.randomSeed = 5489
    early30 = tiny_window((0.0, 30.0))
    sfull = move(cfg, one(8, -.5, .25, .25, 0), zero, 0)
    srest = move(cfg, one(8, -.5, .25, .25, 0), early30, 0)
    cfg.restartCheckpoint = 30
    srest = move(cfg, srest, zero, 0)
    for f in ("i", "j", "k", "age"):
        assert srest[f][0] == sfull[f][0], f
    checks += 4

    # schedule independence: many particles at once equal one at a time (:84-100)
    cfg.restartCheckpoint = float("nan")
    batch = make_particles(64, ids=np.arange(100, 164, dtype=np.uint64), k=-.5, j=.25, i=.25)
    together = move(cfg, batch.copy(), zero, 0)
    for idx in (0, 17, 63):
        alone = move(cfg, batch[idx:idx + 1].copy(), zero, 0)
        for f in ("i", "j", "k"):
            assert together[f][idx] == alone[f][0]
    checks += 9

    # restarted forward (:102-114)
    cfg.random = False
    early40 = tiny_window((0.0, 40.0), u_fn=_u_frame1(80.0 / 65.0))
    rf = move(cfg, one(5, -.5, .25, .25, 0), early40, 0)
    cfg.restartCheckpoint = 40
    rf = move(cfg, rf, win, 0)
    assert abs(rf["i"][0] - full["i"][0]) < 1e-8 and abs(rf["age"][0] - full["age"][0]) < 1e-12
    # restarted backward (:116-129)
    cfg.trackingDirection = -1
    cfg.restartCheckpoint = float("nan")

    def late_u(u):
        u[0] = 80.0 / 65.0
        u[1] = 2.0
    late = tiny_window((40.0, 65.0), u_fn=late_u)
    rb = move(cfg, one(6, -.5, full["j"][0], full["i"][0], 65), late, 1)
    cfg.restartCheckpoint = 40
    rb = move(cfg, rb, win, 1)
    assert abs(rb["i"][0] - .25) < 1e-8 and abs(rb["age"][0] - 65) < 1e-12
    checks += 4

    # vertical velocity at k=-0.5 over one second (:131-139)
    cfg.trackingDirection = 1
    cfg.restartCheckpoint = float("nan")

    def w_top(w):
        w[:, 2, :, :] = 2.0
    vert = tiny_window((0.0, 1.0), w_fn=w_top)
    v = move(cfg, one(7, -.5, .25, .25, 0), vert, 0)
    assert abs(v["k"][0] + .48) < 1e-12
    checks += 1

    # leeway forward/backward reversal (:141-155)
    cfg.sv = 0
    cfg.driftModel = 1
    cfg.driftObjectType = PIW
    cfg.driftSide = RIGHT
    cfg.hasWind = True
    cfg.windU10 = 10
    cfg.windV10 = 0
    lf = move(cfg, one(9, -.5, .25, .25, 0, PIW, RIGHT), zero, 0)
    assert lf["i"][0] > .25 and lf["j"][0] > .25
    cfg.trackingDirection = -1
    lb = move(cfg, one(10, -.5, lf["j"][0], lf["i"][0], 65, PIW, RIGHT), zero, 1)
    assert abs(lb["i"][0] - .25) < 1e-8 and abs(lb["j"][0] - .25) < 1e-8
    checks += 2

    # coefficient ensembles (:157-175)
    cfg.leewayCoefficientEnsemble = True
    cfg.trackingDirection = 1
    e0 = move(cfg, one(20, -.5, .25, .25, 0, PIW, RIGHT), zero, 0)
    e0r = move(cfg, one(20, -.5, .25, .25, 0, PIW, RIGHT), zero, 0)
    e1 = move(cfg, one(21, -.5, .25, .25, 0, PIW, RIGHT), zero, 0)
    assert e0["i"][0] == e0r["i"][0] and e0["j"][0] == e0r["j"][0]
    assert e0["i"][0] != e1["i"][0] or e0["j"][0] != e1["j"][0]
    cfg.trackingDirection = -1
    eb = move(cfg, one(20, -.5, e0["j"][0], e0["i"][0], 65, PIW, RIGHT), zero, 1)
    assert abs(eb["i"][0] - .25) < 1e-8 and abs(eb["j"][0] - .25) < 1e-8
    cfg.leewayCoefficientEnsemble = False
    checks += 3

    # wind error: restart equality and identity sensitivity (:177-191)
    cfg.windErrorStdDev = 1.5
    cfg.trackingDirection = 1
    ff = move(cfg, one(22, -.5, .25, .25, 0, PIW, RIGHT), zero, 0)
    fr = move(cfg, one(22, -.5, .25, .25, 0, PIW, RIGHT), early30, 0)
    cfg.restartCheckpoint = 30
    fr = move(cfg, fr, zero, 0)
    cfg.restartCheckpoint = float("nan")
    fo = move(cfg, one(23, -.5, .25, .25, 0, PIW, RIGHT), zero, 0)
    assert ff["i"][0] == fr["i"][0] and ff["j"][0] == fr["j"][0]
    assert ff["i"][0] != fo["i"][0] or ff["j"][0] != fo["j"][0]
    cfg.windErrorStdDev = 0
    checks += 2

    # jibing with an hourly probability of one (:193-221)
    cfg.leewayJibeProbabilityHourly = 1
    cfg.trackingDirection = 1
    jf = move(cfg, one(30, -.5, .25, .25, 0, PIW, RIGHT), zero, 0)
    jr = move(cfg, one(30, -.5, .25, .25, 0, PIW, RIGHT), early30, 0)
    cfg.restartCheckpoint = 30
    jr = move(cfg, jr, zero, 0)
    assert jf["i"][0] == jr["i"][0] and jf["j"][0] == jr["j"][0]
    assert jf["driftSide"][0] == jr["driftSide"][0] == LEFT
    cfg.trackingDirection = -1
    cfg.restartCheckpoint = float("nan")
    jbf = move(cfg, one(31, -.5, .25, .25, 65, PIW, RIGHT), zero, 1)
    late35 = tiny_window((35.0, 65.0))
    jbr = move(cfg, one(31, -.5, .25, .25, 65, PIW, RIGHT), late35, 1)
    cfg.restartCheckpoint = 35
    jbr = move(cfg, jbr, zero, 1)
    assert jbf["i"][0] == jbr["i"][0] and jbf["j"][0] == jbr["j"][0]
    assert jbf["driftSide"][0] == jbr["driftSide"][0]
    cfg.leewayJibeProbabilityHourly = 0
    cfg.restartCheckpoint = float("nan")
    checks += 4

    # coupled wind and Stokes fields (:223-237)
    T = 2
    wind = (np.full((T, 2, 2), 10.0, np.float32), np.zeros((T, 2, 2), np.float32))
    stokes = (np.full((T, 2, 2), .2, np.float32), np.full((T, 2, 2), -.1, np.float32))
    coupled = tiny_window((0.0, 65.0), wind=wind, stokes=stokes)
    cfg.trackingDirection = 1
    cf = move(cfg, one(11, -.5, .25, .25, 0, PIW, RIGHT), coupled, 0)
    assert cf["i"][0] > lf["i"][0]
    cfg.trackingDirection = -1
    cb = move(cfg, one(12, -.5, cf["j"][0], cf["i"][0], 65, PIW, RIGHT), coupled, 1)
    assert abs(cb["i"][0] - .25) < 1e-8 and abs(cb["j"][0] - .25) < 1e-8
    checks += 2

    # explicit midpoint: order of accuracy on u = b*i (:239-266)
    mc = kat_config()

    def shear(u):
        u[:, :, :, 1] = 10.0
    hour = tiny_window((0.0, 3600.0), u_fn=shear)
    exact = .25 * math.exp(10.0 * 3600.0 / xdist)

    def shear_error(integrator, dti):
        mc.integrator = integrator
        mc.dti = dti
        p = move(mc, one(40, -.5, .25, .25, 0), hour, 0)
        assert p["health"][0] > 0
        return abs(p["i"][0] - exact)
    e600, e300 = shear_error(1, 600), shear_error(1, 300)
    m600, m300 = shear_error(2, 600), shear_error(2, 300)
    assert 1.8 < e600 / e300 < 2.2
    assert 3.6 < m600 / m300 < 4.4
    assert m600 < e600 / 20
    checks += 3

    # midpoint backward return (:268-276)
    mc.integrator = 2
    mc.dti = 300
    sf = move(mc, one(41, -.5, .25, .25, 0), hour, 0)
    mc.trackingDirection = -1
    sb = move(mc, one(42, -.5, sf["j"][0], sf["i"][0], 3600), hour, 1)
    assert abs(sb["i"][0] - .25) < 2 * m300 and abs(sb["age"][0] - 3600) < 1e-12
    checks += 1

    # continuous and restarted midpoint take the same substeps (:278-287)
    mc.trackingDirection = 1
    half = tiny_window((0.0, 1800.0), u_fn=shear)
    sr = move(mc, one(41, -.5, .25, .25, 0), half, 0)
    mc.restartCheckpoint = 1800
    sr = move(mc, sr, hour, 0)
    assert abs(sr["i"][0] - sf["i"][0]) < 1e-12 and abs(sr["age"][0] - sf["age"][0]) < 1e-12
    mc.restartCheckpoint = float("nan")
    checks += 1

    # a midpoint outside the domain falls back to the Euler step (:289-299)
    step = tiny_window((0.0, 600.0), u_fn=shear)
    mc.dti = 600
    mc.integrator = 1
    ee = move(mc, one(43, -.5, .25, .99, 0), step, 0)
    mc.integrator = 2
    em = move(mc, one(43, -.5, .25, .99, 0), step, 0)
    for f in ("i", "j", "k", "health"):
        assert em[f][0] == ee[f][0]
    checks += 4
    return checks


def concentration_kat(count):
    """ConcentrationTest.cpp:5-28: 100,000 particles in one cell keep their count; a particle
    outside the grid and a dead one are not counted. `count(records, t, n_times, s_rho, eta, xi)`
    returns the [n_times][s_rho][eta][xi] grid."""
    n = 100000
    p = make_particles(n + 2, k=-1, j=1, i=1)
    p["j"][n] = 4
    p["health"][n + 1] = 0
    grid = count(p, 0, 1, 3, 3, 3)
    assert grid[0, 1, 1, 1] == n  # logical k=-1 is storage level 1 of 3
    assert grid.sum() == n
    return 2
