"""The C restatement against the reference's own Particle::move compiled from its sources
(oracle/_ref), record for record, over randomized inputs of every closure, both integrators,
diffusion and the drift model. Skipped where the reference build is absent."""
import itertools

import numpy as np
import pytest

from helpers import records_equal
from oracle import bindings as ob
from wacommplusplus_b200 import synthetic as syn
from wacommplusplus_b200.types import default_config

pytestmark = pytest.mark.skipif(not ob.ref_available(), reason="oracle/_ref not built")


@pytest.fixture(scope="module")
def scene():
    rf = syn.RealisticForcing(eta=48, xi=40, s_rho=8, n_frames=3, seed=21, water_border=4,
                              dlon=0.002, dlat=0.002)
    win = rf.window()
    rng = np.random.default_rng(22)
    T = win.T
    win.windU10 = (8 + 2 * rng.standard_normal((T, win.eta, win.xi))).astype(np.float32)
    win.windV10 = (1 + 2 * rng.standard_normal((T, win.eta, win.xi))).astype(np.float32)
    win.stokesU = (0.1 * rng.standard_normal((T, win.eta, win.xi))).astype(np.float32)
    win.stokesV = (0.1 * rng.standard_normal((T, win.eta, win.xi))).astype(np.float32)
    p = rf.release(1024, n_sources=16, seed=23)
    p["time"] = win.times[0] + rng.uniform(0, 3600, len(p))
    return win, p, rng


@pytest.mark.parametrize("integrator,random,drift",
                         list(itertools.product((1, 2), (False, True), (0, 1))))
def test_restatement_is_bit_exact(scene, integrator, random, drift):
    win, p0, rng = scene
    for up, lo, hor in itertools.product((1, 2, 3), (1, 2, 3), (1, 2, 3)):
        cfg = default_config(random=random, integrator=integrator, upperClosure=up,
                             lowerClosure=lo, horizontalClosure=hor, dti=15.0)
        p = p0.copy()
        if drift:
            cfg.driftModel = 1
            cfg.windErrorStdDev = 1.0
            cfg.leewayCoefficientEnsemble = True
            cfg.leewayResidualCorrelation = -0.3
            cfg.leewayJibeProbabilityHourly = 0.3
            p["driftObjectType"] = np.random.default_rng(up * 9 + lo * 3 + hor).integers(1, 23, len(p))
            p["driftSide"] = 1 - 2 * (np.arange(len(p)) % 2)
        # The reference reads out of bounds once a particle reaches a zero cell height (0/0 in its
        # vertical index, Particle.cpp:579,657,231): run it only on trajectories the oracle finds
        # finite.
        probe = p.copy()
        keep = np.ones(len(p), dtype=bool)
        for t in (0, 1):
            ob.oracle_move(cfg, probe, win, t, threads=4)
            keep &= np.isfinite(probe["k"]) & np.isfinite(probe["j"]) & np.isfinite(probe["i"])
        p = p[keep].copy()
        assert keep.mean() > 0.9
        a, b = p.copy(), p.copy()
        for t in (0, 1):
            ob.oracle_move(cfg, a, win, t, threads=4)
            ob.ref_move(cfg, b, win, t, threads=4)
        assert records_equal(a, b), (up, lo, hor)
