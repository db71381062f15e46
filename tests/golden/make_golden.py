"""Generates the golden fixtures of tests/golden/ by running the reference's own code.

Run from the repository root after ``make -C oracle`` has built oracle/_ref (which needs the
reference tree):

    python tests/golden/make_golden.py

It writes
  * rng.json         - uniform/normal/forcing-error draws of NumericalHelpers.hpp:104-120 and
                       DriftModel.hpp:118-140 for a lattice of keys;
  * emission.json    - sourceEmissionTimes (SourceEmission.hpp:38-79) for a set of schedules;
  * move_cases.npz   - inputs and reference Particle::move outputs (two intervals forward, one
                       backward) for small synthetic windows covering every closure, both
                       integrators, diffusion, leeway, wind error, jibing and Stokes drift;
  * concentration.npz - Concentration::evaluate float counts for the first move case.
The fixtures travel with the repository so that the oracle is pinned where the reference is
absent.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import bindings as ob  # noqa: E402
from wacommplusplus_b200 import synthetic as syn  # noqa: E402
from wacommplusplus_b200.types import PARTICLE_DTYPE, default_config  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

WINDOW_FIELDS = ("times", "mask", "lonRad", "latRad", "h", "sWValues", "depthIntervals", "zeta",
                 "u", "v", "w", "akt", "windU10", "windV10", "stokesU", "stokesV", "lon", "lat")

CONFIG_FIELDS = ("random", "dti", "survprob", "tau0", "sv", "crid", "sigma", "shoreLimit",
                 "upperClosure", "lowerClosure", "horizontalClosure", "randomSeed",
                 "backwardDiffusion", "integrator", "driftModel", "leewayCoefficientEnsemble",
                 "leewayResidualCorrelation", "leewayJibeProbabilityHourly", "windErrorStdDev",
                 "windErrorComponentCorrelation", "windErrorSpatialScale",
                 "windErrorTemporalScale", "windU10", "windV10")


def rng_fixture(lib):
    keys = []
    for seed in (0, 1, 5489, 2 ** 63 + 5):
        for particle in (0, 7, 42, 9007199254740993):
            for interval in (0, 3600, 1675900800, -(2 ** 63)):
                for substep in (0, 2, 119):
                    for component in (0, 1, 5, 0x4a494245):
                        keys.append((seed, particle, interval, substep, component))
    out = {"uniform": [], "normal": [], "forcing_error": []}
    for k in keys:
        out["uniform"].append([*map(str, k), lib.ref_uniform(*k).hex()])
        out["normal"].append([*map(str, k), lib.ref_normal(*k).hex()])
    for lon, lat, t, spatial, temporal in ((.1, .5, 1200, 10000, 3600), (.100001, .500001, 1250, 10000, 3600),
                                           (.24, .71, 4800, 0, 3600), (.24, .71, 4800, 5000, 0),
                                           (.0024, .0035, 1200, 10000, 3600)):
        args = (5489, 99, 9, 7, 0x57494e4455, lon, lat, t, spatial, temporal)
        out["forcing_error"].append([*map(repr, args), lib.ref_forcing_error_normal(*args).hex()])
    return out


def emission_fixture():
    cases = []
    for mode in (0, 1, 2):
        for value in (0, 1, 3, 7.5, 100):
            for src in ((0.0, -1.0), (1800.0, -1.0), (0.0, 5400.0), (3600.0, 3600.0), (900.5, 2000.0)):
                for interval in ((0.0, 3600.0), (3600.0, 7200.0)):
                    times = ob.emission_times("ref", mode, value, src[0], src[1], *interval)
                    cases.append({"mode": mode, "value": value, "source": list(src),
                                  "interval": list(interval),
                                  "times": None if times is None else [t.hex() for t in times]})
    return cases


def window_arrays(win):
    out = {}
    for f in WINDOW_FIELDS:
        value = getattr(win, f, None)
        if value is not None:
            out["win_" + f] = np.asarray(value)
    return out


def move_cases():
    """(name, window, config overrides, particles) of the fixture scenarios."""
    rf = syn.RealisticForcing(eta=24, xi=20, s_rho=4, n_frames=3, seed=11, water_border=3,
                              dlon=0.004, dlat=0.004)
    win = rf.window()
    rng = np.random.default_rng(12)
    T = win.T
    win.windU10 = (6 + 2 * rng.standard_normal((T, win.eta, win.xi))).astype(np.float32)
    win.windV10 = (1 + 2 * rng.standard_normal((T, win.eta, win.xi))).astype(np.float32)
    win.stokesU = (0.1 * rng.standard_normal((T, win.eta, win.xi))).astype(np.float32)
    win.stokesV = (0.1 * rng.standard_normal((T, win.eta, win.xi))).astype(np.float32)
    p = rf.release(256, n_sources=8, seed=13, spread=0.6)
    p["time"] = win.times[0] + rng.uniform(0, 3600, len(p))
    drift = p.copy()
    drift["driftObjectType"] = rng.integers(1, 23, len(p))
    drift["driftSide"] = rng.choice([-1, 1], len(p))
    cases = []
    for integrator in (1, 2):
        for closures in ((1, 2, 3), (3, 1, 1), (2, 3, 2)):
            cases.append((f"realistic_i{integrator}_c{''.join(map(str, closures))}", win,
                          dict(random=True, integrator=integrator, upperClosure=closures[0],
                               lowerClosure=closures[1], horizontalClosure=closures[2], dti=20.0),
                          p))
        cases.append((f"drift_i{integrator}", win,
                      dict(random=True, integrator=integrator, driftModel=1, dti=20.0,
                           windErrorStdDev=1.0, windErrorComponentCorrelation=0.3,
                           leewayCoefficientEnsemble=True, leewayResidualCorrelation=-0.35,
                           leewayJibeProbabilityHourly=0.4, windU10=8.0, windV10=-2.0),
                      drift))
    c1 = syn.config1_window(n_frames=3, eta=16, xi=16, s_rho=10)
    q = syn.uniform_particles(200, c1.eta, c1.xi, seed=1)
    for integrator in (1, 2):
        cases.append((f"config1_i{integrator}", c1, dict(random=False, integrator=integrator), q))
    return cases


def main():
    if not ob.ref_available():
        raise SystemExit("oracle/_ref is not built: run make -C oracle with the reference present")
    lib = ob.ref_lib()
    with open(os.path.join(HERE, "rng.json"), "w") as fh:
        json.dump(rng_fixture(lib), fh)
    with open(os.path.join(HERE, "emission.json"), "w") as fh:
        json.dump(emission_fixture(), fh)
    arrays = {}
    names = []
    seen = {}
    for name, win, overrides, particles in move_cases():
        particles = well_defined(win, overrides, particles)
        wid = seen.setdefault(id(win), f"w{len(seen)}")
        if wid + "_win_times" not in arrays:
            for key, value in window_arrays(win).items():
                arrays[f"{wid}_{key}"] = value
        cfg = default_config(**overrides)
        start = particles.copy()
        a = start.copy()
        ob.ref_move(cfg, a, win, 0, threads=1)
        after1 = a.copy()
        ob.ref_move(cfg, a, win, 1, threads=1)
        after2 = a.copy()
        cfg.trackingDirection = -1
        b = after2.copy()
        ob.ref_move(cfg, b, win, win.T - 1, threads=1)
        arrays[f"{name}_start"] = start
        arrays[f"{name}_after1"] = after1
        arrays[f"{name}_after2"] = after2
        arrays[f"{name}_back"] = b
        arrays[f"{name}_config"] = np.array(json.dumps(overrides))
        arrays[f"{name}_window"] = np.array(wid)
        names.append(name)
    arrays["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "move_cases.npz"), **arrays)
    first = names[0]
    wid = str(arrays[f"{first}_window"])
    win = load_window(arrays, wid)
    conc = ob.ref_concentration(arrays[f"{first}_after2"], 2, 3, win)
    np.savez_compressed(os.path.join(HERE, "concentration.npz"), conc=conc, case=first)
    print("wrote", len(names), "move cases")


def well_defined(win, overrides, particles):
    """Drops particles whose trajectory reaches a state where the reference's behaviour is
    undefined: a zero cell height (h + zeta == 0, e.g. on a dry node) gives a 0/0 vertical index
    and then an out-of-bounds read (Particle.cpp:579,657,231). The oracle, which clamps those
    reads, finds them; the reference is then run only on the rest."""
    keep = np.ones(len(particles), dtype=bool)
    for direction_pass in (0, 1):
        cfg = default_config(**overrides)
        a = particles.copy()
        for t in range(win.T - 1):
            ob.oracle_move(cfg, a, win, t, threads=1)
            keep &= np.isfinite(a["k"]) & np.isfinite(a["j"]) & np.isfinite(a["i"])
        if direction_pass == 1:
            cfg.trackingDirection = -1
            ob.oracle_move(cfg, a, win, win.T - 1, threads=1)
            keep &= np.isfinite(a["k"]) & np.isfinite(a["j"]) & np.isfinite(a["i"])
    return particles[keep].copy()


def load_window(arrays, wid):
    fields = {}
    for f in WINDOW_FIELDS:
        key = f"{wid}_win_{f}"
        if key in arrays:
            fields[f] = arrays[key]
    return syn.Window(**fields)


if __name__ == "__main__":
    main()
