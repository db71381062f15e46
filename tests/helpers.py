"""Shared builders for the tests: the reference's 2x2 test grid, fixture loading, comparisons."""
import json
import math
import os

import numpy as np

from wacommplusplus_b200 import synthetic as syn
from wacommplusplus_b200.types import PARTICLE_DTYPE, default_config, make_particles

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DEG = 0.017453292519943295


def tiny_window(times=(0.0, 65.0), u_fn=None, w_fn=None, akt=0.0, wind=None, stokes=None):
    """The 2x2x{2,3} grid of the reference's particle and parity tests
    (tests/ParticleMoveTest.cpp:10-23, tests/CudaParticleParityTest.cu:35-70): lon/lat nodes one
    degree apart at the equator, h=100 m, sW={-1,-.5,0}, depthIntervals=.5, zeta=0."""
    T = len(times)
    lon = np.array([[0.0, 1.0], [0.0, 1.0]])
    lat = np.array([[0.0, 0.0], [1.0, 1.0]])
    u = np.zeros((T, 2, 2, 2), np.float32)
    w = np.zeros((T, 3, 2, 2), np.float32)
    if u_fn is not None:
        u_fn(u)
    if w_fn is not None:
        w_fn(w)
    win = syn.Window(times=np.array(times, dtype=np.float64), mask=np.ones((2, 2)), lon=lon, lat=lat,
                     lonRad=lon * DEG, latRad=lat * DEG, h=np.full((2, 2), 100.0),
                     sWValues=np.array([-1.0, -0.5, 0.0]), depthIntervals=np.array([0.5, 0.5]),
                     zeta=np.zeros((T, 2, 2), np.float32), u=u, v=np.zeros((T, 2, 2, 2), np.float32),
                     w=w, akt=np.full((T, 3, 2, 2), akt, np.float32))
    if wind is not None:
        win.windU10, win.windV10 = wind
    if stokes is not None:
        win.stokesU, win.stokesV = stokes
    return win


def kat_config(**kw):
    """config of ParticleMoveTest.cpp:24-31 (a value-initialised config_data, so integrator 0:
    neither midpoint nor Euler by name, which selects the legacy Euler step)."""
    base = dict(random=False, deltat=3600.0, dti=30.0, survprob=0.0, tau0=86400.0, crid=1.0,
                sigma=3.46, shoreLimit=0.25, upperClosure=1, lowerClosure=1, horizontalClosure=1,
                trackingDirection=1, restartCheckpoint=float("nan"), integrator=0,
                randomSeed=0, leewayRightSideProbability=0.0)
    base.update(kw)
    return default_config(**base)


def one(id_, k, j, i, time, drift_type=0, side=0, health=1.0, age=0.0):
    return make_particles(1, ids=np.array([id_], np.uint64), k=k, j=j, i=i, time=time,
                          health=health, age=age, drift_type=drift_type, drift_side=side)


def load_move_cases():
    data = np.load(os.path.join(GOLDEN, "move_cases.npz"))
    cases = []
    windows = {}
    for name in data["names"]:
        name = str(name)
        wid = str(data[f"{name}_window"])
        if wid not in windows:
            fields = {}
            for key in data.files:
                if key.startswith(wid + "_win_"):
                    fields[key[len(wid) + 5:]] = data[key]
            windows[wid] = syn.Window(**fields)
        overrides = json.loads(str(data[f"{name}_config"]))
        cases.append(dict(name=name, window=windows[wid], overrides=overrides,
                          start=data[f"{name}_start"], after1=data[f"{name}_after1"],
                          after2=data[f"{name}_after2"], back=data[f"{name}_back"]))
    return cases


def records_equal(a, b):
    """Field-by-field bit equality of two record arrays (NaN equal to NaN)."""
    return all(np.array_equal(a[f], b[f], equal_nan=True) for f in PARTICLE_DTYPE.names)


def max_abs_diff(a, b, fields=("k", "j", "i", "health", "age")):
    out = {}
    for f in fields:
        x, y = a[f].astype(np.float64), b[f].astype(np.float64)
        both_nan = np.isnan(x) & np.isnan(y)
        d = np.abs(x - y)
        d[both_nan] = 0.0
        out[f] = float(np.nanmax(d)) if len(d) else 0.0
    return out


def great_circle_m(win_lon_deg, win_lat_deg, a, b):
    """Great-circle distance in metres between the positions of two record arrays on a
    rectilinear grid given by node longitudes/latitudes (degrees)."""
    def to_geo(rec):
        xi = win_lon_deg.shape[1]
        eta = win_lat_deg.shape[0]
        lon = np.interp(rec["i"], np.arange(xi), win_lon_deg[0])
        lat = np.interp(rec["j"], np.arange(eta), win_lat_deg[:, 0])
        return np.radians(lon), np.radians(lat)
    lon1, lat1 = to_geo(a)
    lon2, lat2 = to_geo(b)
    d = np.sin(0.5 * (lat2 - lat1)) ** 2 + np.cos(lat1) * np.cos(lat2) * np.sin(0.5 * (lon2 - lon1)) ** 2
    return 2 * 6371000.0 * np.arcsin(np.sqrt(np.clip(d, 0, 1)))
