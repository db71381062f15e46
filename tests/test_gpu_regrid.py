"""Device regridding of wind and Stokes fields (wacomm_b200_regrid_environment) against the oracle.

The oracle's restatement of EnvironmentalRegridder.cpp is pinned bit for bit against the
reference's own build (tests/test_oracle_regrid.py); here the device plan-and-apply path must give
the same float32 values bit for bit, for the curvilinear 3 km wind grid and the rectilinear
0.05-degree Stokes grid of the batched workload, at coinciding and at blended forcing times. A
rejected input leaves the field unset. A run fed by the regridded fields equals, record for record,
a run whose frames carry the same fields uploaded from the host.
"""
import numpy as np
import pytest

from oracle import bindings as ob
from wacommplusplus_b200 import synthetic as syn
from wacommplusplus_b200._native import WacommError
from wacommplusplus_b200.engine import Engine
from wacommplusplus_b200.types import default_config

pytestmark = pytest.mark.gpu


def oracle_env(method, lon, lat, times, u, v, win):
    """Oracle: regrid every source record to the rho nodes, then align to the forcing times."""
    out = []
    for comp in (u, v):
        rc, spatial = ob.regrid("oracle", method, lon, lat, comp, win.lon, win.lat)
        assert rc == 0
        rc, aligned = ob.align_times(times, spatial, win.times)
        assert rc == 0
        out.append(aligned)
    return out


def engine_on(win):
    e = Engine(0, arithmetic="fp32", storage="fp32")
    e.load_window(win)
    e.set_geo_grid(win.lon, win.lat, win.sWValues)
    return e


@pytest.fixture(scope="module")
def setting():
    win = syn.config1_window(n_frames=7)
    env = syn.environment(win.times[0], 6, wind_n=120)
    return win, env


@pytest.mark.parametrize("field,method", [("wind", "curvilinear"), ("stokes", "geographic"),
                                          ("stokes", "curvilinear")])
def test_device_regrid_matches_oracle(cuda_device, setting, field, method):
    win, env = setting
    lon, lat, times, u, v = env[field]
    e = engine_on(win)
    e.regrid_environment(field, method, lon, lat, times, u, v)
    want_u, want_v = oracle_env(method, lon, lat, times, u, v, win)
    for t in range(win.T):
        got_u, got_v = e.environment(field, t)
        assert got_u.tobytes() == want_u[t].tobytes(), (field, method, t)
        assert got_v.tobytes() == want_v[t].tobytes(), (field, method, t)
    e.close()


def test_rejections_leave_the_field_unset(cuda_device, setting):
    win, env = setting
    lon, lat, times, u, v = env["stokes"]
    e = engine_on(win)
    cases = [
        # a source grid west of the ocean grid (lon 13.50-13.95)
        ("geographic", lon[:, :10], lat[:, :10], times, u[:, :, :10], v[:, :, :10]),
        # a non-rectilinear source for the rectilinear method
        ("geographic", lon + 1e-3 * lat, lat, times, u, v),
        # forcing times after the last source time
        ("geographic", lon, lat, times[:2], u[:2], v[:2]),
        # a non-finite source value
        ("curvilinear", lon, lat, times, np.where(np.arange(u.size).reshape(u.shape) == 7,
                                                   np.float32(np.nan), u), v),
    ]
    for method, a, b, t, fu, fv in cases:
        with pytest.raises(WacommError):
            e.regrid_environment("stokes", method, a, b, t, fu, fv)
        with pytest.raises(WacommError):
            e.environment("stokes", 0)
    e.close()


def test_regridded_fields_feed_the_step(cuda_device, setting):
    """Leeway objects of the catalogue and Stokes drift: the run fed by the regridded fields
    equals the run whose records carry the same fields from the host."""
    win, env = setting
    cfg = default_config(random=False, driftModel=1)
    parts = syn.uniform_particles(20000, win.eta, win.xi, seed=4)
    parts["driftObjectType"] = 1 + np.arange(len(parts)) % 22
    parts["driftSide"] = np.where(np.arange(len(parts)) % 2, 1, -1)
    a = engine_on(win)
    a.set_config(cfg)
    for field, method in (("wind", "curvilinear"), ("stokes", "geographic")):
        a.regrid_environment(field, method, *env[field])
    wind = [a.environment("wind", t) for t in range(win.T)]
    stokes = [a.environment("stokes", t) for t in range(win.T)]
    b = Engine(0, arithmetic="fp32", storage="fp32")
    b.set_config(cfg)
    b.set_grid(win.eta, win.xi, win.sRho, win.sW, win.lonRad, win.latRad, win.h,
               win.depthIntervals, win.mask)
    b.set_times(win.times)
    for t in range(win.T):
        f = win.frame(t)
        b.upload_frame(t, f["zeta"], f["u"], f["v"], f["w"], f["akt"], wind[t][0], wind[t][1],
                       stokes[t][0], stokes[t][1])
    for e in (a, b):
        e.set_particles(parts)
        for t in range(win.T - 1):
            e.move_interval(t)
    pa, pb = a.get_particles(), b.get_particles()
    for f in pa.dtype.names:
        assert pa[f].tobytes() == pb[f].tobytes(), f
    moved = np.hypot(pa["i"] - parts["i"], pa["j"] - parts["j"])
    assert moved.max() > 0
    a.close()
    b.close()
