"""The reference's analytic end-to-end check (ApplicationEndToEndTest.cpp:252-257, 363-393)
restated on the analytic grid: in a uniform current (u, v) with w = 0 and no diffusion, a particle
follows the rhumb line dlat = v T / R, dlon = (u / v) ln(tan(pi/4 + lat1/2) / tan(pi/4 + lat0/2)).
The end position must lie within 0.1 % of the path, the age equal the elapsed time, the level stay
unchanged, and tracking back over the same intervals must return to the release point within
1 mm."""
import math

import numpy as np
import pytest

from wacommplusplus_b200 import synthetic as syn
from wacommplusplus_b200.engine import Engine
from wacommplusplus_b200.types import PARTICLE_DTYPE, default_config

pytestmark = pytest.mark.gpu

R_EARTH = 6371000.0
U, V = 0.2, 0.1
HOURS = 5


def _analytic_end(lon, lat, T):
    lat_end = lat + V * T / R_EARTH * 180.0 / math.pi
    phi0, phi1 = np.radians(lat), np.radians(lat_end)
    ratio = np.tan(math.pi / 4 + phi1 / 2) / np.tan(math.pi / 4 + phi0 / 2)
    lon_end = lon + (U / V) * np.log(ratio) * 180.0 / math.pi
    return lon_end, lat_end


@pytest.mark.parametrize("arithmetic,round_trip_m", [("reference", 1e-3), ("fp32", 1e-3)])
def test_rhumb_line_forward_and_back(cuda_device, arithmetic, round_trip_m):
    win = syn.config1_window(n_frames=HOURS + 1, u=U, v=V)
    rng = np.random.default_rng(17)
    n = 4096
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    p["id"] = np.arange(1, n + 1)
    p["i"] = rng.uniform(5, win.xi - 40, n)   # ~27 cells east in 5 h
    p["j"] = rng.uniform(5, win.eta - 25, n)  # ~14 cells north
    p["k"] = -0.5
    p["health"] = 1.0
    p["time"] = win.times[0]
    cfg = default_config(random=False)
    T = HOURS * 3600.0
    with Engine(cuda_device, arithmetic=arithmetic) as e:
        e.load_window(win)
        e.set_config(cfg)
        e.set_geo_grid(win.lon, win.lat, win.sWValues)
        e.set_particles(p)
        _, lat0, lon0 = e.geo_positions()
        for t in range(HOURS):
            e.move_interval(t)
        end = e.get_particles()
        _, lat1, lon1 = e.geo_positions()
        lon_end, lat_end = _analytic_end(lon0, lat0, T)
        dx = np.radians(lon1 - lon_end) * R_EARTH * np.cos(np.radians(lat_end))
        dy = np.radians(lat1 - lat_end) * R_EARTH
        error = np.hypot(dx, dy)
        path = math.hypot(U, V) * T
        assert np.all(end["health"] > 0)
        assert error.max() < 1e-3 * path, error.max()
        assert np.abs(end["age"] - T).max() < 1e-3
        assert np.abs(end["k"] - p["k"]).max() < 1e-12
        cfg.trackingDirection = -1
        e.set_config(cfg)
        for t in range(HOURS, 0, -1):
            e.move_interval(t)
        _, lat2, lon2 = e.geo_positions()
        back = e.get_particles()
    trip = np.hypot(np.radians(lon2 - lon0) * R_EARTH * np.cos(np.radians(lat0)),
                    np.radians(lat2 - lat0) * R_EARTH)
    print(f"\n{arithmetic}: end error vs rhumb line max {error.max():.3g} m "
          f"(0.1 % of the {path:.0f} m path: {1e-3 * path:.3g} m); round trip max {trip.max():.3g} m")
    assert np.abs(back["k"] - p["k"]).max() < 1e-12
    assert trip.max() < round_trip_m, trip.max()
