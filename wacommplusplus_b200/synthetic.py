"""Seeded synthetic forcing windows and particle sets.

The reference's benchmark forcing (the Sarno ROMS run) is not available, so every workload
here is generated from a fixed seed with the shapes, sizes and value distributions the
benchmark configurations describe. Arrays follow the reference device layout
(kernel.cu:63-69): zeta/wind/Stokes [T][eta][xi]; u,v [T][sRho][eta][xi];
w,akt [T][sW][eta][xi] (storage level = logical k + levels - 1, level 0 at the bottom);
depthIntervals[sW-1] indexed kI+sW-2 with depthIntervals(k) = sW(k) - sW(k-1)
(WacommAdapter.cpp:101-103); sWValues[sW] indexed k+sW-1; 2-D fields [eta][xi].
lonRad/latRad use the adapters' factor 0.0174533 (WacommAdapter.cpp:109-110), or exact
pi/180 when ``exact_pi`` is set.
"""
import math

import numpy as np

from .types import PARTICLE_DTYPE

ADAPTER_DEG2RAD = 0.0174533
EXACT_DEG2RAD = math.pi / 180.0
# 2021-07-01T00:00Z in seconds since 1968-05-23 (the reference's modified-Julian origin).
EPOCH_2021_07_01 = 1675900800.0


class Window:
    """A forcing window plus its grid; attribute names follow the reference contract."""

    def __init__(self, **fields):
        self.windU10 = self.windV10 = self.stokesU = self.stokesV = None
        for key, value in fields.items():
            setattr(self, key, value)
        self.T = len(self.times)
        self.eta, self.xi = self.h.shape
        self.sW = len(self.sWValues)
        self.sRho = self.sW - 1

    def frame(self, t):
        """Fields of forcing record ``t`` (views)."""
        out = {"zeta": self.zeta[t], "u": self.u[t], "v": self.v[t], "w": self.w[t],
               "akt": self.akt[t]}
        for name in ("windU10", "windV10", "stokesU", "stokesV"):
            field = getattr(self, name)
            out[name] = None if field is None else field[t]
        return out

    @property
    def nbytes_frame(self):
        plane = self.eta * self.xi
        n = plane * (1 + 2 * self.sRho + 2 * self.sW)
        n += plane * sum(getattr(self, f) is not None
                         for f in ("windU10", "windV10", "stokesU", "stokesV"))
        return 4 * n


def _depth_intervals(sw_values):
    return np.ascontiguousarray(np.diff(sw_values)[0:], dtype=np.float64)


def rectilinear_grid(eta, xi, lon0, lon1, lat0, lat1, exact_pi=False):
    lon = np.broadcast_to(np.linspace(lon0, lon1, xi)[None, :], (eta, xi)).copy()
    lat = np.broadcast_to(np.linspace(lat0, lat1, eta)[:, None], (eta, xi)).copy()
    factor = EXACT_DEG2RAD if exact_pi else ADAPTER_DEG2RAD
    return lon, lat, factor * lon, factor * lat


def config1_window(n_frames=6, exact_pi=False, t0=EPOCH_2021_07_01, u=0.2, v=0.1,
                   akt=1.0e-4, eta=128, xi=128, s_rho=10):
    """Plain analytic case: 128x128 rho nodes over lon 14.00-14.20 E, lat 40.70-40.90 N,
    10 sigma levels with sW=k/10, h=50 m, zeta=0, no land, uniform u=0.2, v=0.1 m/s, w=0,
    AKT=1e-4 m2/s, hourly frames."""
    lon, lat, lon_rad, lat_rad = rectilinear_grid(eta, xi, 14.0, 14.2, 40.7, 40.9, exact_pi)
    s_w = s_rho + 1
    sw_values = np.array([k / s_rho for k in range(-s_w + 1, 1)], dtype=np.float64)
    T = n_frames
    shape3 = (T, eta, xi)
    return Window(
        times=t0 + 3600.0 * np.arange(T, dtype=np.float64),
        mask=np.ones((eta, xi)), lon=lon, lat=lat, lonRad=lon_rad, latRad=lat_rad,
        h=np.full((eta, xi), 50.0), sWValues=sw_values,
        depthIntervals=_depth_intervals(sw_values),
        zeta=np.zeros(shape3, dtype=np.float32),
        u=np.full((T, s_rho, eta, xi), u, dtype=np.float32),
        v=np.full((T, s_rho, eta, xi), v, dtype=np.float32),
        w=np.zeros((T, s_w, eta, xi), dtype=np.float32),
        akt=np.full((T, s_w, eta, xi), akt, dtype=np.float32),
    )


def uniform_particles(n, eta, xi, seed=1, depth_max=5.0, h=50.0, sw1=0.1, time=0.0,
                      first_id=0):
    """``n`` passive particles uniform over the interpolation domain (0<=j<eta-1,
    0<=i<xi-1) at depths uniform in [0, depth_max] m. On a flat-bottom grid with
    sW(-1)=-sw1 the inverse vertical map of deplatlon2kji (OceanModelAdapter.cpp:426-441)
    is k = -dep/(h*sw1) inside the upper W interval."""
    rng = np.random.default_rng(seed)
    out = np.zeros(n, dtype=PARTICLE_DTYPE)
    out["id"] = np.arange(first_id, first_id + n, dtype=np.uint64)
    out["j"] = rng.uniform(0.0, eta - 1, n)
    out["i"] = rng.uniform(0.0, xi - 1, n)
    out["k"] = -rng.uniform(0.0, depth_max, n) / (h * sw1)
    out["health"] = 1.0
    out["time"] = time
    return out


# ------------------------------------------------------------------ realistic ROMS-like case


def _smooth_field(rng, eta, xi, length_cells):
    """Zero-mean, unit-variance Gaussian random field with a Gaussian spectrum."""
    noise = rng.standard_normal((eta, xi))
    ky = np.fft.fftfreq(eta)[:, None]
    kx = np.fft.rfftfreq(xi)[None, :]
    filt = np.exp(-0.5 * (2 * np.pi * length_cells) ** 2 * (kx ** 2 + ky ** 2))
    field = np.fft.irfft2(np.fft.rfft2(noise) * filt, s=(eta, xi))
    field -= field.mean()
    return field / (field.std() + 1e-30)


def vtransform2_sw(n_levels, theta_s=5.0, theta_b=0.4, hc=20.0, h_ref=100.0):
    """Depth fractions of W levels under ROMS Vtransform 2 / Vstretching 4 for a
    reference depth, from the bottom (-1) to the surface (0)."""
    s = (np.arange(n_levels + 1) - n_levels) / n_levels
    c = (1.0 - np.cosh(theta_s * s)) / (np.cosh(theta_s) - 1.0)
    c = (np.exp(theta_b * c) - 1.0) / (1.0 - np.exp(-theta_b))
    z = (hc * s + h_ref * c) / (hc + h_ref)
    z[0], z[-1] = -1.0, 0.0
    return z.astype(np.float64)


class RealisticForcing:
    """ROMS-shaped synthetic forcing: Vtransform-2 levels, 10-200 m bathymetry from a smooth
    random field, ~20% land inside a wet border (h=0, mask=0 as ROMSAdapter.cpp:244-252 sets it), u,v from a
    divergence-free streamfunction of 64 random Fourier modes (rms 0.3 m/s, wavelengths
    2-50 km, phases advancing hourly), w ~ N(0, 1e-4) m/s, AKT log-normal (median 1e-4,
    sigma 1). Frames are generated on demand from the seed."""

    def __init__(self, eta=1024, xi=1024, s_rho=30, n_frames=24, seed=2, t0=EPOCH_2021_07_01,
                 dlon=0.001, dlat=0.001, lon0=13.9, lat0=40.2, land_fraction=0.2, modes=64,
                 water_border=4):
        self.eta, self.xi, self.s_rho, self.s_w = eta, xi, s_rho, s_rho + 1
        self.n_frames, self.seed = n_frames, seed
        rng = np.random.default_rng(seed)
        lon1, lat1 = lon0 + dlon * (xi - 1), lat0 + dlat * (eta - 1)
        self.lon, self.lat, self.lonRad, self.latRad = rectilinear_grid(eta, xi, lon0, lon1,
                                                                        lat0, lat1)
        self.times = t0 + 3600.0 * np.arange(n_frames, dtype=np.float64)
        depth = _smooth_field(rng, eta, xi, max(eta, xi) / 24.0)
        h = 10.0 + 190.0 * (0.5 + 0.5 * np.tanh(depth))
        land_noise = _smooth_field(rng, eta, xi, max(eta, xi) / 32.0)
        land = land_noise > np.quantile(land_noise, 1.0 - land_fraction)
        if water_border > 0:
            # Open boundaries stay wet: a particle reflected at the domain edge
            # (NumericalHelpers.hpp:67-74) is placed without a land test, and a fully dry
            # cell there would give a zero cell height (0/0 in the reference step).
            b = water_border
            land[:b, :] = land[-b:, :] = False
            land[:, :b] = land[:, -b:] = False
        self.mask = np.where(land, 0.0, 1.0)
        self.h = np.where(land, 0.0, h)
        self.sWValues = vtransform2_sw(s_rho)
        self.depthIntervals = _depth_intervals(self.sWValues)
        # Fourier modes of the streamfunction, metres and seconds
        R = 6371000.0
        self.dx = R * math.cos(math.radians(0.5 * (lat0 + lat1))) * math.radians(dlon)
        self.dy = R * math.radians(dlat)
        wavelength = np.exp(rng.uniform(np.log(2000.0), np.log(50000.0), modes))
        theta = rng.uniform(0, 2 * np.pi, modes)
        self.kx = 2 * np.pi / wavelength * np.cos(theta)
        self.ky = 2 * np.pi / wavelength * np.sin(theta)
        self.phase = rng.uniform(0, 2 * np.pi, modes)
        self.omega = rng.uniform(-0.5, 0.5, modes)  # phase advance per hour
        amp = rng.standard_normal(modes)
        # velocity amplitude of mode m is amp*|k|; normalise to rms 0.3 m/s overall
        kmag = np.hypot(self.kx, self.ky)
        self.amp = amp * 0.3 / np.sqrt(0.5 * np.sum((amp * kmag) ** 2))
        self.water = ~land

    def window(self, frames=None):
        """A Window holding ``frames`` (default: all) generated records."""
        frames = range(self.n_frames) if frames is None else frames
        frames = list(frames)
        T = len(frames)
        e, x = self.eta, self.xi
        out = dict(zeta=np.zeros((T, e, x), np.float32),
                   u=np.zeros((T, self.s_rho, e, x), np.float32),
                   v=np.zeros((T, self.s_rho, e, x), np.float32),
                   w=np.zeros((T, self.s_w, e, x), np.float32),
                   akt=np.zeros((T, self.s_w, e, x), np.float32))
        for n, t in enumerate(frames):
            f = self.frame(t)
            for key in out:
                out[key][n] = f[key]
        return Window(times=self.times[frames].copy(), mask=self.mask, lon=self.lon,
                      lat=self.lat, lonRad=self.lonRad, latRad=self.latRad, h=self.h,
                      sWValues=self.sWValues, depthIntervals=self.depthIntervals, **out)

    def frame(self, t):
        e, x = self.eta, self.xi
        rng = np.random.default_rng((self.seed, 1000 + t))
        X = (np.arange(x) * self.dx)[None, :]
        Y = (np.arange(e) * self.dy)[:, None]
        u = np.zeros((e, x))
        v = np.zeros((e, x))
        for m in range(len(self.amp)):
            arg = self.kx[m] * X + self.ky[m] * Y + self.phase[m] + self.omega[m] * t
            s = np.sin(arg)
            # psi = amp cos(arg): u = -dpsi/dy, v = dpsi/dx
            u += self.amp[m] * self.ky[m] * s
            v -= self.amp[m] * self.kx[m] * s
        u *= self.water
        v *= self.water
        s_rho_mid = 0.5 * (self.sWValues[1:] + self.sWValues[:-1])
        decay = (1.0 + 0.5 * s_rho_mid)[:, None, None]
        frame = {
            "zeta": (0.2 * np.sin(2 * np.pi * t / 12.4) * self.water).astype(np.float32),
            "u": (decay * u[None]).astype(np.float32),
            "v": (decay * v[None]).astype(np.float32),
            "w": (rng.standard_normal((self.s_w, e, x)) * 1.0e-4 * self.water).astype(np.float32),
            "akt": (1.0e-4 * np.exp(rng.standard_normal((self.s_w, e, x))) * self.water).astype(
                np.float32),
        }
        return frame

    def frame_device(self, t, device="cuda"):
        """Record t as ``frame`` builds it, evaluated with torch on ``device`` (FP64 mode sums as
        in ``frame``; the w and AKT noise from torch's generator seeded by (seed, t), so it
        differs from ``frame``'s NumPy draws) and returned as host float32 arrays: a second
        for the 24 records of the 1024x1024x30 grid instead of about fifty."""
        import torch
        e, x = self.eta, self.xi
        dev = torch.device(device)
        X = (torch.arange(x, device=dev, dtype=torch.float64) * self.dx)[None, :]
        Y = (torch.arange(e, device=dev, dtype=torch.float64) * self.dy)[:, None]
        u = torch.zeros((e, x), device=dev, dtype=torch.float64)
        v = torch.zeros((e, x), device=dev, dtype=torch.float64)
        for m in range(len(self.amp)):
            s = torch.sin(self.kx[m] * X + self.ky[m] * Y + self.phase[m] + self.omega[m] * t)
            u += self.amp[m] * self.ky[m] * s
            v -= self.amp[m] * self.kx[m] * s
        water = torch.as_tensor(self.water, device=dev)
        u = torch.where(water, u, 0.0)
        v = torch.where(water, v, 0.0)
        s_rho_mid = 0.5 * (self.sWValues[1:] + self.sWValues[:-1])
        decay = torch.as_tensor(1.0 + 0.5 * s_rho_mid, device=dev)[:, None, None]
        gen = torch.Generator(device=dev)
        gen.manual_seed(int(self.seed) * 1_000_003 + 1000 + int(t))
        shape = (self.s_w, e, x)
        w = torch.randn(shape, generator=gen, device=dev, dtype=torch.float32) * 1.0e-4
        akt = 1.0e-4 * torch.exp(torch.randn(shape, generator=gen, device=dev, dtype=torch.float32))
        water32 = water.to(torch.float32)
        zeta = 0.2 * math.sin(2 * math.pi * t / 12.4) * water32
        return {"zeta": zeta.cpu().numpy(),
                "u": (decay * u[None]).to(torch.float32).cpu().numpy(),
                "v": (decay * v[None]).to(torch.float32).cpu().numpy(),
                "w": (w * water32).cpu().numpy(),
                "akt": (akt * water32).cpu().numpy()}

    def window_of(self, frames, records):
        """A Window of the given record indices from already generated ``records`` (dicts as
        ``frame`` returns them, in the same order)."""
        out = {key: np.stack([r[key] for r in records]) for key in records[0]}
        frames = list(frames)
        return Window(times=self.times[frames].copy(), mask=self.mask, lon=self.lon,
                      lat=self.lat, lonRad=self.lonRad, latRad=self.latRad, h=self.h,
                      sWValues=self.sWValues, depthIntervals=self.depthIntervals, **out)

    def sources(self, n_sources=64, seed=3):
        """Point sources on water cells away from land: (k, j, i) positions."""
        rng = np.random.default_rng(seed)
        water = self.water.copy()
        deep = water & (self.h > 20.0)
        cand = np.argwhere(deep[2:-2, 2:-2]) + 2
        pick = cand[rng.choice(len(cand), n_sources, replace=False)]
        j = pick[:, 0] + rng.uniform(0, 1, n_sources)
        i = pick[:, 1] + rng.uniform(0, 1, n_sources)
        k = -rng.uniform(0.0, 0.5, n_sources)
        return np.stack([k, j, i], axis=1)

    def release(self, n_particles, n_sources=64, seed=3, spread=0.25):
        """``n_particles`` particles from ``n_sources`` point sources at uniform rates over the
        window: release times (n+1/2)*3600/R after the first record (SourceEmission.hpp:68-77)
        with ids in time order, positions jittered by ``spread`` index units like the seeded
        source offsets (SourceEmission.hpp:20-23)."""
        rng = np.random.default_rng(seed)
        src = self.sources(n_sources, seed)
        per_source = n_particles // n_sources
        duration = 3600.0 * (self.n_frames - 1)
        rate = per_source / (duration / 3600.0)
        spacing = 3600.0 / rate
        times = self.times[0] + (np.arange(per_source) + 0.5) * spacing
        all_t = np.repeat(times[None, :], n_sources, axis=0).reshape(-1)
        all_s = np.repeat(np.arange(n_sources)[:, None], per_source, axis=1).reshape(-1)
        order = np.lexsort((all_s, all_t))
        out = np.zeros(len(order), dtype=PARTICLE_DTYPE)
        out["id"] = np.arange(len(order), dtype=np.uint64)
        s_idx = all_s[order]
        out["time"] = all_t[order]
        out["k"] = np.clip(src[s_idx, 0] + spread * rng.standard_normal(len(order)), -1.0, 0.0)
        out["j"] = src[s_idx, 1] + spread * rng.standard_normal(len(order))
        out["i"] = src[s_idx, 2] + spread * rng.standard_normal(len(order))
        out["health"] = 1.0
        return out


# ------------------------------------------------------------------ wind and Stokes on own grids


def wind_grid(n=340, spacing_m=3000.0, lon0=14.1, lat0=40.8, rotation_deg=8.0):
    """A weather-model grid of n x n nodes ``spacing_m`` apart (340 x 340 at 3 km: ~1,000 km
    across), rotated by ``rotation_deg`` and centred on (lon0, lat0): node positions on a local
    tangent plane mapped to degrees with the latitude-dependent longitude scale, so that lon and
    lat both vary along both index directions (curvilinear, like a Lambert-conformal WRF grid).
    Returns lon, lat [n, n] in degrees."""
    R = 6371000.0
    c = (n - 1) / 2.0
    j, i = np.mgrid[0:n, 0:n].astype(np.float64)
    x, y = (i - c) * spacing_m, (j - c) * spacing_m
    r = math.radians(rotation_deg)
    xr, yr = x * math.cos(r) - y * math.sin(r), x * math.sin(r) + y * math.cos(r)
    lat = lat0 + np.degrees(yr / R)
    lon = lon0 + np.degrees(xr / (R * np.cos(np.radians(lat))))
    return lon, lat


def stokes_grid(lon0=13.5, lon1=14.7, lat0=40.2, lat1=41.4, step=0.05):
    """A rectilinear wave-model grid at ``step`` degrees (0.05 by default) around the analytic
    ocean domain. Returns lon, lat [eta, xi] in degrees."""
    lon1d = lon0 + step * np.arange(int(round((lon1 - lon0) / step)) + 1)
    lat1d = lat0 + step * np.arange(int(round((lat1 - lat0) / step)) + 1)
    return np.meshgrid(lon1d, lat1d)


def vector_series(shape, n_times, rms, seed, length_cells, period_records=24.0):
    """(u, v) float32 [n_times, *shape]: smooth random vector fields of rms ``rms`` per component
    turning slowly in time (two random fields per component mixed with phases advancing
    2*pi/period_records per record)."""
    rng = np.random.default_rng(seed)
    eta, xi = shape
    a, b, c, d = (_smooth_field(rng, eta, xi, length_cells) for _ in range(4))
    out_u = np.empty((n_times,) + shape, np.float32)
    out_v = np.empty((n_times,) + shape, np.float32)
    for t in range(n_times):
        ph = 2 * np.pi * t / period_records
        out_u[t] = rms * (math.cos(ph) * a + math.sin(ph) * b)
        out_v[t] = rms * (math.cos(ph) * c + math.sin(ph) * d)
    return out_u, out_v


def environment(t0, hours, wind_n=340, seed=11):
    """The batched workload's native environmental forcing over ``hours`` hours from t0: wind on
    the curvilinear 3 km grid, hourly, rms 8 m/s; Stokes drift on the 0.05-degree grid,
    3-hourly, rms 0.1 m/s. dict of (lon, lat, times, u, v) per field."""
    wlon, wlat = wind_grid(wind_n)
    wt = t0 + 3600.0 * np.arange(hours + 1)
    wu, wv = vector_series(wlon.shape, len(wt), 8.0, seed, wind_n / 12.0)
    slon, slat = stokes_grid()
    st = t0 + 10800.0 * np.arange(hours // 3 + 1 + (hours % 3 > 0))
    su, sv = vector_series(slon.shape, len(st), 0.1, seed + 1, 3.0, period_records=8.0)
    return {"wind": (wlon, wlat, wt, wu, wv), "stokes": (slon, slat, st, su, sv)}


def batched_scenarios(win, n_scenarios=256, seed=5, smallest=1000, largest=256000,
                      release_hours=24.0, first_id=0):
    """Independent drift scenarios batched into one particle set: scenario s has a size drawn
    log-uniform in [smallest, largest] (about 11.8 M in all for 256), its own point source (an
    interior cell of the grid, 0-1 m deep), its own release window (start uniform in the first
    ``release_hours`` hours, 1-6 h long, uniform rate) and its own drift object of the leeway
    catalogue (types 1-22; side left or right per particle). Returns (records, table) with the
    table giving per scenario: first record, size, object type, release start and end (s)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(smallest), np.log(largest), n_scenarios)).astype(np.int64)
    total = int(sizes.sum())
    out = np.zeros(total, dtype=PARTICLE_DTYPE)
    table = np.zeros(n_scenarios, dtype=[("first", "<i8"), ("size", "<i8"), ("type", "<u2"),
                                         ("start", "<f8"), ("end", "<f8")])
    sw1 = 0.1
    at = 0
    for s, n in enumerate(sizes):
        j0, i0 = rng.uniform(8, win.eta - 9), rng.uniform(8, win.xi - 9)
        start = win.times[0] + rng.uniform(0, release_hours * 3600.0)
        length = rng.uniform(1.0, 6.0) * 3600.0
        kind = int(rng.integers(1, 23))
        rec = out[at:at + n]
        rec["id"] = np.arange(first_id + at, first_id + at + n, dtype=np.uint64)
        rec["j"] = j0 + 0.25 * rng.standard_normal(n)
        rec["i"] = i0 + 0.25 * rng.standard_normal(n)
        rec["k"] = -rng.uniform(0.0, 1.0, n) / (win.h[0, 0] * sw1)
        rec["health"] = 1.0
        rec["time"] = start + (np.arange(n) + 0.5) * (length / n)
        rec["driftObjectType"] = kind
        rec["driftSide"] = rng.choice(np.array([-1, 1], np.int8), n)
        table[s] = (at, n, kind, start, start + length)
        at += n
    return out, table
