"""Python face of the engine context (include/wacomm_b200.h).

``Engine`` owns one device context: grid, forcing records and particles stay resident on the
GPU; every method maps to one C entry point and raises ``WacommError`` with the context's message
on a non-zero status.
"""
import ctypes

import numpy as np

from . import _native
from ._native import WacommError, options_t
from .types import PARTICLE_DTYPE, SOURCE_DTYPE, config_data

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)


def _d(a):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _f(a):
    if a is None:
        return None, None
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(_fp)


class Engine:
    """One B200 context: ``Engine(device=0, **options)``.

    Options (defaults in brackets): semantics ["host"|"device"], arithmetic ["fp32"|"reference"],
    storage ["fp32"|"fp16"|"bf16"], rng ["reference"|"philox"], block_size [256],
    substeps_per_launch [0 = whole interval], sort_by_cell [True], fuse_concentration [True],
    launch_shape [-1: 3 for the lean form, 2 for the others], surrogate [False] (needs
    set_surrogate).
    """

    _SEM = {"host": 0, "device": 1}
    _ARITH = {"reference": 0, "fp32": 1}
    _STORE = {"fp32": 0, "fp16": 1, "bf16": 2}
    _RNG = {"reference": 0, "philox": 1}

    def __init__(self, device=0, **options):
        self._lib = _native.lib()
        handle = ctypes.c_void_p()
        status = self._lib.wacomm_b200_context_create(device, ctypes.byref(handle))
        if status != 0:
            raise WacommError(status, f"cannot create a context on CUDA device {device} "
                                      f"({self._lib.wacomm_b200_device_count()} visible)")
        self._ctx = handle
        self.device = device
        self.window = None
        if options:
            self.set_options(**options)

    # -------------------------------------------------------------- plumbing
    def _check(self, status):
        if status != 0:
            raise WacommError(status, self._lib.wacomm_b200_last_error(self._ctx).decode())

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.wacomm_b200_context_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -------------------------------------------------------------- setup
    def options(self):
        o = options_t()
        self._check(self._lib.wacomm_b200_get_options(self._ctx, ctypes.byref(o)))
        return o

    def set_options(self, **kw):
        o = self.options()
        table = {"semantics": self._SEM, "arithmetic": self._ARITH, "storage": self._STORE,
                 "rng": self._RNG}
        for key, value in kw.items():
            if key in table and isinstance(value, str):
                value = table[key][value]
            setattr(o, key, int(value))
        self._check(self._lib.wacomm_b200_set_options(self._ctx, ctypes.byref(o)))

    def set_surrogate(self, weights=None):
        """Uploads the surrogate's weights: a name -> array mapping (surrogate.PARAMETERS), a
        path to a weights file, or None for the weights shipped with the package."""
        from . import surrogate
        if weights is None or isinstance(weights, str):
            weights = surrogate.load_weights(weights or surrogate.DEFAULT_WEIGHTS)
        flat = surrogate.flatten(weights)
        self._surrogate = flat
        self._check(self._lib.wacomm_b200_set_surrogate(self._ctx, flat.ctypes.data_as(_fp), len(flat)))

    def set_surrogate_error_limit(self, metres=float("inf")):
        """Particles whose estimated one-interval surrogate error exceeds `metres` take the FP32
        step (infinity: every covered particle stays with the surrogate)."""
        self._check(self._lib.wacomm_b200_set_surrogate_error_limit(self._ctx, float(metres)))

    def surrogate_stats(self):
        """dict of the last surrogate interval: particles moved by the surrogate, particles handed
        to the FP32 step, device ms of the per-cell and per-particle kernels."""
        run, fallback = ctypes.c_size_t(), ctypes.c_size_t()
        cell_ms, step_ms = ctypes.c_float(), ctypes.c_float()
        self._check(self._lib.wacomm_b200_last_surrogate_stats(
            self._ctx, ctypes.byref(run), ctypes.byref(fallback), ctypes.byref(cell_ms),
            ctypes.byref(step_ms)))
        return {"run": run.value, "fallback": fallback.value, "cell_ms": cell_ms.value,
                "step_ms": step_ms.value}

    def set_config(self, cfg):
        assert isinstance(cfg, config_data)
        self._check(self._lib.wacomm_b200_set_config(self._ctx, ctypes.byref(cfg)))

    def set_grid(self, eta, xi, s_rho, s_w, lon_rad, lat_rad, h, depth_intervals, mask=None):
        self._grid_shape = (s_rho, eta, xi)
        keep = [_d(lon_rad), _d(lat_rad), _d(h), _d(depth_intervals), _d(mask)]
        ptrs = [None if k is None else k[1] for k in keep]
        self._check(self._lib.wacomm_b200_set_grid(self._ctx, eta, xi, s_rho, s_w, ptrs[4], ptrs[0],
                                                   ptrs[1], ptrs[2], ptrs[3]))

    def set_times(self, times):
        arr, ptr = _d(times)
        self._check(self._lib.wacomm_b200_set_times(self._ctx, len(arr), ptr))

    def upload_frame(self, t, zeta, u, v, w, akt, wind_u10=None, wind_v10=None, stokes_u=None,
                     stokes_v=None):
        fields = [_f(zeta), _f(u), _f(v), _f(w), _f(akt), _f(wind_u10), _f(wind_v10),
                  _f(stokes_u), _f(stokes_v)]
        self._check(self._lib.wacomm_b200_upload_frame(self._ctx, t, *[p for _, p in fields]))

    def upload_frame_async(self, t, zeta, u, v, w, akt, wind_u10=None, wind_v10=None,
                           stokes_u=None, stokes_v=None):
        """Asynchronous upload of record t (copy stream, ordered after the enqueued kernels). The
        host arrays are kept referenced until synchronize(); pass page-locked arrays (e.g. numpy
        views of pinned torch tensors) for the copy to overlap the kernels."""
        fields = [_f(zeta), _f(u), _f(v), _f(w), _f(akt), _f(wind_u10), _f(wind_v10),
                  _f(stokes_u), _f(stokes_v)]
        self._in_flight = getattr(self, "_in_flight", {})
        self._in_flight.setdefault(t, []).append(fields)
        self._check(self._lib.wacomm_b200_upload_frame_async(self._ctx, t, *[p for _, p in fields]))

    def load_window(self, win, frames=None):
        """Grid, times and forcing records of a ``synthetic.Window``-like object."""
        self.window = win
        self.set_grid(win.eta, win.xi, win.sRho, win.sW, win.lonRad, win.latRad, win.h,
                      win.depthIntervals, win.mask)
        self.set_times(win.times)
        for t in (range(win.T) if frames is None else frames):
            f = win.frame(t)
            self.upload_frame(t, f["zeta"], f["u"], f["v"], f["w"], f["akt"], f["windU10"],
                              f["windV10"], f["stokesU"], f["stokesV"])

    # -------------------------------------------------------------- particles
    def set_particles(self, particles):
        p = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        self._check(self._lib.wacomm_b200_set_particles(self._ctx, p.ctypes.data, len(p)))

    def append_particles(self, particles):
        p = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        self._check(self._lib.wacomm_b200_append_particles(self._ctx, p.ctypes.data, len(p)))

    def count(self):
        n = ctypes.c_size_t()
        self._check(self._lib.wacomm_b200_particle_count(self._ctx, ctypes.byref(n)))
        return n.value

    def get_particles(self):
        n = self.count()
        out = np.zeros(n, dtype=PARTICLE_DTYPE)
        self._check(self._lib.wacomm_b200_get_particles(self._ctx, out.ctypes.data, n))
        return out

    # -------------------------------------------------------------- stepping
    def move_interval(self, time_index):
        self._check(self._lib.wacomm_b200_move_interval(self._ctx, time_index))

    def get_frame(self, t):
        """dict of the ocean fields of loaded record t (zeta, u, v, w, akt) as float32."""
        s_rho, eta, xi = self._grid_shape
        out = {"zeta": np.empty((eta, xi), np.float32),
               "u": np.empty((s_rho, eta, xi), np.float32),
               "v": np.empty((s_rho, eta, xi), np.float32),
               "w": np.empty((s_rho + 1, eta, xi), np.float32),
               "akt": np.empty((s_rho + 1, eta, xi), np.float32)}
        self._check(self._lib.wacomm_b200_get_frame(
            self._ctx, t, *[out[k].ctypes.data_as(_fp) for k in ("zeta", "u", "v", "w", "akt")]))
        return out

    def set_roms_grid(self, mask_u, mask_v, angle=None):
        """u-face mask [eta, xi-1], v-face mask [eta-1, xi] and the grid angle [eta, xi] in
        radians (None: velocities already east/north) for upload_roms_frame."""
        self._roms = [_d(mask_u), _d(mask_v), None if angle is None else _d(angle)]
        self._check(self._lib.wacomm_b200_set_roms_grid(
            self._ctx, self._roms[0][1], self._roms[1][1],
            None if angle is None else self._roms[2][1]))

    def upload_roms_frame(self, t, zeta, u_faces, v_faces, w, akt, wind_u10=None, wind_v10=None,
                          stokes_u=None, stokes_v=None):
        """Forcing record t from a raw ROMS record (u/v on their faces), normalized on the
        device."""
        args = [_f(a) for a in (zeta, u_faces, v_faces, w, akt, wind_u10, wind_v10, stokes_u,
                                stokes_v)]
        self._check(self._lib.wacomm_b200_upload_roms_frame(
            self._ctx, t, *[None if a is None else a[1] for a in args]))

    def graph_capture(self, first_time_index, n_intervals):
        """Records n_intervals intervals from first_time_index on as one CUDA graph."""
        self._check(self._lib.wacomm_b200_graph_capture(self._ctx, first_time_index, n_intervals))

    def graph_launch(self):
        self._check(self._lib.wacomm_b200_graph_launch(self._ctx))

    def graph_release(self):
        self._check(self._lib.wacomm_b200_graph_release(self._ctx))

    def autotune(self, time_index):
        """Times each launch configuration on interval time_index and keeps the fastest;
        returns (chosen launch_shape or block_size, its device ms). The FP32 step's work items
        per thread and the sort cadence it chooses next are in options()."""
        best, ms = ctypes.c_int(), ctypes.c_float()
        self._check(self._lib.wacomm_b200_autotune(self._ctx, time_index, ctypes.byref(best),
                                                   ctypes.byref(ms)))
        return best.value, ms.value

    def move_interval_host(self, time_index, particles):
        """Moves a host record array in place through the pipelined host-buffer entry."""
        assert particles.dtype == PARTICLE_DTYPE and particles.flags.c_contiguous
        self._check(self._lib.wacomm_b200_move_interval_host(self._ctx, time_index,
                                                             particles.ctypes.data,
                                                             len(particles)))
        return particles

    def move_interval_host_ptr(self, time_index, address, n):
        """Same as move_interval_host on a raw host address (e.g. a pinned torch tensor)."""
        self._check(self._lib.wacomm_b200_move_interval_host(self._ctx, time_index, address, n))

    def remove_dead(self):
        self._check(self._lib.wacomm_b200_remove_dead(self._ctx))

    # -------------------------------------------------------------- emission and geography
    def emit(self, sources, interval_start, interval_end, julian_start=0.0):
        """Appends the releases of ``sources`` (SOURCE_DTYPE) in [interval_start, interval_end)
        seconds, merged in time order (Sources::emit); returns how many were appended."""
        src = np.ascontiguousarray(sources, dtype=SOURCE_DTYPE)
        n = ctypes.c_size_t()
        self._check(self._lib.wacomm_b200_emit(self._ctx, src.ctypes.data if len(src) else None,
                                               len(src), julian_start, interval_start,
                                               interval_end, ctypes.byref(n)))
        return n.value

    def set_geo_grid(self, lon, lat, s_w_values):
        """Output grid of geo_positions: lon/lat [eta][xi] and the s_w coordinate values."""
        self._geo = [_d(lon), _d(lat), _d(s_w_values)]
        self._check(self._lib.wacomm_b200_set_geo_grid(self._ctx, self._geo[0][1],
                                                       self._geo[1][1], self._geo[2][1]))

    def save_text(self, path):
        """Text restart of the resident records (Particles::saveAsTxt)."""
        self._check(self._lib.wacomm_b200_save_text(self._ctx, str(path).encode()))

    def save_netcdf(self, path, checkpoint_time, **meta):
        """NetCDF history/restart of the resident records (Particles::saveAsNetCDF); meta are
        history.history_meta's keywords. Returns the number of records stored."""
        from .history import history_meta
        m = history_meta(checkpoint_time, **meta)
        written = ctypes.c_size_t()
        self._check(self._lib.wacomm_b200_save_netcdf(self._ctx, str(path).encode(),
                                                       ctypes.byref(m), ctypes.byref(written)))
        return written.value

    def geo_positions(self):
        """(depth, lat, lon) float64 arrays of the resident records (kji2deplatlon)."""
        n = self.count()
        dep, lat, lon = (np.empty(n, dtype=np.float64) for _ in range(3))
        self._check(self._lib.wacomm_b200_geo_positions(self._ctx, dep.ctypes.data_as(_dp),
                                                        lat.ctypes.data_as(_dp),
                                                        lon.ctypes.data_as(_dp), n))
        return dep, lat, lon

    REGRID_METHODS = {"geographic": _native.REGRID_BILINEAR_GEOGRAPHIC,
                      "curvilinear": _native.REGRID_BILINEAR_CURVILINEAR_GEOGRAPHIC}
    FIELDS = {"wind": _native.FIELD_WIND, "stokes": _native.FIELD_STOKES}

    def regrid_environment(self, field, method, lon, lat, times, u, v):
        """Regrids a wind or Stokes field ("wind"/"stokes") from its own grid lon/lat
        [eta', xi'] (degrees) and times [T'] to the rho nodes of set_geo_grid and the forcing
        times, on the device; u, v [T', eta', xi'] float32. method "geographic" (rectilinear
        source) or "curvilinear"."""
        lon, lat = np.ascontiguousarray(lon, np.float64), np.ascontiguousarray(lat, np.float64)
        times = np.ascontiguousarray(times, np.float64)
        u, v = np.ascontiguousarray(u, np.float32), np.ascontiguousarray(v, np.float32)
        if lon.ndim != 2 or lat.shape != lon.shape or u.shape != (times.size,) + lon.shape or \
                v.shape != u.shape:
            raise ValueError(f"shapes lon {lon.shape} lat {lat.shape} times {times.shape} "
                             f"u {u.shape} v {v.shape}")
        self._check(self._lib.wacomm_b200_regrid_environment(
            self._ctx, self.FIELDS[field], self.REGRID_METHODS[method], lon.shape[0], lon.shape[1],
            lon.ctypes.data_as(_dp), lat.ctypes.data_as(_dp), times.size, times.ctypes.data_as(_dp),
            u.ctypes.data_as(_fp), v.ctypes.data_as(_fp)))

    def clear_environment(self, field):
        self._check(self._lib.wacomm_b200_clear_environment(self._ctx, self.FIELDS[field]))

    def environment(self, field, t):
        """(u, v) float32 [eta, xi] of the regridded field at forcing time t."""
        eta, xi = self._grid_shape[1:]
        u, v = (np.empty((eta, xi), np.float32) for _ in range(2))
        self._check(self._lib.wacomm_b200_get_environment(self._ctx, self.FIELDS[field], t,
                                                          u.ctypes.data_as(_fp),
                                                          v.ctypes.data_as(_fp)))
        return u, v

    def synchronize(self):
        self._check(self._lib.wacomm_b200_synchronize(self._ctx))
        self._in_flight = {}

    def steps_total(self, reset=False):
        """Particle-steps of every interval since creation or the last reset (device-summed)."""
        total = ctypes.c_double()
        self._check(self._lib.wacomm_b200_particle_steps_total(self._ctx, int(bool(reset)),
                                                               ctypes.byref(total)))
        return total.value

    def stats(self):
        """dict of the last interval: device ms of all kernels, ms of the move launches, kernel
        launches and particle-steps."""
        ms, move_ms = ctypes.c_float(), ctypes.c_float()
        launches = ctypes.c_int()
        steps = ctypes.c_double()
        self._check(self._lib.wacomm_b200_last_interval_stats(
            self._ctx, ctypes.byref(ms), ctypes.byref(move_ms), ctypes.byref(launches),
            ctypes.byref(steps)))
        return {"device_ms": ms.value, "move_ms": move_ms.value, "launches": launches.value,
                "particle_steps": steps.value}

    def kernel_times(self, capacity=256):
        """(n, 3) array of device ms of the dominant kernels of the eager intervals enqueued since
        the last call, oldest first: [move, 0, 0] for the plain step, [step kernel, post or walk
        kernel, fallback step] with the surrogate."""
        out = np.zeros((capacity, 3), dtype=np.float32)
        n = ctypes.c_int()
        self._check(self._lib.wacomm_b200_kernel_times(
            self._ctx, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), capacity,
            ctypes.byref(n)))
        return out[:n.value].copy()

    @property
    def stream(self):
        """Address of the context's cudaStream_t (for torch.cuda.ExternalStream)."""
        out = ctypes.c_void_p()
        self._check(self._lib.wacomm_b200_stream(self._ctx, ctypes.byref(out)))
        return out.value

    # -------------------------------------------------------------- concentration
    def concentration_reset(self, n_times):
        self._check(self._lib.wacomm_b200_concentration_reset(self._ctx, n_times))
        self._conc_times = n_times

    def concentration_count(self, conc_time_index):
        self._check(self._lib.wacomm_b200_concentration_count(self._ctx, conc_time_index))

    def _conc_shape(self):
        return (self._conc_times,) + self._grid_shape

    def concentration(self):
        out = np.zeros(self._conc_shape(), dtype=np.uint32)
        self._check(self._lib.wacomm_b200_concentration_get(self._ctx, out.ctypes.data, out.size))
        return out

    def concentration_device(self):
        """(device address, cell count) of the context's uint32 concentration grid."""
        ptr, cells = ctypes.c_void_p(), ctypes.c_size_t()
        self._check(self._lib.wacomm_b200_concentration_device(self._ctx, ctypes.byref(ptr),
                                                               ctypes.byref(cells)))
        return ptr.value, cells.value

    def concentration_view(self, conc_time_index=None):
        """A torch int32 tensor on the context's device aliasing the uint32 concentration grid
        [n_times][s_rho][eta][xi] (or one time slice of it), for collectives across shards; the
        bits are the uint32 counts."""
        import torch
        ptr, cells = self.concentration_device()
        shape = self._conc_shape()
        plane = int(np.prod(shape[1:]))
        if conc_time_index is not None:
            ptr += 4 * plane * conc_time_index
            shape = shape[1:]
        device = torch.device("cuda", self.device)

        class _Grid:
            __cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<i4",
                                        "data": (ptr, False), "version": 3, "strides": None}
        return torch.as_tensor(_Grid(), device=device)

    def concentration_float(self, mask_land=False):
        out = np.zeros(self._conc_shape(), dtype=np.float32)
        self._check(self._lib.wacomm_b200_concentration_get_float(self._ctx, out.ctypes.data,
                                                                  out.size, int(mask_land)))
        return out
