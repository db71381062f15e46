"""ctypes bindings of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loaded only by tests/, by ``__graft_entry__.smoke()`` and by the CPU-baseline leg of
bench.py, as the checker. Two libraries:

* ``liboracle.so``: our plain-C restatement of the reference path (wacomm_oracle.c);
* ``_ref/libwacomm_ref.so``: the reference's own ``Particle::move`` and helpers compiled from
  its sources (present only where it was built; ``ref_available()`` tells).
"""
import ctypes
import os

import numpy as np

from wacommplusplus_b200.types import PARTICLE_DTYPE, SOURCE_DTYPE, config_data

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libwacomm_ref.so")
REF_CUDA_SO = os.path.join(HERE, "_ref", "libwacomm_ref_cuda.so")

SEMANTICS_HOST = 0
SEMANTICS_DEVICE = 1

_c_double_p = ctypes.POINTER(ctypes.c_double)
_c_float_p = ctypes.POINTER(ctypes.c_float)


class _Window(ctypes.Structure):
    _fields_ = [
        ("T", ctypes.c_int), ("sW", ctypes.c_int), ("sRho", ctypes.c_int),
        ("eta", ctypes.c_int), ("xi", ctypes.c_int),
        ("times", _c_double_p), ("mask", _c_double_p), ("lonRad", _c_double_p),
        ("latRad", _c_double_p), ("depthIntervals", _c_double_p), ("h", _c_double_p),
        ("zeta", _c_float_p), ("u", _c_float_p), ("v", _c_float_p), ("w", _c_float_p),
        ("akt", _c_float_p),
        ("windU10", _c_float_p), ("windV10", _c_float_p),
        ("stokesU", _c_float_p), ("stokesV", _c_float_p),
    ]


def _dptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_c_double_p)


def _fptr(a):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_c_float_p)


def _window_struct(win):
    s = _Window()
    s.T, s.sW, s.sRho, s.eta, s.xi = win.T, win.sW, win.sRho, win.eta, win.xi
    s.times, s.mask = _dptr(win.times), _dptr(win.mask)
    s.lonRad, s.latRad = _dptr(win.lonRad), _dptr(win.latRad)
    s.depthIntervals, s.h = _dptr(win.depthIntervals), _dptr(win.h)
    s.zeta, s.u, s.v = _fptr(win.zeta), _fptr(win.u), _fptr(win.v)
    s.w, s.akt = _fptr(win.w), _fptr(win.akt)
    s.windU10, s.windV10 = _fptr(win.windU10), _fptr(win.windV10)
    s.stokesU, s.stokesV = _fptr(win.stokesU), _fptr(win.stokesV)
    return s


_oracle = None
_ref = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"oracle library missing: {ORACLE_SO} (run make -C oracle)")
        lib = ctypes.CDLL(ORACLE_SO)
        u64, i64, d = ctypes.c_uint64, ctypes.c_int64, ctypes.c_double
        lib.wo_uniform.restype = d
        lib.wo_uniform.argtypes = [u64, u64, i64, u64, u64]
        lib.wo_normal.restype = d
        lib.wo_normal.argtypes = [u64, u64, i64, u64, u64]
        lib.wo_mix.restype = u64
        lib.wo_mix.argtypes = [u64]
        lib.wo_forcing_error_normal.restype = d
        lib.wo_forcing_error_normal.argtypes = [u64, u64, i64, u64, u64, d, d, d, d, d]
        lib.wo_jibe_step_probability.restype = d
        lib.wo_jibe_step_probability.argtypes = [d, d]
        lib.wo_correlated_normal.restype = d
        lib.wo_correlated_normal.argtypes = [d, d, d]
        lib.wo_drift_coefficients.restype = ctypes.c_int
        lib.wo_drift_coefficients.argtypes = [ctypes.c_int, _c_double_p]
        lib.wo_compute_leeway.restype = None
        lib.wo_compute_leeway.argtypes = [_c_double_p, d, d, ctypes.c_int, d, d, _c_double_p]
        lib.wo_sample_drift_side.restype = ctypes.c_int
        lib.wo_sample_drift_side.argtypes = [u64, u64, d]
        lib.wo_restart_elapsed.restype = d
        lib.wo_restart_elapsed.argtypes = [d, d, d]
        lib.wo_reflect_cell.restype = d
        lib.wo_reflect_cell.argtypes = [d, ctypes.c_int, d, ctypes.c_int]
        lib.wo_reflect_domain.restype = d
        lib.wo_reflect_domain.argtypes = [d, d]
        lib.wo_move_batch.restype = ctypes.c_int
        lib.wo_move_batch.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long,
                                      ctypes.POINTER(_Window), ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int]
        lib.wo_concentration.restype = None
        lib.wo_concentration.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_void_p]
        lib.wo_concentration_mask.restype = None
        lib.wo_concentration_mask.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_int, _c_double_p]
        lib.wo_source_emission_times.restype = ctypes.c_long
        lib.wo_source_emission_times.argtypes = [ctypes.c_int, d, d, d, d, d, _c_double_p,
                                                 ctypes.c_long]
        lib.wo_source_position_offset.restype = d
        lib.wo_source_position_offset.argtypes = [u64, u64, u64]
        lib.wo_sources_emit.restype = ctypes.c_long
        lib.wo_sources_emit.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, d, d, d,
                                        u64, ctypes.c_void_p, ctypes.c_long]
        geo = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _c_double_p, _c_double_p, _c_double_p,
               _c_double_p, d, d, d, _c_double_p, _c_double_p, _c_double_p]
        lib.wo_kji2deplatlon.restype = ctypes.c_int
        lib.wo_kji2deplatlon.argtypes = geo
        lib.wo_deplatlon2kji.restype = ctypes.c_int
        lib.wo_deplatlon2kji.argtypes = geo
        lib.wo_text_restart.restype = ctypes.c_int
        lib.wo_text_restart.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]
        _oracle = lib
    return _oracle


def ref_available():
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError(f"reference build missing: {REF_SO}")
        lib = ctypes.CDLL(REF_SO)
        u64, i64, d = ctypes.c_uint64, ctypes.c_int64, ctypes.c_double
        vp, i32, lng = ctypes.c_void_p, ctypes.c_int, ctypes.c_long
        lib.ref_move_batch.restype = i32
        lib.ref_move_batch.argtypes = [vp, vp, lng, i32, i32, i32, i32, i32, i32] + [vp] * 16 + [i32]
        lib.ref_concentration.restype = i32
        lib.ref_concentration.argtypes = [vp, lng, i32, i32, i32, i32, i32, vp, i32]
        lib.ref_remove_dead.restype = lng
        lib.ref_remove_dead.argtypes = [vp, lng]
        for name in ("ref_uniform", "ref_normal"):
            getattr(lib, name).restype = d
            getattr(lib, name).argtypes = [u64, u64, i64, u64, u64]
        lib.ref_forcing_error_normal.restype = d
        lib.ref_forcing_error_normal.argtypes = [u64, u64, i64, u64, u64, d, d, d, d, d]
        lib.ref_drift_coefficients.restype = None
        lib.ref_drift_coefficients.argtypes = [i32, _c_double_p]
        lib.ref_compute_leeway.restype = None
        lib.ref_compute_leeway.argtypes = [_c_double_p, d, d, i32, d, d, _c_double_p]
        lib.ref_jibe_step_probability.restype = d
        lib.ref_jibe_step_probability.argtypes = [d, d]
        lib.ref_sample_drift_side.restype = i32
        lib.ref_sample_drift_side.argtypes = [u64, u64, d]
        lib.ref_source_position_offset.restype = d
        lib.ref_source_position_offset.argtypes = [u64, u64, u64]
        lib.ref_source_emission_times.restype = lng
        lib.ref_source_emission_times.argtypes = [i32, d, d, d, d, d, _c_double_p, lng]
        lib.ref_reflect_domain.restype = d
        lib.ref_reflect_domain.argtypes = [d, d]
        lib.ref_reflect_cell.restype = d
        lib.ref_reflect_cell.argtypes = [d, i32, d, i32]
        lib.ref_restart_elapsed.restype = d
        lib.ref_restart_elapsed.argtypes = [d, d, d]
        lib.ref_max_threads.restype = i32
        _ref = lib
    return _ref


def _cfg_ptr(cfg):
    assert isinstance(cfg, config_data)
    return ctypes.cast(ctypes.pointer(cfg), ctypes.c_void_p)


def oracle_move(cfg, particles, win, time_index, semantics=SEMANTICS_HOST, threads=0):
    """Moves ``particles`` (PARTICLE_DTYPE array, updated in place) over one interval with the
    C restatement. Raises on a drift object outside the catalogue in host semantics."""
    assert particles.dtype == PARTICLE_DTYPE and particles.flags.c_contiguous
    ws = _window_struct(win)
    status = oracle_lib().wo_move_batch(_cfg_ptr(cfg), particles.ctypes.data, len(particles),
                                        ctypes.byref(ws), time_index, semantics, threads)
    if status != 0:
        raise RuntimeError("oracle: drift object outside the catalogue")
    return particles


def ref_move(cfg, particles, win, time_index, threads=0):
    """Moves ``particles`` in place with the reference Particle::move (OpenMP dynamic,64)."""
    assert particles.dtype == PARTICLE_DTYPE and particles.flags.c_contiguous
    lib = ref_lib()
    ptr = lambda a: None if a is None else a.ctypes.data
    lib.ref_move_batch(_cfg_ptr(cfg), particles.ctypes.data, len(particles), time_index,
                       win.T, win.sW, win.sRho, win.eta, win.xi,
                       ptr(win.times), ptr(win.mask), ptr(win.lonRad), ptr(win.latRad),
                       ptr(win.sWValues), ptr(win.depthIntervals), ptr(win.h), ptr(win.zeta),
                       ptr(win.u), ptr(win.v), ptr(win.w), ptr(win.akt),
                       ptr(win.windU10), ptr(win.windV10), ptr(win.stokesU), ptr(win.stokesV),
                       threads)
    return particles


def oracle_concentration(particles, conc_time_index, n_times, win):
    """uint32 counts [n_times][sRho][eta][xi] of the alive particles at conc_time_index."""
    conc = np.zeros((n_times, win.sRho, win.eta, win.xi), dtype=np.uint32)
    oracle_lib().wo_concentration(particles.ctypes.data, len(particles), conc_time_index,
                                  n_times, win.sRho, win.eta, win.xi, conc.ctypes.data)
    return conc


def oracle_concentration_float(counts, evaluated, win):
    """The solver's float concentration grid from uint32 counts [n_times][sRho][eta][xi]: counts
    as float, land (mask != 1) set to 1e37 in every level of each evaluated time."""
    conc = np.ascontiguousarray(counts, dtype=np.float32)
    mask = np.ascontiguousarray(win.mask, dtype=np.float64)
    for t in evaluated:
        oracle_lib().wo_concentration_mask(conc.ctypes.data, int(t), win.sRho, win.eta, win.xi,
                                           _dptr(mask))
    return conc


def ref_concentration(particles, conc_time_index, n_times, win, threads=0):
    """Float counts from the reference Concentration::evaluate."""
    conc = np.zeros((n_times, win.sRho, win.eta, win.xi), dtype=np.float32)
    ref_lib().ref_concentration(particles.ctypes.data, len(particles), conc_time_index, n_times,
                                win.sRho, win.eta, win.xi, conc.ctypes.data, threads)
    return conc


def emission_times(lib_kind, mode, value, source_start, source_end, interval_start,
                   interval_end):
    """sourceEmissionTimes through the oracle ("oracle") or the reference ("ref")."""
    cap = 1 << 20
    out = np.zeros(cap, dtype=np.float64)
    if lib_kind == "oracle":
        count = oracle_lib().wo_source_emission_times(mode, value, source_start, source_end,
                                                      interval_start, interval_end,
                                                      _dptr(out), cap)
    else:
        count = ref_lib().ref_source_emission_times(mode, value, source_start, source_end,
                                                    interval_start, interval_end, _dptr(out), cap)
    if count < 0:
        return None
    return out[:min(count, cap)].copy()


def sources_emit(config, sources, julian_start, interval_start, interval_end, first_id):
    """Sources::emit restated by the oracle: the new records (PARTICLE_DTYPE) in emission order,
    or None on an invalid schedule."""
    src = np.ascontiguousarray(sources, dtype=SOURCE_DTYPE)
    lib = oracle_lib()
    count = lib.wo_sources_emit(ctypes.addressof(config), src.ctypes.data, len(src), julian_start,
                                interval_start, interval_end, first_id, None, 0)
    if count < 0:
        return None
    out = np.zeros(count, dtype=PARTICLE_DTYPE)
    lib.wo_sources_emit(ctypes.addressof(config), src.ctypes.data, len(src), julian_start,
                        interval_start, interval_end, first_id, out.ctypes.data, count)
    return out


def kji2deplatlon(grid, k, j, i):
    """(dep, lat, lon) of an index position on ``grid`` (lon/lat in degrees)."""
    dep, lat, lon = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    oracle_lib().wo_kji2deplatlon(grid.eta, grid.xi, grid.sW, _dptr(grid.lon), _dptr(grid.lat),
                                  _dptr(grid.h), _dptr(grid.sWValues), k, j, i,
                                  ctypes.byref(dep), ctypes.byref(lat), ctypes.byref(lon))
    return dep.value, lat.value, lon.value


def deplatlon2kji(grid, dep, lat, lon):
    """(k, j, i) of a geographic position, or None off the grid."""
    k, j, i = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    status = oracle_lib().wo_deplatlon2kji(grid.eta, grid.xi, grid.sW, _dptr(grid.lon),
                                           _dptr(grid.lat), _dptr(grid.h), _dptr(grid.sWValues),
                                           dep, lat, lon, ctypes.byref(k), ctypes.byref(j),
                                           ctypes.byref(i))
    if status != 0:
        return None
    return k.value, j.value, i.value


REF_REGRID_SO = os.path.join(HERE, "_ref", "libwacomm_ref_regrid.so")
REGRID_METHODS = ("geographic", "curvilinear")
_ref_regrid = None


def _regrid_argtypes(fn):
    i32, lng = ctypes.c_int, ctypes.c_long
    fn.restype = i32
    fn.argtypes = [i32, i32, _c_double_p, _c_double_p, i32, _c_float_p, lng, _c_double_p,
                   _c_double_p, _c_float_p]


def ref_regrid_available():
    return os.path.exists(REF_REGRID_SO)


def ref_regrid_lib():
    global _ref_regrid
    if _ref_regrid is None:
        if not ref_regrid_available():
            raise RuntimeError(f"reference regridder build missing: {REF_REGRID_SO}")
        lib = ctypes.CDLL(REF_REGRID_SO)
        _regrid_argtypes(lib.ref_regrid_geographic)
        _regrid_argtypes(lib.ref_regrid_curvilinear)
        _ref_regrid = lib
    return _ref_regrid


def regrid(lib_kind, method, lon, lat, src, target_lon, target_lat):
    """Bilinear regridding of src[T, eta, xi] (or [eta, xi]) from the source grid lon/lat
    [eta, xi] (degrees) to the targets; returns (code, out[T, *target.shape]). lib_kind is
    "oracle" (the restatement) or "ref" (the reference's EnvironmentalRegridder)."""
    lon = np.ascontiguousarray(lon, dtype=np.float64)
    lat = np.ascontiguousarray(lat, dtype=np.float64)
    src = np.ascontiguousarray(src, dtype=np.float32)
    squeeze = src.ndim == 2
    if squeeze:
        src = src[None]
    tshape = np.shape(target_lon)
    tlon = np.ascontiguousarray(target_lon, dtype=np.float64).ravel()
    tlat = np.ascontiguousarray(target_lat, dtype=np.float64).ravel()
    out = np.zeros((src.shape[0], tlon.size), dtype=np.float32)
    if lib_kind == "oracle":
        fn = getattr(oracle_lib(), f"wo_regrid_{method}")
        if fn.argtypes is None:
            _regrid_argtypes(fn)
    else:
        fn = getattr(ref_regrid_lib(), f"ref_regrid_{method}")
    eta, xi = lon.shape
    rc = fn(eta, xi, _dptr(lon), _dptr(lat), src.shape[0], _fptr(src), tlon.size, _dptr(tlon),
            _dptr(tlat), _fptr(out))
    out = out.reshape((src.shape[0],) + tshape)
    return rc, (out[0] if squeeze else out)


def align_times(src_times, src, dst_times):
    """wo_align_times: src[nSrc, ...] at src_times to dst_times; returns (code, out)."""
    lib = oracle_lib()
    fn = lib.wo_align_times
    if fn.argtypes is None:
        fn.restype = ctypes.c_int
        fn.argtypes = [ctypes.c_int, _c_double_p, ctypes.c_long, _c_float_p, ctypes.c_int,
                       _c_double_p, _c_float_p]
    st = np.ascontiguousarray(src_times, dtype=np.float64)
    dt = np.ascontiguousarray(dst_times, dtype=np.float64)
    src = np.ascontiguousarray(src, dtype=np.float32)
    plane = int(np.prod(src.shape[1:]))
    out = np.zeros((dt.size,) + src.shape[1:], dtype=np.float32)
    rc = fn(st.size, _dptr(st), plane, _fptr(src), dt.size, _dptr(dt), _fptr(out))
    return rc, out


def roms_normalize(mask_rho, mask_u, mask_v, angle, zeta, u, v, w, akt):
    """wo_roms_normalize on one ROMS record; returns (code, zeta, u, v, w, akt) on the rho grid.
    angle None: u/v already east/north."""
    lib = oracle_lib()
    fn = lib.wo_roms_normalize
    if fn.argtypes is None:
        fn.restype = ctypes.c_int
        fn.argtypes = [ctypes.c_int] * 3 + [_c_double_p] * 4 + [_c_float_p] * 10
    f64 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    mask_rho, mask_u, mask_v, angle = f64(mask_rho), f64(mask_u), f64(mask_v), f64(angle)
    zeta, u, v, w, akt = f32(zeta), f32(u), f32(v), f32(w), f32(akt)
    eta, xi = mask_rho.shape
    s_rho = u.shape[0]
    outs = [np.zeros((eta, xi), np.float32), np.zeros((s_rho, eta, xi), np.float32),
            np.zeros((s_rho, eta, xi), np.float32), np.zeros((s_rho + 1, eta, xi), np.float32),
            np.zeros((s_rho + 1, eta, xi), np.float32)]
    rc = fn(eta, xi, s_rho, _dptr(mask_rho), _dptr(mask_u), _dptr(mask_v), _dptr(angle),
            _fptr(zeta), _fptr(u), _fptr(v), _fptr(w), _fptr(akt), *[_fptr(o) for o in outs])
    return (rc, *outs)


def text_restart_file(path, records):
    """The oracle's text restart of ``records`` (Particles.cpp:28-55), written on one thread."""
    records = np.ascontiguousarray(records, dtype=PARTICLE_DTYPE)
    if oracle_lib().wo_text_restart(str(path).encode(), records.ctypes.data, len(records)):
        raise OSError(f"cannot write {path}")
