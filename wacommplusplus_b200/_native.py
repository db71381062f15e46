"""ctypes binding of libwacomm_b200.so (the C ABI of include/wacomm_b200.h).

The library is built in-tree by ``wacommplusplus_b200/csrc/Makefile`` (``__graft_entry__.build()``).
There is no fallback: when the library is missing, loading raises, and every engine call needs a
CUDA device.
"""
import ctypes
import os

from .types import config_data

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwacomm_b200.so")

OK = 0
ERR_ARGUMENT = 1
ERR_CUDA = 2
ERR_STATE = 3
ERR_DRIFT_OBJECT = 4
ERR_CAPACITY = 5
ERR_IO = 6

SEMANTICS_HOST, SEMANTICS_DEVICE = 0, 1
ARITH_REFERENCE, ARITH_FP32 = 0, 1
STORAGE_FP32, STORAGE_FP16, STORAGE_BF16 = 0, 1, 2
RNG_REFERENCE, RNG_PHILOX = 0, 1
EMISSION_UNIFORM_RATE, EMISSION_FORCING_INTERVAL_BATCH, EMISSION_SINGLE_PULSE = 0, 1, 2
FIELD_WIND, FIELD_STOKES = 0, 1
REGRID_BILINEAR_GEOGRAPHIC, REGRID_BILINEAR_CURVILINEAR_GEOGRAPHIC = 0, 1


class options_t(ctypes.Structure):
    _fields_ = [
        ("semantics", ctypes.c_int), ("arithmetic", ctypes.c_int), ("storage", ctypes.c_int),
        ("rng", ctypes.c_int), ("block_size", ctypes.c_int),
        ("substeps_per_launch", ctypes.c_int), ("sort_by_cell", ctypes.c_int),
        ("fuse_concentration", ctypes.c_int), ("launch_shape", ctypes.c_int),
        ("surrogate", ctypes.c_int), ("particles_per_thread", ctypes.c_int),
    ]


class history_meta_t(ctypes.Structure):
    """wacomm_b200_history_meta: provenance and run attributes of a NetCDF history."""
    _fields_ = [
        ("git_revision", ctypes.c_char_p), ("compiler", ctypes.c_char_p),
        ("cmake_options", ctypes.c_char_p), ("configuration_file", ctypes.c_char_p),
        ("configuration", ctypes.c_char_p), ("proj_version", ctypes.c_char_p),
        ("ocean_model", ctypes.c_char_p), ("checkpoint_time", ctypes.c_double),
    ]


class restart_expect_t(ctypes.Structure):
    """wacomm_b200_restart_expect: what a NetCDF restart must match."""
    _fields_ = [
        ("ocean_model", ctypes.c_char_p), ("backward", ctypes.c_int),
        ("random_seed", ctypes.c_uint64), ("leeway", ctypes.c_int),
    ]


# Every symbol include/wacomm_b200.h declares, with (restype, argtypes).
_vp, _i, _sz, _d = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_double
_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
SIGNATURES = {
    "wacomm_b200_version": (ctypes.c_char_p, []),
    "wacomm_b200_device_count": (_i, []),
    "wacomm_b200_context_create": (_i, [_i, ctypes.POINTER(_vp)]),
    "wacomm_b200_context_destroy": (_i, [_vp]),
    "wacomm_b200_last_error": (ctypes.c_char_p, [_vp]),
    "wacomm_b200_default_options": (_i, [ctypes.POINTER(options_t)]),
    "wacomm_b200_set_options": (_i, [_vp, ctypes.POINTER(options_t)]),
    "wacomm_b200_get_options": (_i, [_vp, ctypes.POINTER(options_t)]),
    "wacomm_b200_set_config": (_i, [_vp, ctypes.POINTER(config_data)]),
    "wacomm_b200_set_grid": (_i, [_vp, _i, _i, _i, _i, _dp, _dp, _dp, _dp, _dp]),
    "wacomm_b200_set_times": (_i, [_vp, _i, _dp]),
    "wacomm_b200_upload_frame": (_i, [_vp, _i] + [_fp] * 9),
    "wacomm_b200_upload_frame_async": (_i, [_vp, _i] + [_fp] * 9),
    "wacomm_b200_set_particles": (_i, [_vp, _vp, _sz]),
    "wacomm_b200_append_particles": (_i, [_vp, _vp, _sz]),
    "wacomm_b200_get_particles": (_i, [_vp, _vp, _sz]),
    "wacomm_b200_particle_count": (_i, [_vp, ctypes.POINTER(_sz)]),
    "wacomm_b200_move_interval": (_i, [_vp, _i]),
    "wacomm_b200_move_interval_host": (_i, [_vp, _i, _vp, _sz]),
    "wacomm_b200_remove_dead": (_i, [_vp]),
    "wacomm_b200_emit": (_i, [_vp, _vp, _i, _d, _d, _d, ctypes.POINTER(_sz)]),
    "wacomm_b200_set_geo_grid": (_i, [_vp, _dp, _dp, _dp]),
    "wacomm_b200_geo_positions": (_i, [_vp, _dp, _dp, _dp, _sz]),
    "wacomm_b200_regrid_environment": (_i, [_vp, _i, _i, _i, _i, _dp, _dp, _i, _dp, _fp, _fp]),
    "wacomm_b200_clear_environment": (_i, [_vp, _i]),
    "wacomm_b200_get_frame": (_i, [_vp, _i] + [_fp] * 5),
    "wacomm_b200_set_roms_grid": (_i, [_vp, _dp, _dp, _dp]),
    "wacomm_b200_upload_roms_frame": (_i, [_vp, _i] + [_fp] * 9),
    "wacomm_b200_particle_steps_total": (_i, [_vp, _i, _dp]),
    "wacomm_b200_graph_capture": (_i, [_vp, _i, _i]),
    "wacomm_b200_graph_launch": (_i, [_vp]),
    "wacomm_b200_graph_release": (_i, [_vp]),
    "wacomm_b200_autotune": (_i, [_vp, _i, ctypes.POINTER(_i), ctypes.POINTER(ctypes.c_float)]),
    "wacomm_b200_get_environment": (_i, [_vp, _i, _i, _fp, _fp]),
    "wacomm_b200_concentration_reset": (_i, [_vp, _i]),
    "wacomm_b200_concentration_count": (_i, [_vp, _i]),
    "wacomm_b200_concentration_get": (_i, [_vp, _vp, _sz]),
    "wacomm_b200_concentration_get_float": (_i, [_vp, _vp, _sz, _i]),
    "wacomm_b200_concentration_device": (_i, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_sz)]),
    "wacomm_b200_synchronize": (_i, [_vp]),
    "wacomm_b200_last_interval_stats": (_i, [_vp, _fp, _fp, ctypes.POINTER(_i), _dp]),
    "wacomm_b200_kernel_times": (_i, [_vp, _fp, _i, ctypes.POINTER(_i)]),
    "wacomm_b200_set_surrogate_error_limit": (_i, [_vp, ctypes.c_double]),
    "wacomm_b200_stream": (_i, [_vp, ctypes.POINTER(_vp)]),
    "wacomm_b200_set_surrogate": (_i, [_vp, _fp, _sz]),
    "wacomm_b200_last_surrogate_stats": (_i, [_vp, ctypes.POINTER(_sz), ctypes.POINTER(_sz), _fp,
                                              _fp]),
    "wacomm_b200_cuda_move_particle": (_i, [_vp, _vp, _i, _i, _i, _i, _i, _i] + [_vp] * 15 +
                                       [_i, _i, _i, _vp]),
    "wacomm_b200_cuda_move_particle_noalloc": (_i, [_vp, _vp, _i, _i, _i, _i, _i, _i] +
                                               [_vp] * 15 + [_i, _i, _i, _vp]),
    "wacomm_b200_text_write": (_i, [ctypes.c_char_p, _vp, _sz]),
    "wacomm_b200_text_read": (_i, [ctypes.c_char_p, _vp, _sz, ctypes.POINTER(_sz)]),
    "wacomm_b200_save_text": (_i, [_vp, ctypes.c_char_p]),
    "wacomm_b200_save_netcdf": (_i, [_vp, ctypes.c_char_p, ctypes.POINTER(history_meta_t),
                                     ctypes.POINTER(_sz)]),
    "wacomm_b200_netcdf_read": (_i, [ctypes.c_char_p, ctypes.POINTER(restart_expect_t), _vp, _sz,
                                     ctypes.POINTER(_sz), _dp, ctypes.POINTER(_i)]),
    "wacomm_b200_file_error": (ctypes.c_char_p, []),
    "wacomm_b200_mlp_train_work_floats": (_sz, [_i]),
    "wacomm_b200_mlp_train_step": (_i, [_vp] * 4 + [_i] + [_vp] * 6 + [_i, ctypes.c_float, _i, _vp]),
}

_lib = None


class WacommError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"wacomm_b200 error {code}: {message}")
        self.code = code


def lib():
    """The loaded library; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `make -C wacommplusplus_b200/csrc` "
                "(or __graft_entry__.build()); there is no CPU fallback")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = handle
    return _lib


def device_count():
    return lib().wacomm_b200_device_count()


def default_options():
    o = options_t()
    lib().wacomm_b200_default_options(ctypes.byref(o))
    return o
