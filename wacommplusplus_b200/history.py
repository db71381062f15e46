"""Particle history and restart files, mirroring the reference's Particles file methods
(Particles.cpp:28-55 saveAsTxt, 320-364 loadFromTxt, 116-273 saveAsNetCDF, 373-480
loadFromNetCDF) over the library's C ABI. Writing the resident records of a context is
``Engine.save_text`` / ``Engine.save_netcdf``; these functions read files and write host records.
Errors raise ``WacommError`` with the library's message (code ``ERR_IO``).
"""
import ctypes

import numpy as np

from . import _native
from ._native import WacommError
from .types import PARTICLE_DTYPE

RANDOM_KEY_SCHEME = "ordered-splitmix64-v2"


def _fail(status):
    if status != 0:
        raise WacommError(status, _native.lib().wacomm_b200_file_error().decode())


def save_txt(path, records):
    """Text restart of host records (Particles::saveAsTxt)."""
    records = np.ascontiguousarray(records, dtype=PARTICLE_DTYPE)
    _fail(_native.lib().wacomm_b200_text_write(str(path).encode(), records.ctypes.data,
                                                len(records)))


def load_txt(path):
    """Records of a text restart, C++ or Fortran layout (Particles::loadFromTxt)."""
    lib, n = _native.lib(), ctypes.c_size_t()
    _fail(lib.wacomm_b200_text_read(str(path).encode(), None, 0, ctypes.byref(n)))
    out = np.zeros(n.value, dtype=PARTICLE_DTYPE)
    _fail(lib.wacomm_b200_text_read(str(path).encode(), out.ctypes.data, n.value,
                                    ctypes.byref(n)))
    return out[:n.value]


def load_netcdf(path, ocean_model, backward=False, random_seed=0, leeway=False):
    """(records, checkpoint_time or None) of a NetCDF restart checked against the run
    (Particles::loadFromNetCDF)."""
    lib = _native.lib()
    expect = _native.restart_expect_t(ocean_model.encode(), int(backward), int(random_seed),
                                      int(leeway))
    n, checkpoint, has = ctypes.c_size_t(), ctypes.c_double(), ctypes.c_int()
    args = (ctypes.byref(n), ctypes.byref(checkpoint), ctypes.byref(has))
    _fail(lib.wacomm_b200_netcdf_read(str(path).encode(), ctypes.byref(expect), None, 0, *args))
    out = np.zeros(n.value, dtype=PARTICLE_DTYPE)
    _fail(lib.wacomm_b200_netcdf_read(str(path).encode(), ctypes.byref(expect), out.ctypes.data,
                                      n.value, *args))
    return out[:n.value], (checkpoint.value if has.value else None)


def history_meta(checkpoint_time, ocean_model="ROMS", git_revision="", compiler="",
                 cmake_options="", configuration_file="", configuration="", proj_version=None):
    """The wacomm_b200_history_meta of a NetCDF history (Provenance.hpp:20-27 and the run's
    attributes, Particles.cpp:156-160)."""
    enc = lambda s: None if s is None else s.encode()
    return _native.history_meta_t(enc(git_revision), enc(compiler), enc(cmake_options),
                                  enc(configuration_file), enc(configuration), enc(proj_version),
                                  enc(ocean_model), float(checkpoint_time))
