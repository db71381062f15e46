"""The C-ABI library without a GPU: it loads, exports every entry point the public headers
declare, keeps the reference record layouts, and fails cleanly when no device is visible."""
import ctypes
import os
import re
import subprocess

import pytest

from wacommplusplus_b200 import _native
from wacommplusplus_b200.types import config_data, particle_data

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_c_functions():
    names = set()
    for header in os.listdir(INCLUDE):
        if not header.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, header)).read()
        names.update(re.findall(r"^(?:int|const char \*|size_t)\s*(wacomm_b200_\w+)\(", text, re.M))
    return names


def exported_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", _native.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_exports_every_declared_entry_point():
    declared = declared_c_functions()
    assert len(declared) >= 25
    exported = exported_symbols()
    missing = declared - exported
    assert not missing, missing
    assert set(_native.SIGNATURES) == declared
    lib = _native.lib()
    for name in declared:
        assert getattr(lib, name) is not None


def test_dropin_symbol_matches_reference_mangling():
    # cuda/kernel.h:7 declares cudaMoveParticle(config_data*, particle_data*, int x6, double* x6,
    # float* x9, int x3, cudaStream_t) with C++ linkage.
    mangled = ("_Z16cudaMoveParticleP11config_dataP13particle_dataiiiiiiPdS3_S3_S3_S3_S3_"
               "PfS4_S4_S4_S4_S4_S4_S4_S4_iiiP11CUstream_st")
    assert mangled in exported_symbols()


def test_record_layouts_match_the_c_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(r'''
#include <stddef.h>
#include <stdio.h>
#include "wacomm_b200.h"
int main(void) {
    printf("%zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(wacomm_b200_config),
           sizeof(wacomm_b200_particle), offsetof(wacomm_b200_config, randomSeed),
           offsetof(wacomm_b200_config, restartCheckpoint),
           offsetof(wacomm_b200_config, observationalCalibrationRegions),
           offsetof(wacomm_b200_config, windU10), offsetof(wacomm_b200_particle, driftSide),
           sizeof(wacomm_b200_options));
    return 0;
}
''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", INCLUDE, str(src), "-o", str(exe)], check=True)
    values = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                             check=True).stdout.split()]
    assert values == [ctypes.sizeof(config_data), ctypes.sizeof(particle_data),
                      config_data.randomSeed.offset, config_data.restartCheckpoint.offset,
                      config_data.observationalCalibrationRegions.offset,
                      config_data.windU10.offset, particle_data.driftSide.offset,
                      ctypes.sizeof(_native.options_t)]
    assert values[:2] == [1248, 64]


def test_defaults_and_version():
    o = _native.default_options()
    assert (o.semantics, o.arithmetic, o.storage, o.rng) == (0, 1, 0, 0)
    assert (o.block_size, o.substeps_per_launch, o.sort_by_cell, o.fuse_concentration) == (256, 0, 1, 1)
    assert o.launch_shape == -1  # by compiled form
    assert b"sm_100a" in _native.lib().wacomm_b200_version()


def test_no_device_is_reported_not_faked():
    if _native.device_count() > 0:
        pytest.skip("a CUDA device is visible")
    handle = ctypes.c_void_p()
    assert _native.lib().wacomm_b200_context_create(0, ctypes.byref(handle)) == _native.ERR_ARGUMENT
    assert not handle.value
