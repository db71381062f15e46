"""Binary record types shared with the reference interface.

``config_data`` and ``particle_data`` keep the exact layouts of the reference structs
(Config.hpp:36-72, 1248 bytes; Particle.hpp:31-41, 64 bytes) because both cross the
boundary verbatim: the reference copies ``config_data`` to the device as raw bytes
(Wacomm.cpp:443,477) and moves ``particle_data`` records in and out of device memory
(Wacomm.cpp:554,591). The numpy dtype ``PARTICLE_DTYPE`` views the same 64-byte records.
"""
import ctypes

import numpy as np

MAX_OBSERVATIONAL_CALIBRATION_REGIONS = 16

# Closure and integrator codes (Config.hpp:201-207).
CLOSURE_MODE_CONSTRAINT = 1
CLOSURE_MODE_KILL = 2
CLOSURE_MODE_REFLECTION = 3
TRACKING_FORWARD = 1
TRACKING_BACKWARD = -1
INTEGRATOR_EULER = 1
INTEGRATOR_MIDPOINT = 2

# DriftObjectType / DriftSide ids (DriftModel.hpp:14-44).
PASSIVE = 0
PERSON_IN_WATER = 1
PERSON_IN_WATER_SURVIVAL_SUIT = 7
SIDE_LEFT, SIDE_UNDEFINED, SIDE_RIGHT = -1, 0, 1


class observational_calibration_region(ctypes.Structure):
    _fields_ = [
        ("west", ctypes.c_double), ("south", ctypes.c_double),
        ("east", ctypes.c_double), ("north", ctypes.c_double),
        ("windErrorStdDev", ctypes.c_double),
        ("windErrorComponentCorrelation", ctypes.c_double),
        ("windErrorSpatialScale", ctypes.c_double),
        ("windErrorTemporalScale", ctypes.c_double),
    ]


class config_data(ctypes.Structure):
    _fields_ = [
        ("random", ctypes.c_bool), ("randomSources", ctypes.c_bool),
        ("deltat", ctypes.c_double), ("dti", ctypes.c_double),
        ("survprob", ctypes.c_double), ("tau0", ctypes.c_double),
        ("sv", ctypes.c_double), ("crid", ctypes.c_double),
        ("sigma", ctypes.c_double), ("shoreLimit", ctypes.c_double),
        ("upperClosure", ctypes.c_int), ("lowerClosure", ctypes.c_int),
        ("horizontalClosure", ctypes.c_int),
        ("randomSeed", ctypes.c_uint64),
        ("trackingDirection", ctypes.c_int), ("backwardDiffusion", ctypes.c_int),
        ("integrator", ctypes.c_int),
        ("restartCheckpoint", ctypes.c_double),
        ("driftModel", ctypes.c_int),
        ("leewayCoefficientEnsemble", ctypes.c_bool),
        ("leewayResidualCorrelation", ctypes.c_double),
        ("leewayRandomSide", ctypes.c_bool),
        ("leewayRightSideProbability", ctypes.c_double),
        ("leewayJibeProbabilityHourly", ctypes.c_double),
        ("windErrorStdDev", ctypes.c_double),
        ("windErrorComponentCorrelation", ctypes.c_double),
        ("windErrorSpatialScale", ctypes.c_double),
        ("windErrorTemporalScale", ctypes.c_double),
        ("observationalCalibrationRegionCount", ctypes.c_uint32),
        ("observationalCalibrationRegions",
         observational_calibration_region * MAX_OBSERVATIONAL_CALIBRATION_REGIONS),
        ("driftObjectType", ctypes.c_uint16),
        ("driftSide", ctypes.c_int8),
        ("hasWind", ctypes.c_bool),
        ("windU10", ctypes.c_double), ("windV10", ctypes.c_double),
    ]


class particle_data(ctypes.Structure):
    _fields_ = [
        ("id", ctypes.c_uint64),
        ("k", ctypes.c_double), ("j", ctypes.c_double), ("i", ctypes.c_double),
        ("health", ctypes.c_double), ("age", ctypes.c_double), ("time", ctypes.c_double),
        ("driftObjectType", ctypes.c_uint16),
        ("driftSide", ctypes.c_int8),
    ]


assert ctypes.sizeof(config_data) == 1248
assert ctypes.sizeof(particle_data) == 64

PARTICLE_DTYPE = np.dtype({
    "names": ["id", "k", "j", "i", "health", "age", "time", "driftObjectType", "driftSide"],
    "formats": ["<u8", "<f8", "<f8", "<f8", "<f8", "<f8", "<f8", "<u2", "i1"],
    "offsets": [0, 8, 16, 24, 32, 40, 48, 56, 58],
    "itemsize": 64,
})


# Release point of wacomm_b200_emit (the fields of Source, Source.hpp:19-60): grid indices, start
# and end in days (negative: run start / open end), the emission value and schedule, and the
# source's own mode (only mode 1 emits).
SOURCE_DTYPE = np.dtype({
    "names": ["k", "j", "i", "start", "end", "emission_value", "emission_mode", "mode"],
    "formats": ["<f8", "<f8", "<f8", "<f8", "<f8", "<f8", "<i4", "<i4"],
    "offsets": [0, 8, 16, 24, 32, 40, 48, 52],
    "itemsize": 56,
})
EMISSION_MODES = {"uniform_rate": 0, "forcing_interval_batch": 1, "single_pulse": 2}


def make_sources(rows):
    """A SOURCE_DTYPE array from (k, j, i, start, end, value, schedule[, mode]) tuples, schedule
    a name of EMISSION_MODES or its number; mode defaults to 1."""
    out = np.zeros(len(rows), dtype=SOURCE_DTYPE)
    for n, row in enumerate(rows):
        k, j, i, start, end, value, schedule = row[:7]
        out[n] = (k, j, i, start, end, value,
                  EMISSION_MODES.get(schedule, schedule), row[7] if len(row) > 7 else 1)
    return out


def default_config(**overrides):
    """A ``config_data`` holding the reference defaults (Config.cpp:46-205): dti 30 s,
    deltat 3600 s, tau0 86400 s, survprob 1e-4, sv 0, crid 1, sigma 3.46, shore 0.25 m,
    random on with seed 5489, explicit midpoint, closures upper=constraint, lower=kill,
    horizontal=reflection, forward tracking, no restart checkpoint, passive objects."""
    cfg = config_data()
    cfg.random = True
    cfg.deltat = 3600.0
    cfg.dti = 30.0
    cfg.survprob = 1.0e-4
    cfg.tau0 = 86400.0
    cfg.sv = 0.0
    cfg.crid = 1.0
    cfg.sigma = 3.46
    cfg.shoreLimit = 0.25
    cfg.upperClosure = CLOSURE_MODE_CONSTRAINT
    cfg.lowerClosure = CLOSURE_MODE_KILL
    cfg.horizontalClosure = CLOSURE_MODE_REFLECTION
    cfg.randomSeed = 5489
    cfg.trackingDirection = TRACKING_FORWARD
    cfg.integrator = INTEGRATOR_MIDPOINT
    cfg.restartCheckpoint = float("nan")
    cfg.leewayRightSideProbability = 0.5
    for key, value in overrides.items():
        setattr(cfg, key, value)
    return cfg


def make_particles(n, ids=None, k=0.0, j=0.0, i=0.0, health=1.0, age=0.0, time=0.0,
                   drift_type=PASSIVE, drift_side=SIDE_UNDEFINED):
    """A numpy array of ``n`` particle records (fields broadcast from the arguments)."""
    out = np.zeros(n, dtype=PARTICLE_DTYPE)
    out["id"] = np.arange(n, dtype=np.uint64) if ids is None else ids
    out["k"], out["j"], out["i"] = k, j, i
    out["health"], out["age"], out["time"] = health, age, time
    out["driftObjectType"], out["driftSide"] = drift_type, drift_side
    return out
