"""ROMS records normalized on the device (wacomm_b200_upload_roms_frame) against the oracle's
restatement of ROMSAdapter::process (itself pinned on ROMSAdapterTest.cpp's known answers).

A 96x80 grid with ~25 % land, face masks derived from the rho mask as ROMS derives them, a
varying grid angle, NaN on dry faces and fill values in zeta: every normalized field of two
records bit for bit; the earth-relative form; the rejections (NaN on a wet face, a mask other
than 0/1, a NaN angle on a wet node). A run on the device-normalized records equals the run on
the oracle-normalized records uploaded as plain records.
"""
import numpy as np
import pytest

from oracle import bindings as ob
from wacommplusplus_b200 import synthetic as syn
from wacommplusplus_b200._native import WacommError
from wacommplusplus_b200.engine import Engine
from wacommplusplus_b200.types import default_config

pytestmark = pytest.mark.gpu

ETA, XI, S_RHO = 96, 80, 6


def roms_case(seed):
    rng = np.random.default_rng(seed)
    land = syn._smooth_field(rng, ETA, XI, 6.0) > 0.7
    land[:3, :] = land[-3:, :] = False
    land[:, :3] = land[:, -3:] = False
    mask = np.where(land, 0.0, 1.0)
    mask_u = mask[:, :-1] * mask[:, 1:]
    mask_v = mask[:-1, :] * mask[1:, :]
    angle = np.pi * syn._smooth_field(rng, ETA, XI, 10.0)
    angle[land] = np.nan                     # undefined on land, as ROMS files may hold it
    records = []
    for t in range(2):
        u = rng.normal(0, 0.3, (S_RHO, ETA, XI - 1)).astype(np.float32)
        v = rng.normal(0, 0.3, (S_RHO, ETA - 1, XI)).astype(np.float32)
        u[:, mask_u == 0] = np.nan
        v[:, mask_v == 0] = np.nan
        w = rng.normal(0, 1e-4, (S_RHO + 1, ETA, XI)).astype(np.float32)
        akt = np.exp(rng.normal(-9, 1, (S_RHO + 1, ETA, XI))).astype(np.float32)
        zeta = rng.normal(0, 0.2, (ETA, XI)).astype(np.float32)
        zeta[land] = 1e37
        records.append(dict(zeta=zeta, u=u, v=v, w=w, akt=akt))
    sw = syn.vtransform2_sw(S_RHO)
    lon, lat, lon_rad, lat_rad = syn.rectilinear_grid(ETA, XI, 14.0, 14.08, 40.7, 40.796)
    h = np.where(land, 0.0, 20.0 + 30.0 * rng.random((ETA, XI)))
    grid = dict(mask=mask, mask_u=mask_u, mask_v=mask_v, angle=angle, sw=sw, lon_rad=lon_rad,
                lat_rad=lat_rad, h=h, times=syn.EPOCH_2021_07_01 + 3600.0 * np.arange(2))
    return grid, records


def engine_for(grid, angle=True):
    e = Engine(0, arithmetic="fp32", storage="fp32")
    e.set_grid(ETA, XI, S_RHO, S_RHO + 1, grid["lon_rad"], grid["lat_rad"], grid["h"],
               np.diff(grid["sw"]), grid["mask"])
    e.set_times(grid["times"])
    e.set_roms_grid(grid["mask_u"], grid["mask_v"], grid["angle"] if angle else None)
    return e


def oracle(grid, rec, angle=True):
    rc, *out = ob.roms_normalize(grid["mask"], grid["mask_u"], grid["mask_v"],
                                 grid["angle"] if angle else None, rec["zeta"], rec["u"],
                                 rec["v"], rec["w"], rec["akt"])
    assert rc == 0
    return dict(zip(("zeta", "u", "v", "w", "akt"), out))


@pytest.mark.parametrize("angle", [True, False])
def test_normalized_records_match_oracle(cuda_device, angle):
    grid, records = roms_case(3)
    e = engine_for(grid, angle)
    for t, rec in enumerate(records):
        e.upload_roms_frame(t, rec["zeta"], rec["u"], rec["v"], rec["w"], rec["akt"])
        got, want = e.get_frame(t), oracle(grid, rec, angle)
        for name in want:
            assert got[name].tobytes() == want[name].tobytes(), (t, name)
    e.close()


def test_rejections(cuda_device):
    grid, records = roms_case(4)
    e = engine_for(grid)
    rec = dict(records[0])
    bad = rec["u"].copy()
    wet = np.argwhere(grid["mask_u"] > 0)[0]
    bad[2, wet[0], wet[1]] = np.nan
    with pytest.raises(WacommError):
        e.upload_roms_frame(0, rec["zeta"], bad, rec["v"], rec["w"], rec["akt"])
    with pytest.raises(WacommError):
        e.get_frame(0)
    half = grid["mask_u"].copy()
    half[5, 5] = 0.5
    with pytest.raises(WacommError):
        e.set_roms_grid(half, grid["mask_v"], grid["angle"])
    wet_nan = grid["angle"].copy()
    wet_nan[np.argwhere(grid["mask"] > 0)[0][0], np.argwhere(grid["mask"] > 0)[0][1]] = np.nan
    with pytest.raises(WacommError):
        e.set_roms_grid(grid["mask_u"], grid["mask_v"], wet_nan)
    e.close()


def test_step_on_normalized_records(cuda_device):
    grid, records = roms_case(5)
    cfg = default_config(random=True, randomSeed=3)
    a = engine_for(grid)
    b = engine_for(grid)
    for t, rec in enumerate(records):
        a.upload_roms_frame(t, rec["zeta"], rec["u"], rec["v"], rec["w"], rec["akt"])
        o = oracle(grid, rec)
        b.upload_frame(t, o["zeta"], o["u"], o["v"], o["w"], o["akt"])
    rng = np.random.default_rng(9)
    wet = np.argwhere(grid["mask"][:-1, :-1] > 0)
    pick = wet[rng.integers(0, len(wet), 20000)]
    parts = syn.uniform_particles(20000, ETA, XI, seed=6)
    parts["j"] = pick[:, 0] + rng.random(20000)
    parts["i"] = pick[:, 1] + rng.random(20000)
    parts["k"] = -rng.random(20000) * 0.5
    for e in (a, b):
        e.set_config(cfg)
        e.set_particles(parts)
        e.move_interval(0)
    pa, pb = a.get_particles(), b.get_particles()
    for f in pa.dtype.names:
        assert pa[f].tobytes() == pb[f].tobytes(), f
    a.close()
    b.close()
