"""The oracle's ROMS record normalization (ROMSAdapter.cpp:228-306, uv2rho :309-368,
wakt2wakt :431-462) against the known answers of the reference's tests/ROMSAdapterTest.cpp.

The adapter reads NetCDF, which is not installed here, so it is not built; its test's fixture
(a 2x3 rho grid with 2 s_rho levels, u = 2 and 4 on the two u faces of each row, v = 6) and
assertions are restated: the face averages 2, 3, 4 and 6, the rotation for five grid angles, the
per-node angles with a NaN angle on a dry node, and the rejection of a NaN angle on a wet node.
"""
import math

import numpy as np
import pytest

from oracle import bindings as ob


def fixture(angle=0.0, mask_rho=None):
    eta, xi, s_rho = 2, 3, 2
    mask_rho = np.ones((eta, xi)) if mask_rho is None else np.asarray(mask_rho, float)
    mask_u, mask_v = np.ones((eta, xi - 1)), np.ones((eta - 1, xi))
    u = np.zeros((s_rho, eta, xi - 1), np.float32)
    u[:, :, 0], u[:, :, 1] = 2, 4
    v = np.full((s_rho, eta - 1, xi), 6, np.float32)
    w = np.zeros((s_rho + 1, eta, xi), np.float32)
    zeta = np.zeros((eta, xi), np.float32)
    ang = np.broadcast_to(np.asarray(angle, float), (eta, xi)).copy()
    return mask_rho, mask_u, mask_v, ang, zeta, u, v, w, w.copy()


def test_face_averages_known_answer():
    # ROMSAdapterTest.cpp:71-76
    rc, _, u, v, _, _ = ob.roms_normalize(*fixture())
    assert rc == 0
    for i, want in enumerate((2, 3, 4)):
        assert np.all(np.abs(u[:, :, i] - want) < 1e-6)
    assert np.all(np.abs(v - 6) < 1e-6)


@pytest.mark.parametrize("theta", [0.0, .5 * math.pi, -.5 * math.pi, math.pi, .25 * math.pi])
def test_rotation_known_answers(theta):
    # ROMSAdapterTest.cpp:84-97
    rc, _, u, v, _, _ = ob.roms_normalize(*fixture(theta))
    assert rc == 0
    for i in range(3):
        gu, gv = 2.0 + i, 6.0
        assert np.all(np.abs(u[:, :, i] - (gu * math.cos(theta) - gv * math.sin(theta))) < 1e-6)
        assert np.all(np.abs(v[:, :, i] - (gu * math.sin(theta) + gv * math.cos(theta))) < 1e-6)
        assert np.all(np.abs(np.hypot(u[:, :, i], v[:, :, i]) - math.hypot(gu, gv)) < 1e-6)
    # earth-relative input is not rotated (ROMSAdapterTest.cpp:98-111, 159-173)
    args = list(fixture(theta))
    args[3] = None
    rc, _, ue, ve, _, _ = ob.roms_normalize(*args)
    assert rc == 0 and ue[0, 0, 1] == 3 and ve[0, 0, 1] == 6


def test_per_node_angles_and_dry_node_known_answers():
    # ROMSAdapterTest.cpp:113-124: angles {0, pi/2, -pi/2, pi, pi/4, NaN}, the NaN one dry
    angles = np.array([[0, .5 * math.pi, -.5 * math.pi], [math.pi, .25 * math.pi, np.nan]])
    mask = np.array([[1, 1, 1], [1, 1, 0]], float)
    rc, _, u, v, _, _ = ob.roms_normalize(*fixture(angles, mask))
    assert rc == 0
    assert abs(u[1, 0, 1] + 6) < 1e-6 and abs(v[1, 0, 1] - 3) < 1e-6
    assert u[1, 1, 2] == 0 and v[1, 1, 2] == 0
    # the same NaN angle on a wet node is rejected (ROMSAdapterTest.cpp:125-130)
    rc = ob.roms_normalize(*fixture(angles))[0]
    assert rc == -2


def test_masks_fill_values_and_rejections():
    m, mu, mv, ang, zeta, u, v, w, akt = fixture(0.3, [[1, 0, 1], [1, 1, 1]])
    zeta = np.array([[0.5, 0.7, 2e36], [-0.2, 0.1, 0.3]], np.float32)
    w = np.arange(w.size, dtype=np.float32).reshape(w.shape) + 1
    rc, z, uo, vo, wo, ao = ob.roms_normalize(m, mu, mv, ang, zeta, u, v, w, w * 2)
    assert rc == 0
    assert list(z[0]) == [np.float32(0.5), 0.0, 0.0] and z[1, 0] == np.float32(-0.2)
    assert np.all(wo[:, 0, 1] == 0) and np.all(wo[:, 0, 0] == w[:, 0, 0])
    assert np.all(ao[:, 0, 1] == 0) and np.all(uo[:, 0, 1] == 0) and np.all(vo[:, 0, 1] == 0)
    # a wet face without a value, a mask other than 0/1
    bad = u.copy()
    bad[1, 0, 1] = np.nan
    assert ob.roms_normalize(m, mu, mv, ang, zeta, bad, v, w, akt)[0] == -3
    mu2 = mu.copy()
    mu2[0, 0] = 0.5
    assert ob.roms_normalize(m, mu2, mv, ang, zeta, u, v, w, akt)[0] == -1
    # dry faces may hold anything
    mu3 = mu.copy()
    mu3[0, 1] = 0
    bad2 = u.copy()
    bad2[:, 0, 1] = np.nan
    rc, _, uo, _, _, _ = ob.roms_normalize(m, mu3, mv, ang, zeta, bad2, v, w, akt)
    assert rc == 0 and np.all(np.isfinite(uo))
    # a rotated velocity outside the float range
    huge = np.full_like(u, 3e38)
    assert ob.roms_normalize(m, mu, mv, ang, zeta, huge, v, w, akt)[0] == -4
