"""The oracle's environmental regridding (EnvironmentalRegridder.cpp:14-334) on the CPU.

* The known answers of the reference's tests/EnvironmentalRegridderTest.cpp (affine and constant
  fields, the cyclic and descending axes, the curved cell, the indexed 21x31 curvilinear grid, and
  the rejected inputs: a target outside, a non-rectilinear source, a folded cell), restated.
* Record-for-record against the reference's own EnvironmentalRegridder compiled from its source
  (oracle/_ref/libwacomm_ref_regrid.so): rectilinear grids with rising and falling axes and
  dateline crossings, curvilinear warped grids, targets on nodes, on shared cell edges, just
  inside and just outside the grid -- values bit for bit, and the same inputs rejected.
* The time alignment (no reference counterpart) on its own definition.
"""
import numpy as np
import pytest

from oracle import bindings as ob

GEO, CURV = "geographic", "curvilinear"


def regrid(method, lon, lat, src, tlon, tlat, lib="oracle"):
    return ob.regrid(lib, method, lon, lat, src, tlon, tlat)


def affine_case():
    lon = np.array([[10 + i for i in range(2)] for j in range(2)], float)
    lat = np.array([[40 + j for i in range(2)] for j in range(2)], float)
    affine = np.array([[[2 * lon[j, i] + 3 * lat[j, i] + 5 * t for i in range(2)]
                        for j in range(2)] for t in range(2)], np.float32)
    tlon = np.array([[10 + .5 * i for i in range(3)] for j in range(3)])
    tlat = np.array([[40 + .5 * j for i in range(3)] for j in range(3)])
    return lon, lat, affine, tlon, tlat


@pytest.mark.parametrize("method", [GEO, CURV])
def test_affine_and_constant_known_answers(method):
    # EnvironmentalRegridderTest.cpp:10-26
    lon, lat, affine, tlon, tlat = affine_case()
    rc, out = regrid(method, lon, lat, affine, tlon, tlat)
    assert rc == 0
    for t in range(2):
        assert np.abs(out[t] - (2 * tlon + 3 * tlat + 5 * t)).max() < 1e-6
    rc, kept = regrid(method, lon, lat, np.full((2, 2, 2), 7.25, np.float32), tlon, tlat)
    assert rc == 0 and np.all(kept == np.float32(7.25))


def test_rejections_known_answers():
    # EnvironmentalRegridderTest.cpp:27-37: a target outside, a non-rectilinear source
    lon, lat, affine, tlon, tlat = affine_case()
    rc, _ = regrid(GEO, lon, lat, affine, np.array([[12.0]]), np.array([[40.5]]))
    assert rc == -2
    bent = lon.copy()
    bent[1, 0] = 10.1
    rc, _ = regrid(GEO, bent, lat, affine, tlon, tlat)
    assert rc == -1


def test_cyclic_and_descending_known_answers():
    # EnvironmentalRegridderTest.cpp:39-63
    lon = np.array([[179.0, -179.0], [179.0, -179.0]])
    lat = np.array([[10.0, 10.0], [11.0, 11.0]])
    field = np.array([[[0, 2], [0, 2]]], np.float32)
    rc, out = regrid(GEO, lon, lat, field, np.array([[179.0, 180.0, -179.0]]),
                     np.array([[10.5, 10.5, 10.5]]))
    assert rc == 0 and list(out[0, 0]) == [0, 1, 2]
    dlon = np.array([[11.0 - i for i in range(2)] for j in range(2)])
    dlat = np.array([[41.0 - j for i in range(2)] for j in range(2)])
    dfield = (2 * dlon + 3 * dlat)[None].astype(np.float32)
    rc, out = regrid(GEO, dlon, dlat, dfield, np.array([[10.5]]), np.array([[40.5]]))
    assert rc == 0 and abs(out[0, 0, 0] - 142.5) < 1e-6


def test_curved_and_indexed_known_answers():
    # EnvironmentalRegridderTest.cpp:65-96
    clon = np.array([[0.0, 2.0], [.2, 2.4]])
    clat = np.array([[0.0, .1], [2.0, 2.2]])
    field = np.array([[[1, 3], [4, 6]]], np.float32)
    rc, out = regrid(CURV, clon, clat, field, np.array([[.6875]]), np.array([[1.54375]]))
    assert rc == 0 and abs(out[0, 0, 0] - 3.75) < 1e-6
    eta, xi = 21, 31
    j, i = np.mgrid[0:eta, 0:xi].astype(float)
    lon = 170 + .08 * i + .006 * j * j / eta
    lat = 30 + .07 * j + .004 * i * i / xi
    f = (2 * lon + 3 * lat)[None].astype(np.float32)
    tlon = (.63 * .38 * lon[:-1, :-1] + .37 * .38 * lon[:-1, 1:] + .63 * .62 * lon[1:, :-1] +
            .37 * .62 * lon[1:, 1:])
    tlat = (.63 * .38 * lat[:-1, :-1] + .37 * .38 * lat[:-1, 1:] + .63 * .62 * lat[1:, :-1] +
            .37 * .62 * lat[1:, 1:])
    rc, out = regrid(CURV, lon, lat, f, tlon, tlat)
    assert rc == 0 and np.abs(out[0] - (2 * tlon + 3 * tlat)).max() < 1e-4


def test_folded_cell_rejected_known_answer():
    # EnvironmentalRegridderTest.cpp:244-249
    lon = np.array([[0.0, 1.0], [1.0, 0.0]])
    lat = np.array([[0.0, 0.0], [1.0, 1.0]])
    field = np.array([[[1, 3], [4, 6]]], np.float32)
    rc, _ = regrid(CURV, lon, lat, field, np.array([[.5]]), np.array([[.5]]))
    assert rc == -4


def test_non_finite_source_rejected():
    lon, lat, affine, tlon, tlat = affine_case()
    bad = affine.copy()
    bad[1, 0, 1] = np.nan
    for method in (GEO, CURV):
        assert regrid(method, lon, lat, bad, tlon, tlat)[0] == -3


# --- randomized comparison with the reference build ----------------------------------------------

needs_ref = pytest.mark.skipif(not ob.ref_regrid_available(),
                               reason="reference regridder not built (oracle/Makefile)")


def rectilinear_grid(rng, eta, xi, dateline):
    x0 = 179.2 if dateline else rng.uniform(-30, 30)
    dx = np.cumsum(rng.uniform(.02, .2, xi))
    dx -= dx[0]
    lon1 = x0 + dx
    if dateline:
        lon1 = (lon1 + 180) % 360 - 180
    lat1 = rng.uniform(-60, 50) + np.concatenate([[0], np.cumsum(rng.uniform(.02, .2, eta - 1))])
    if rng.random() < .5:
        lon1 = lon1[::-1].copy()
    if rng.random() < .5:
        lat1 = lat1[::-1].copy()
    return np.tile(lon1, (eta, 1)), np.tile(lat1[:, None], (1, xi))


def curvilinear_grid(rng, eta, xi, dateline):
    j, i = np.mgrid[0:eta, 0:xi].astype(float)
    a, b = rng.uniform(.03, .1), rng.uniform(.03, .1)
    rot = rng.uniform(-.4, .4)
    x = (179.0 if dateline else rng.uniform(-20, 20)) + a * i * np.cos(rot) - b * j * np.sin(rot)
    y = rng.uniform(-40, 40) + a * i * np.sin(rot) + b * j * np.cos(rot)
    x = x + .15 * a * np.sin(.3 * j + .2 * i)
    y = y + .15 * b * np.cos(.25 * i - .1 * j)
    if dateline:
        x = (x + 180) % 360 - 180
    return x, y


def targets(rng, lon, lat, n):
    """Random interior points (cell parameters), every node, points on shared edges, and a few
    points just outside."""
    eta, xi = lon.shape
    ref = lon[0, 0]
    ulon = lon.copy()
    ulon = np.where(ulon - ref > 180, ulon - 360, ulon)
    ulon = np.where(ulon - ref < -180, ulon + 360, ulon)
    j = rng.integers(0, eta - 1, n)
    i = rng.integers(0, xi - 1, n)
    x, y = rng.random(n), rng.random(n)
    x[: n // 8] = 0.0                       # on a shared edge
    y[n // 8: n // 4] = 1.0
    def at(f):
        return ((1 - x) * (1 - y) * f[j, i] + x * (1 - y) * f[j, i + 1] + (1 - x) * y * f[j + 1, i]
                + x * y * f[j + 1, i + 1])
    tlon = np.concatenate([at(ulon), lon.ravel(), [ulon.min() - 1e-3, ulon.max() + .5]])
    tlat = np.concatenate([at(lat), lat.ravel(), [lat.mean(), lat.mean()]])
    tlon = (tlon + 180) % 360 - 180
    return tlon, tlat


@needs_ref
@pytest.mark.parametrize("seed", range(12))
@pytest.mark.parametrize("method", [GEO, CURV])
def test_matches_reference_build(method, seed):
    rng = np.random.default_rng(1000 * seed + (method == CURV))
    eta, xi = int(rng.integers(2, 30)), int(rng.integers(2, 30))
    dateline = seed % 3 == 0
    grid = rectilinear_grid if method == GEO or seed % 4 == 1 else curvilinear_grid
    lon, lat = grid(rng, eta, xi, dateline)
    src = rng.normal(0, 5, (3, eta, xi)).astype(np.float32)
    tlon, tlat = targets(rng, lon, lat, 400)
    inside = slice(0, tlon.size - 2)
    for sl, expect_ok in ((inside, True), (slice(None), False)):
        rc_o, out_o = regrid(method, lon, lat, src, tlon[sl], tlat[sl], "oracle")
        rc_r, out_r = regrid(method, lon, lat, src, tlon[sl], tlat[sl], "ref")
        assert (rc_o == 0) == (rc_r == 0)
        assert (rc_o == 0) == expect_ok, (rc_o, rc_r)
        if rc_o == 0:
            assert out_o.tobytes() == out_r.tobytes()


@needs_ref
def test_reference_rejections_agree():
    lon, lat, affine, tlon, tlat = affine_case()
    cases = [
        (GEO, lon, lat, affine, np.array([[12.0]]), np.array([[40.5]])),
        (GEO, np.array([[10.0, 11.0], [10.1, 11.0]]), lat, affine, tlon, tlat),
        (GEO, np.array([[10.0, 10.0], [10.0, 10.0]]), lat, affine, np.array([[10.0]]),
         np.array([[40.5]])),
        (CURV, np.array([[0.0, 1.0], [1.0, 0.0]]), np.array([[0.0, 0.0], [1.0, 1.0]]), affine,
         np.array([[.5]]), np.array([[.5]])),
        (CURV, lon, lat, affine, np.array([[np.nan]]), np.array([[40.5]])),
    ]
    for method, a, b, f, x, y in cases:
        assert regrid(method, a, b, f, x, y, "oracle")[0] != 0
        assert regrid(method, a, b, f, x, y, "ref")[0] != 0


# --- time alignment -------------------------------------------------------------------------------

def test_align_times_copies_and_blends():
    src_t = np.array([0.0, 10800.0, 21600.0])
    src = np.stack([np.full((2, 3), v, np.float32) for v in (1.0, 4.0, -2.0)])
    rc, out = ob.align_times(src_t, src, np.arange(0, 21601, 3600.0))
    assert rc == 0
    want = [1.0, 2.0, 3.0, 4.0, 2.0, 0.0, -2.0]
    assert np.allclose(out[:, 0, 0], want, atol=1e-6)
    assert out[0, 0, 0] == np.float32(1.0) and out[3, 0, 0] == np.float32(4.0)
    rc, out = ob.align_times(src_t, src, np.array([1e-7, 21600.0 + 5e-7]))
    assert rc == 0 and out[0, 0, 0] == 1.0 and out[1, 0, 0] == -2.0
    assert ob.align_times(src_t, src, np.array([-1.0]))[0] != 0
    assert ob.align_times(src_t, src, np.array([21601.0]))[0] != 0
    assert ob.align_times(np.array([0.0, 0.0]), src[:2], np.array([0.0]))[0] != 0
