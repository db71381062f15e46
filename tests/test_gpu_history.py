"""History and restart files written from the resident records (device select, kji2deplatlon,
compaction and big-endian payload; host header and formatting), checked against the CPU
restatement of the formats (oracle/history.py) and the oracle's kji2deplatlon."""
import time

import numpy as np
import pytest

from oracle import bindings as ob
from oracle import history as oh
from wacommplusplus_b200 import history
from wacommplusplus_b200 import synthetic as syn
from wacommplusplus_b200.engine import Engine
from wacommplusplus_b200.types import PARTICLE_DTYPE, default_config

pytestmark = pytest.mark.gpu

META = dict(ocean_model="ROMS", git_revision="abc123", compiler="nvcc 12.9",
            cmake_options="-DWACOMM_USE_CUDA=ON", configuration_file="run.json",
            configuration='{"physics": {"random_seed": 5489}}')


def _setting(n, seed=3, backward=False):
    forcing = syn.RealisticForcing(eta=64, xi=48, s_rho=10, n_frames=2, seed=4)
    win = forcing.window()
    rng = np.random.default_rng(seed)
    r = np.zeros(n, dtype=PARTICLE_DTYPE)
    r["id"] = np.arange(n, dtype=np.uint64) * 7919 + 2**60
    r["k"] = rng.uniform(-win.sW + 0.5, 0.3, n)
    r["j"] = rng.uniform(-1.5, win.eta + 0.5, n)
    r["i"] = rng.uniform(-1.5, win.xi + 0.5, n)
    r["health"] = rng.uniform(-1, 1, n)
    r["age"] = rng.uniform(0, 1e6, n)
    r["time"] = rng.uniform(1.6e9, 1.7e9, n)
    r["driftObjectType"] = rng.integers(0, 23, n)
    r["driftSide"] = rng.integers(-1, 2, n)
    cfg = default_config(randomSeed=5489, trackingDirection=-1 if backward else 1)
    grid = type("G", (), dict(eta=win.eta, xi=win.xi, sW=win.sW, lon=win.lon, lat=win.lat,
                             h=win.h, sWValues=win.sWValues))
    return win, r, cfg, grid


def _engine(device, win, records, cfg):
    e = Engine(device)
    e.load_window(win)
    e.set_config(cfg)
    e.set_geo_grid(win.lon, win.lat, win.sWValues)
    e.set_particles(records)
    return e


def test_netcdf_history_matches_the_oracle(cuda_device, tmp_path):
    win, recs, cfg, grid = _setting(20000)
    path = tmp_path / "history.nc"
    with _engine(cuda_device, win, recs, cfg) as e:
        written = e.save_netcdf(path, 7200.5, **META)
    keep, dep, lat, lon = oh.netcdf_records(recs, grid)
    assert written == len(keep) and 0 < written < len(recs)
    f = oh.read_cdf(path)
    assert f["version"] == 5 and f["dims"] == [("particles", written), ("particle_time", 1)]
    atts = {k: v[1] for k, v in f["atts"].items()}
    assert list(atts)[:6] == ["wacomm_git_revision", "wacomm_compiler", "wacomm_cmake_options",
                              "wacomm_configuration_file", "wacomm_configuration",
                              "wacomm_random_key_scheme"]
    assert atts["wacomm_git_revision"] == "abc123" and atts["wacomm_configuration_file"] == "run.json"
    assert atts["wacomm_random_key_scheme"] == "ordered-splitmix64-v2"
    assert "wacomm_proj_version" not in atts
    assert (atts["wacomm_restart_version"], atts["tracking_direction"], atts["ocean_model"]) == (
        "3", "forward", "ROMS")
    assert f["atts"]["checkpoint_time"][0] == oh.NC_DOUBLE and atts["checkpoint_time"][0] == 7200.5
    assert f["atts"]["random_seed"][0] == oh.NC_UINT64 and atts["random_seed"][0] == 5489
    assert f["order"] == ["particle_time", "id", "object_type", "drift_side", "lat", "lon", "depth",
                          "k", "j", "i", "health", "age", "time"]
    v = f["vars"]
    assert v["particle_time"]["data"].tolist() == [7200.5]
    assert v["particle_time"]["atts"]["units"][1] == "seconds since 1968-05-23 00:00:00 GMT"
    assert v["id"]["type"] == oh.NC_UINT64 and v["id"]["atts"]["cf_role"][1] == "trajectory_id"
    assert v["object_type"]["type"] == oh.NC_UINT and v["drift_side"]["type"] == oh.NC_INT
    assert v["depth"]["atts"]["positive"][1] == "up" and v["depth"]["dims"] == ["particles",
                                                                                 "particle_time"]
    assert v["health"]["atts"]["coordinates"][1] == "ocean_time lon lat depth"
    assert np.array_equal(v["id"]["data"], keep["id"])
    assert np.array_equal(v["object_type"]["data"], keep["driftObjectType"])
    assert np.array_equal(v["drift_side"]["data"], keep["driftSide"])
    for name, want in (("lat", lat), ("lon", lon), ("depth", dep)):
        assert v[name]["data"][:, 0].tobytes() == want.tobytes(), name
    for name in ("k", "j", "i", "health", "age", "time"):
        assert v[name]["data"][:, 0].tobytes() == keep[name].tobytes(), name
    # the library's reader takes its own file back
    back, checkpoint = history.load_netcdf(path, "ROMS", random_seed=5489)
    assert checkpoint == 7200.5
    for name in ("id", "k", "j", "i", "health", "age", "time", "driftObjectType", "driftSide"):
        assert back[name].tobytes() == keep[name].tobytes(), name


def test_empty_history_keeps_zero_length_variables(cuda_device, tmp_path):
    """Particles.cpp:240-241: no stored record leaves the variables empty; the particles
    dimension is then the unlimited one, as the reference's size-0 dimension is."""
    win, recs, cfg, grid = _setting(100, backward=True)
    recs["k"] = 0.5  # all above the surface: none stored
    path = tmp_path / "empty.nc"
    with _engine(cuda_device, win, recs, cfg) as e:
        e.set_particles(recs)
        assert e.save_netcdf(path, 0.0, **META, proj_version="9.4.0") == 0
    f = oh.read_cdf(path)
    assert f["dims"] == [("particles", 0), ("particle_time", 1)] and f["numrecs"] == 0
    assert f["atts"]["tracking_direction"][1] == "backward"
    assert f["atts"]["wacomm_proj_version"][1] == "9.4.0"
    assert len(f["vars"]["id"]["data"]) == 0 and f["vars"]["particle_time"]["data"].tolist() == [0.0]
    got, _ = history.load_netcdf(path, "ROMS", backward=True, random_seed=5489)
    assert len(got) == 0


def test_text_restart_matches_the_oracle(cuda_device, tmp_path):
    win, recs, cfg, _ = _setting(50000)
    ours, theirs = tmp_path / "ours.txt", tmp_path / "oracle.txt"
    with _engine(cuda_device, win, recs, cfg) as e:
        e.save_text(ours)
    ob.text_restart_file(theirs, recs)
    assert ours.read_bytes() == theirs.read_bytes()
    back = history.load_txt(ours)
    for name in ("id", "k", "j", "i", "health", "age", "time", "driftObjectType", "driftSide"):
        assert back[name].tobytes() == recs[name].tobytes(), name


def test_writer_rates(cuda_device, tmp_path):
    """Records per second of the NetCDF and text writers at 4,194,304 resident records, beside the
    oracle's one-thread text loop (the reference's own loop shape) on a 262,144-record sample."""
    n = 1 << 22
    win, recs, cfg, _ = _setting(n, seed=11)
    with _engine(cuda_device, win, recs, cfg) as e:
        e.save_netcdf(tmp_path / "warm.nc", 0.0, **META)
        t0 = time.perf_counter()
        kept = e.save_netcdf(tmp_path / "h.nc", 0.0, **META)
        t_nc = time.perf_counter() - t0
        t0 = time.perf_counter()
        e.save_text(tmp_path / "h.txt")
        t_txt = time.perf_counter() - t0
    sample = recs[:1 << 18]
    t0 = time.perf_counter()
    ob.text_restart_file(tmp_path / "o.txt", sample)
    t_oracle = time.perf_counter() - t0
    print(f"\nNetCDF history: {n / t_nc:.3g} records/s ({kept} stored, "
          f"{(tmp_path / 'h.nc').stat().st_size / t_nc / 1e9:.2f} GB/s of file); text restart: "
          f"{n / t_txt:.3g} records/s; oracle one-thread text loop: "
          f"{len(sample) / t_oracle:.3g} records/s")
    assert kept > 0


def test_writers_with_no_records_and_their_errors(cuda_device, tmp_path):
    """No resident records: a header-only text restart and an empty history. A history without
    the kji2deplatlon grid, or a path that cannot be written, is an error, not a partial file."""
    from wacommplusplus_b200._native import ERR_IO, ERR_STATE, WacommError
    win, recs, cfg, _ = _setting(10)
    with Engine(cuda_device) as e:
        e.load_window(win)
        e.set_config(cfg)
        e.set_particles(recs[:0])
        with pytest.raises(WacommError) as err:
            e.save_netcdf(tmp_path / "nogeo.nc", 0.0, **META)
        assert err.value.code == ERR_STATE
        e.set_geo_grid(win.lon, win.lat, win.sWValues)
        e.save_text(tmp_path / "none.txt")
        assert (tmp_path / "none.txt").read_bytes() == b"\t0\n"
        assert len(history.load_txt(tmp_path / "none.txt")) == 0
        assert e.save_netcdf(tmp_path / "none.nc", 1.0, **META) == 0
        assert oh.read_cdf(tmp_path / "none.nc")["dims"][0] == ("particles", 0)
        e.set_particles(recs)
        for call in (lambda p: e.save_text(p), lambda p: e.save_netcdf(p, 0.0, **META)):
            with pytest.raises(WacommError) as err:
                call(tmp_path / "missing-dir" / "x")
            assert err.value.code == ERR_IO
