"""History and restart files without a GPU: the text writer and reader, and the NetCDF restart
reader, against the reference's own restart test (RestartTest.cpp) and the CPU restatement of the
formats in oracle/history.py."""
import numpy as np
import pytest

from oracle import history as oh
from wacommplusplus_b200 import history
from wacommplusplus_b200._native import ERR_IO, WacommError
from wacommplusplus_b200.types import PARTICLE_DTYPE

SEED = 5489


def _record(id_, k, j, i, health, age, time, obj=0, side=0):
    r = np.zeros(1, dtype=PARTICLE_DTYPE)
    r["id"], r["k"], r["j"], r["i"] = id_, k, j, i
    r["health"], r["age"], r["time"] = health, age, time
    r["driftObjectType"], r["driftSide"] = obj, side
    return r


def _same(a, b):
    for f in ("id", "k", "j", "i", "health", "age", "time", "driftObjectType", "driftSide"):
        assert a[f].tobytes() == b[f].tobytes(), f


def test_text_round_trip_of_the_reference_test(tmp_path):
    """RestartTest.cpp:105-123: exact 64-bit identity and full double precision."""
    r = _record(9007199254740993, -.123456789012345, 5.85472728621506, 5.32375564640966,
                .920044414487148, 7200.0000133514404, 1675900800.25, obj=1, side=1)
    path = tmp_path / "restart.txt"
    history.save_txt(path, r)
    assert path.read_bytes() == oh.text_restart(r)
    _same(history.load_txt(path), r)


def test_text_format_matches_printf_on_awkward_values(tmp_path):
    rng = np.random.default_rng(7)
    n = 5000
    r = np.zeros(n, dtype=PARTICLE_DTYPE)
    r["id"] = rng.integers(0, 2**63, n, dtype=np.uint64) * 2 + rng.integers(0, 2, n).astype(np.uint64)
    for f in ("k", "j", "i", "health", "age", "time"):
        r[f] = rng.standard_normal(n) * 10.0 ** rng.integers(-300, 300, n)
    specials = [0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, 1.7976931348623157e308, 1e16, 0.1,
                1 / 3, -1.0, 1675900800.25]
    r["i"][:len(specials)] = specials
    r["driftObjectType"] = rng.integers(0, 65536, n)
    r["driftSide"] = rng.integers(-128, 128, n)
    r["id"][0], r["id"][1] = 0, 2**64 - 1
    path = tmp_path / "awkward.txt"
    history.save_txt(path, r)
    assert path.read_bytes() == oh.text_restart(r)
    back = history.load_txt(path)
    finite = np.isfinite(r["i"])
    for f in ("id", "k", "j", "health", "age", "time", "driftObjectType", "driftSide"):
        assert back[f].tobytes() == r[f].tobytes(), f
    assert back["i"][finite].tobytes() == r["i"][finite].tobytes()
    assert np.isnan(back["i"][~finite & np.isnan(r["i"])]).all()


def test_text_reader_line_rules(tmp_path):
    """Particles.cpp:320-364: the first line is skipped; 5 fields are a Fortran record (id = line
    number, time = -1); 7 fields leave the drift object passive; 6 fields are refused."""
    path = tmp_path / "mixed.txt"
    path.write_text("anything at all\n"
                    "1.5 2.5 -0.5 0.9 3600\n"
                    "  77\t1 2 -0.25 1 0 1.5e9\r\n"
                    "78 1 2 -0.25 1 0 1.5e9 6 -1 extra\n"
                    "0.5 0.5 -0.1 1 10")
    got = history.load_txt(path)
    assert list(got["id"]) == [1, 77, 78, 4]
    assert got["i"][0] == 1.5 and got["j"][0] == 2.5 and got["k"][0] == -0.5
    assert got["health"][0] == 0.9 and got["age"][0] == 3600 and got["time"][0] == -1
    assert got["time"][1] == 1.5e9 and got["driftObjectType"][1] == 0 and got["driftSide"][1] == 0
    assert got["driftObjectType"][2] == 6 and got["driftSide"][2] == -1
    assert got["age"][3] == 10 and got["time"][3] == -1
    bad = tmp_path / "bad.txt"
    bad.write_text("\t1\n1 2 3 4 5 6\n")
    with pytest.raises(WacommError) as e:
        history.load_txt(bad)
    assert e.value.code == ERR_IO and "Invalid particle restart record" in str(e.value)
    empty_line = tmp_path / "empty_line.txt"
    empty_line.write_text("\t1\n1.5 2.5 -0.5 0.9 3600\n\n")
    with pytest.raises(WacommError):
        history.load_txt(empty_line)
    assert len(history.load_txt(_write(tmp_path / "header_only.txt", "\t0\n"))) == 0


def _write(path, text):
    path.write_text(text)
    return path


def test_text_reader_parallel_chunks_keep_line_numbers(tmp_path):
    """Fortran ids are line numbers: a file split over many reader threads keeps them."""
    n = 300000
    lines = ["\t%d\n" % n] + ["%d.5 2.5 -0.5 1 %d\n" % (q % 100, q) for q in range(n)]
    path = _write(tmp_path / "big.txt", "".join(lines))
    got = history.load_txt(path)
    assert np.array_equal(got["id"], np.arange(1, n + 1))
    assert np.array_equal(got["age"], np.arange(n, dtype=np.float64))


@pytest.mark.parametrize("version", [5, 2, 1])
def test_netcdf_restart_of_the_reference_test(tmp_path, version):
    """RestartTest.cpp:38-75 on the same restart (particle_time of length 2: the first column is
    read) as a CDF-5 file, and as CDF-2 / CDF-1 files with an int id."""
    path = tmp_path / "restart.nc"
    kw = {} if version == 5 else dict(id_type=oh.NC_INT, identity=12345)
    oh.reference_test_restart(path, version=version, **kw)
    got, checkpoint = history.load_netcdf(path, "ROMS", backward=False, random_seed=SEED)
    assert len(got) == 1 and checkpoint == 450
    assert got["id"][0] == (9007199254740993 if version == 5 else 12345)
    assert (got["i"][0], got["j"][0], got["k"][0]) == (1.25, 2.5, -.5)
    assert (got["health"][0], got["age"][0], got["time"][0]) == (.75, 450, 0)
    assert got["driftObjectType"][0] == 1 and got["driftSide"][0] == -1


@pytest.mark.parametrize("case,kwargs,expect", [
    ("backward configuration", {}, dict(backward=True)),
    ("other seed", {}, dict(random_seed=SEED + 1)),
    ("other ocean model", {}, dict(ocean_model="NEMO")),
    ("other random-key scheme", dict(random_key_scheme="xor-splitmix64-v1"), {}),
    ("unsupported version", dict(restart_version="4"), {}),
    ("version 2 under leeway", dict(restart_version="2"), dict(leeway=True)),
])
def test_netcdf_restart_refusals(tmp_path, case, kwargs, expect):
    """RestartTest.cpp:76-103 and Particles.cpp:380-429: a restart that does not match the run is
    refused."""
    path = tmp_path / "restart.nc"
    oh.reference_test_restart(path, **kwargs)
    args = dict(ocean_model="ROMS", backward=False, random_seed=SEED, leeway=False)
    args.update(expect)
    with pytest.raises(WacommError) as e:
        history.load_netcdf(path, **args)
    assert e.value.code == ERR_IO


def test_netcdf_restart_accepts_matching_scheme_and_version_2(tmp_path):
    path = tmp_path / "restart.nc"
    oh.reference_test_restart(path, random_key_scheme="ordered-splitmix64-v2")
    assert len(history.load_netcdf(path, "ROMS", random_seed=SEED)[0]) == 1
    oh.reference_test_restart(path, restart_version="2")
    assert len(history.load_netcdf(path, "ROMS", random_seed=SEED)[0]) == 1


def test_not_a_classic_file_is_refused(tmp_path):
    path = _write(tmp_path / "x.nc", "\x89HDF\r\n\x1a\n")
    with pytest.raises(WacommError) as e:
        history.load_netcdf(path, "ROMS")
    assert "nccopy" in str(e.value)


def test_restart_header_larger_than_its_file_is_refused(tmp_path):
    """A header that claims more records than the file holds is an error, not an allocation of
    the claimed size."""
    path = tmp_path / "restart.nc"
    oh.reference_test_restart(path)
    raw = bytearray(path.read_bytes())
    # CDF-5: magic, numrecs, NC_DIMENSION tag, dimension count, name length, "particles" (12 B)
    at = 4 + 8 + 4 + 8 + 8 + 12
    assert int.from_bytes(raw[at:at + 8], "big") == 1
    raw[at:at + 8] = (10 ** 12).to_bytes(8, "big")
    path.write_bytes(bytes(raw))
    with pytest.raises(WacommError) as e:
        history.load_netcdf(path, "ROMS", random_seed=SEED)
    assert e.value.code == ERR_IO
