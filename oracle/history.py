"""CPU restatement of the particle history and restart formats -- TEST INFRASTRUCTURE ONLY.

Used by tests/ as the checker of the library's writers and readers, never by the product:

* ``text_restart``: Particles::saveAsTxt (Particles.cpp:28-55): "\\t<count>" then per record
  ``id i j k health age time object side``, the reals as the reference's ostream prints them
  with setprecision(max_digits10 = 17) in the default float format, i.e. printf "%.17g";
* ``netcdf_records``: the records Particles::netcdfRecords keeps (Particles.cpp:116-148);
* ``read_cdf`` / ``write_cdf``: the NetCDF classic file format (CDF-1, CDF-2 and CDF-5, after the
  published NetCDF file-format specification), read and written independently of the library,
  to check its CDF-5 writer and to produce restart fixtures shaped like the reference's own
  test files (RestartTest.cpp:12-36).
"""
import numpy as np

from . import bindings as ob

NC_BYTE, NC_CHAR, NC_SHORT, NC_INT, NC_FLOAT, NC_DOUBLE = 1, 2, 3, 4, 5, 6
NC_UBYTE, NC_USHORT, NC_UINT, NC_INT64, NC_UINT64 = 7, 8, 9, 10, 11
_NP = {NC_BYTE: ">i1", NC_CHAR: "S1", NC_SHORT: ">i2", NC_INT: ">i4", NC_FLOAT: ">f4",
       NC_DOUBLE: ">f8", NC_UBYTE: ">u1", NC_USHORT: ">u2", NC_UINT: ">u4", NC_INT64: ">i8",
       NC_UINT64: ">u8"}
_SIZE = {t: np.dtype(d).itemsize for t, d in _NP.items()}


def _g17(x):
    return "%.17g" % x


def text_restart(records):
    """Bytes of the text restart of ``records`` (Particles.cpp:28-39)."""
    lines = ["\t%d\n" % len(records)]
    for r in records:
        lines.append("%d %s %s %s %s %s %s %d %d\n" % (
            int(r["id"]), _g17(r["i"]), _g17(r["j"]), _g17(r["k"]), _g17(r["health"]),
            _g17(r["age"]), _g17(r["time"]), int(r["driftObjectType"]), int(r["driftSide"])))
    return "".join(lines).encode()


def netcdf_records(records, grid):
    """(kept records, dep, lat, lon) of Particles::netcdfRecords (Particles.cpp:121-146): records
    inside the interpolation domain (j >= 0, i >= 0, k <= 0) with a position on the grid."""
    keep, dep, lat, lon = [], [], [], []
    for n, r in enumerate(records):
        if r["j"] < 0 or r["i"] < 0 or r["k"] > 0:
            continue
        d, la, lo = ob.kji2deplatlon(grid, float(r["k"]), float(r["j"]), float(r["i"]))
        if d == 1e37 or la == 1e37 or lo == 1e37:
            continue
        keep.append(n)
        dep.append(d)
        lat.append(la)
        lon.append(lo)
    return records[keep], np.array(dep), np.array(lat), np.array(lon)


# ------------------------------------------------------------------ classic NetCDF files

class _In:
    def __init__(self, data, version):
        self.d, self.at = data, 4
        self.nn = 8 if version == 5 else 4           # NON_NEG
        self.off = 4 if version == 1 else 8           # OFFSET

    def u(self, n):
        v = int.from_bytes(self.d[self.at:self.at + n], "big")
        self.at += n
        return v

    def padded(self, n):
        s = self.d[self.at:self.at + n]
        self.at += (n + 3) // 4 * 4
        return s

    def name(self):
        return self.padded(self.u(self.nn)).decode()

    def atts(self):
        tag, n = self.u(4), self.u(self.nn)
        assert tag in (0, 0x0C) and (tag or not n)
        out = {}
        for _ in range(n):
            name = self.name()
            t, count = self.u(4), self.u(self.nn)
            raw = self.padded(count * _SIZE[t])
            out[name] = (t, raw.decode() if t == NC_CHAR else np.frombuffer(raw, _NP[t]))
        return out


def read_cdf(path):
    """dict(version, numrecs, dims=[(name, length)], atts={name: (type, value)},
    vars={name: dict(dims, atts, type, vsize, begin, data)}); a record variable's data holds its
    numrecs records."""
    data = open(path, "rb").read()
    assert data[:3] == b"CDF" and data[3] in (1, 2, 5), data[:4]
    r = _In(data, data[3])
    numrecs = r.u(r.nn)
    tag, n = r.u(4), r.u(r.nn)
    assert tag in (0, 0x0A)
    dims = [(r.name(), r.u(r.nn)) for _ in range(n)]
    gatts = r.atts()
    tag, n = r.u(4), r.u(r.nn)
    assert tag in (0, 0x0B)
    variables, order = {}, []
    for _ in range(n):
        name = r.name()
        ids = [r.u(r.nn) for _ in range(r.u(r.nn))]
        atts = r.atts()
        t, vsize, begin = r.u(4), r.u(r.nn), r.u(r.off)
        variables[name] = dict(dims=[dims[i][0] for i in ids], dim_ids=ids, atts=atts, type=t,
                               vsize=vsize, begin=begin)
        order.append(name)
    header_end = r.at
    recsize = sum(v["vsize"] for v in variables.values()
                  if v["dim_ids"] and dims[v["dim_ids"][0]][1] == 0)
    for name in order:
        v = variables[name]
        shape = [dims[i][1] for i in v["dim_ids"]]
        item = np.dtype(_NP[v["type"]])
        if v["dim_ids"] and shape[0] == 0:  # record variable
            inner = int(np.prod(shape[1:])) if len(shape) > 1 else 1
            rows = [np.frombuffer(data, item, inner, v["begin"] + rec * recsize)
                    for rec in range(numrecs)]
            arr = np.array(rows, dtype=item).reshape([numrecs] + shape[1:])
        else:
            count = int(np.prod(shape)) if shape else 1
            arr = np.frombuffer(data, item, count, v["begin"]).reshape(shape)
        v["data"] = arr.astype(item.newbyteorder("="))
    return dict(version=data[3], numrecs=numrecs, dims=dims, atts=gatts, vars=variables,
                order=order, header_end=header_end, size=len(data))


class _Out:
    def __init__(self, version):
        self.b = bytearray()
        self.nn = 8 if version == 5 else 4
        self.off = 4 if version == 1 else 8

    def u(self, v, n):
        self.b += int(v).to_bytes(n, "big")

    def padded(self, raw):
        self.b += raw + b"\0" * ((4 - len(raw) % 4) % 4)

    def name(self, s):
        self.u(len(s), self.nn)
        self.padded(s.encode())

    def atts(self, atts):
        if not atts:
            self.u(0, 4)
            self.u(0, self.nn)
            return
        self.u(0x0C, 4)
        self.u(len(atts), self.nn)
        for name, (t, value) in atts.items():
            self.name(name)
            self.u(t, 4)
            raw = value.encode() if t == NC_CHAR else np.asarray(value, _NP[t]).tobytes()
            self.u(len(raw) // _SIZE[t], self.nn)
            self.padded(raw)


def write_cdf(path, version, dims, atts, variables):
    """A classic file with fixed-size dimensions only. ``dims``: [(name, length)]; ``atts``:
    {name: (type, value)}; ``variables``: [(name, [dim names], type, {atts}, array)]."""
    dim_index = {d: n for n, (d, _) in enumerate(dims)}

    def header(begins):
        h = _Out(version)
        h.b += b"CDF" + bytes([version])
        h.u(0, h.nn)
        h.u(0x0A, 4)
        h.u(len(dims), h.nn)
        for d, length in dims:
            h.name(d)
            h.u(length, h.nn)
        h.atts(atts)
        h.u(0x0B, 4)
        h.u(len(variables), h.nn)
        for (name, vdims, t, vatts, arr), begin in zip(variables, begins):
            h.name(name)
            h.u(len(vdims), h.nn)
            for d in vdims:
                h.u(dim_index[d], h.nn)
            h.atts(vatts)
            h.u(t, 4)
            size = np.asarray(arr, _NP[t]).nbytes
            h.u((size + 3) // 4 * 4, h.nn)
            h.u(begin, h.off)
        return bytes(h.b)

    size = len(header([0] * len(variables)))
    begins, at = [], size
    for _, _, t, _, arr in variables:
        begins.append(at)
        at += (np.asarray(arr, _NP[t]).nbytes + 3) // 4 * 4
    body = bytearray(header(begins))
    for _, _, t, _, arr in variables:
        raw = np.asarray(arr, _NP[t]).tobytes()
        body += raw + b"\0" * ((4 - len(raw) % 4) % 4)
    open(path, "wb").write(bytes(body))


def reference_test_restart(path, version=5, random_key_scheme=None, restart_version="3",
                           direction="forward", id_type=NC_UINT64, identity=9007199254740993):
    """The restart RestartTest.cpp:12-36 creates (one particle, particle_time of length 2), as a
    classic file of ``version`` (CDF-1 and CDF-2 have no unsigned 64-bit type: pass an int
    ``id_type`` and a small ``identity`` there)."""
    atts = {"wacomm_restart_version": (NC_CHAR, restart_version)}
    if random_key_scheme:
        atts["wacomm_random_key_scheme"] = (NC_CHAR, random_key_scheme)
    atts.update({"tracking_direction": (NC_CHAR, direction), "ocean_model": (NC_CHAR, "ROMS"),
                 "checkpoint_time": (NC_DOUBLE, [450.0]),
                 "random_seed": (NC_UINT64 if version == 5 else NC_INT, [5489])})
    two = ["particles", "particle_time"]
    variables = [
        ("id", ["particles"], id_type, {}, [identity]),
        ("object_type", ["particles"], NC_UINT if version == 5 else NC_INT, {}, [1]),
        ("drift_side", ["particles"], NC_INT, {}, [-1]),
        ("i", two, NC_DOUBLE, {}, [[1.25, 9]]), ("j", two, NC_DOUBLE, {}, [[2.5, 9]]),
        ("k", two, NC_DOUBLE, {}, [[-.5, 9]]), ("health", two, NC_DOUBLE, {}, [[.75, 9]]),
        ("age", two, NC_DOUBLE, {}, [[450, 9]]), ("time", two, NC_DOUBLE, {}, [[0, 9]]),
    ]
    write_cdf(path, version, [("particles", 1), ("particle_time", 2)], atts, variables)
