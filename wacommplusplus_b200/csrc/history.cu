// Particle history and restart files on either side of the step (Particles.cpp:28-55,116-273,
// 320-480): the text restart, and the NetCDF history/restart of schema version 3.
//
// * Text: the device hands the records over in one copy; the host formats them on all its threads
//   with std::to_chars (general, 17 significant digits: by the C++ standard the output of printf
//   "%.17g", which is what the reference's ostream with setprecision(max_digits10) prints) and
//   writes the chunks in order. The reader follows loadFromTxt's line rules, parsing chunks of
//   lines on all threads.
// * NetCDF: the device selects the records the reference stores (j >= 0, i >= 0, k <= 0 and a
//   position on the grid), compacts them with a scan and writes every variable's payload in file
//   order and byte order (big-endian), so the host only writes a header and one block. The file is
//   CDF-5 (the classic format's 64-bit-data variant, which carries the schema's uint64 and uint
//   variables); the reader takes CDF-1, CDF-2 and CDF-5.
#include <algorithm>
#include <cerrno>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"
#include "move_kernels.cuh"

namespace wb {

namespace {

thread_local std::string fileError;

int file_fail(const std::string &message) {
    fileError = message;
    return WACOMM_B200_ERR_IO;
}

int host_threads() {
    const unsigned t = std::thread::hardware_concurrency();
    return t == 0 ? 1 : (int)std::min(t, 64u);
}

// ------------------------------------------------------------------ text restart

// One record as Particles::writeTxtRecord prints it (Particles.cpp:33-39); at most 256 bytes.
char *text_record(char *p, const wacomm_b200_particle &r) {
    char *const end = p + 256;
    p = std::to_chars(p, end, r.id).ptr;
    const double reals[6] = {r.i, r.j, r.k, r.health, r.age, r.time};
    for (int f = 0; f < 6; f++) {
        *p++ = ' ';
        p = std::to_chars(p, end, reals[f], std::chars_format::general, 17).ptr;
    }
    *p++ = ' ';
    p = std::to_chars(p, end, (int)r.driftObjectType).ptr;
    *p++ = ' ';
    p = std::to_chars(p, end, (int)r.driftSide).ptr;
    *p++ = '\n';
    return p;
}

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }

// Fields of one line [b, e): up to 9 token starts; returns the token count (all of them).
int tokens_of(const char *b, const char *e, const char *start[9]) {
    int n = 0;
    while (b < e) {
        while (b < e && is_space(*b)) b++;
        if (b == e) break;
        if (n < 9) start[n] = b;
        n++;
        while (b < e && !is_space(*b)) b++;
    }
    return n;
}

// Parses record line `number` (1-based: the header is line 0) as Particles::loadFromTxt does
// (Particles.cpp:327-360). The buffer is NUL-terminated past its end, so strto* stop there.
bool text_line(const char *b, const char *e, uint64_t number, wacomm_b200_particle &r,
               std::string &error) {
    const char *t[9];
    const int n = tokens_of(b, e, t);
    r = wacomm_b200_particle{};
    if (n == 5) {  // Fortran WaComM: i j k health age
        r.id = number;
        r.i = strtod(t[0], nullptr);
        r.j = strtod(t[1], nullptr);
        r.k = strtod(t[2], nullptr);
        r.health = strtod(t[3], nullptr);
        r.age = strtod(t[4], nullptr);
        r.time = -1;
        return true;
    }
    if (n >= 7) {  // id i j k health age time [object side]
        char *after = nullptr;
        errno = 0;
        const unsigned long long id = strtoull(t[0], &after, 10);
        if (after == t[0] || errno == ERANGE) {
            error = "Invalid particle id on restart line " + std::to_string(number);
            return false;
        }
        r.id = id;
        r.i = strtod(t[1], nullptr);
        r.j = strtod(t[2], nullptr);
        r.k = strtod(t[3], nullptr);
        r.health = strtod(t[4], nullptr);
        r.age = strtod(t[5], nullptr);
        r.time = strtod(t[6], nullptr);
        if (n >= 9) {
            r.driftObjectType = (uint16_t)(int)strtol(t[7], nullptr, 10);
            r.driftSide = (int8_t)(int)strtol(t[8], nullptr, 10);
        }
        return true;
    }
    error = "Invalid particle restart record on line " + std::to_string(number);
    return false;
}

}  // namespace

int history_text_write(const char *path, const wacomm_b200_particle *records, size_t n) {
    FILE *f = fopen(path, "wb");
    if (!f) return file_fail(std::string("Unable to write the text history ") + path);
    char head[32];
    const int h = snprintf(head, sizeof(head), "\t%d\n", (int)n);
    bool ok = fwrite(head, 1, (size_t)h, f) == (size_t)h;
    // batches of records formatted on all threads, written in order
    const int threads = host_threads();
    const size_t batch = (size_t)threads << 16;
    std::vector<std::vector<char>> out(threads);
    std::vector<size_t> used(threads);
    for (size_t b0 = 0; ok && b0 < n; b0 += batch) {
        const size_t b1 = std::min(n, b0 + batch), per = (b1 - b0 + threads - 1) / threads;
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; t++) {
            const size_t s0 = std::min(b1, b0 + t * per), s1 = std::min(b1, s0 + per);
            pool.emplace_back([&, t, s0, s1] {
                out[t].resize((s1 - s0) * 256);
                char *p = out[t].data();
                for (size_t r = s0; r < s1; r++) p = text_record(p, records[r]);
                used[t] = (size_t)(p - out[t].data());
            });
        }
        for (auto &th : pool) th.join();
        for (int t = 0; t < threads && ok; t++) ok = fwrite(out[t].data(), 1, used[t], f) == used[t];
    }
    ok = (fclose(f) == 0) && ok;
    if (!ok) return file_fail(std::string("Unable to write the text history ") + path);
    return WACOMM_B200_OK;
}

int history_text_read(const char *path, std::vector<wacomm_b200_particle> &records) {
    records.clear();
    FILE *f = fopen(path, "rb");
    if (!f) return file_fail(std::string("Unable to read the text restart ") + path);
    std::vector<char> buf;
    char chunk[1 << 16];
    size_t got;
    while ((got = fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
    const bool readError = ferror(f) != 0;
    fclose(f);
    if (readError) return file_fail(std::string("Unable to read the text restart ") + path);
    const size_t size = buf.size();
    buf.push_back('\0');
    // lines as std::getline gives them: split at '\n', no empty line after a final '\n'
    const char *data = buf.data();
    const char *firstEnd = (const char *)memchr(data, '\n', size);
    if (!firstEnd) return WACOMM_B200_OK;  // the header alone (or nothing)
    const size_t bodyStart = (size_t)(firstEnd - data) + 1;
    if (bodyStart >= size) return WACOMM_B200_OK;
    // chunks of whole lines, one per thread
    const int threads = host_threads();
    std::vector<size_t> cut{bodyStart};
    for (int t = 1; t < threads; t++) {
        size_t c = bodyStart + (size - bodyStart) * t / threads;
        if (c <= cut.back()) continue;
        const char *nl = (const char *)memchr(data + c, '\n', size - c);
        c = nl ? (size_t)(nl - data) + 1 : size;
        if (c > cut.back() && c < size) cut.push_back(c);
    }
    cut.push_back(size);
    const int parts = (int)cut.size() - 1;
    std::vector<size_t> lines(parts, 0);
    for (int t = 0; t < parts; t++) {
        for (const char *p = data + cut[t], *e = data + cut[t + 1]; p < e;) {
            const char *nl = (const char *)memchr(p, '\n', (size_t)(e - p));
            lines[t]++;
            p = nl ? nl + 1 : e;
        }
    }
    std::vector<size_t> first(parts, 1);
    for (int t = 1; t < parts; t++) first[t] = first[t - 1] + lines[t - 1];
    std::vector<std::vector<wacomm_b200_particle>> out(parts);
    std::vector<std::string> errors(parts);
    std::vector<std::thread> pool;
    for (int t = 0; t < parts; t++) {
        pool.emplace_back([&, t] {
            out[t].resize(lines[t]);
            size_t line = 0;
            for (const char *p = data + cut[t], *e = data + cut[t + 1]; p < e; line++) {
                const char *nl = (const char *)memchr(p, '\n', (size_t)(e - p));
                const char *le = nl ? nl : e;
                if (!text_line(p, le, first[t] + line, out[t][line], errors[t])) return;
                p = nl ? nl + 1 : e;
            }
        });
    }
    for (auto &th : pool) th.join();
    for (int t = 0; t < parts; t++)
        if (!errors[t].empty()) return file_fail(errors[t] + " of " + path);
    size_t total = 0;
    for (int t = 0; t < parts; t++) total += out[t].size();
    records.reserve(total);
    for (int t = 0; t < parts; t++) records.insert(records.end(), out[t].begin(), out[t].end());
    return WACOMM_B200_OK;
}

// ------------------------------------------------------------------ NetCDF classic files

namespace {

// nc_type codes and sizes of the classic formats.
enum : int {
    NC_BYTE = 1, NC_CHAR = 2, NC_SHORT = 3, NC_INT = 4, NC_FLOAT = 5, NC_DOUBLE = 6,
    NC_UBYTE = 7, NC_USHORT = 8, NC_UINT = 9, NC_INT64 = 10, NC_UINT64 = 11
};
constexpr uint32_t TAG_DIMENSION = 0x0A, TAG_VARIABLE = 0x0B, TAG_ATTRIBUTE = 0x0C;

int type_size(int type) {
    switch (type) {
        case NC_BYTE: case NC_CHAR: case NC_UBYTE: return 1;
        case NC_SHORT: case NC_USHORT: return 2;
        case NC_INT: case NC_FLOAT: case NC_UINT: return 4;
        case NC_DOUBLE: case NC_INT64: case NC_UINT64: return 8;
        default: return 0;
    }
}

size_t pad4(size_t n) { return (n + 3) & ~(size_t)3; }

// CDF-5 header: big-endian, 32-bit tags and types, 64-bit counts, sizes and offsets.
struct Cdf5Header {
    std::string b;
    void u32(uint32_t v) {
        for (int s = 24; s >= 0; s -= 8) b.push_back((char)(v >> s));
    }
    void u64(uint64_t v) {
        for (int s = 56; s >= 0; s -= 8) b.push_back((char)(v >> s));
    }
    void bytes(const std::string &s) {
        b += s;
        b.append(pad4(s.size()) - s.size(), '\0');
    }
    void name(const std::string &s) {
        u64(s.size());
        bytes(s);
    }
    void text_att(const std::string &n, const std::string &v) {
        name(n);
        u32(NC_CHAR);
        u64(v.size());
        bytes(v);
    }
    void double_att(const std::string &n, double v) {
        uint64_t bits;
        memcpy(&bits, &v, 8);
        name(n);
        u32(NC_DOUBLE);
        u64(1);
        u64(bits);
    }
    void uint64_att(const std::string &n, uint64_t v) {
        name(n);
        u32(NC_UINT64);
        u64(1);
        u64(v);
    }
};

struct TextAtt {
    const char *name, *value;
};

// The particle variables after particle_time, in definition order (Particles.cpp:174-233): name,
// type, per-record bytes, attributes.
struct VarSpec {
    const char *name;
    int type;
    int bytes;
    bool twoD;  // [particles][particle_time] rather than [particles]
    std::vector<TextAtt> atts;
};

const std::vector<VarSpec> &history_vars() {
    static const std::vector<VarSpec> v = {
        {"id", NC_UINT64, 8, false, {{"long_name", "id"}, {"cf_role", "trajectory_id"}}},
        {"object_type", NC_UINT, 4, false, {{"long_name", "drift object type identifier"}}},
        {"drift_side", NC_INT, 4, false,
         {{"long_name", "crosswind orientation: -1 left, 0 undefined, 1 right"}}},
        {"lat", NC_DOUBLE, 8, true,
         {{"long_name", "latitude of particle"}, {"unit", "degree_north"},
          {"standard_name", "latitude"}}},
        {"lon", NC_DOUBLE, 8, true,
         {{"long_name", "longitude of particle"}, {"unit", "degree_east"},
          {"standard_name", "longitude"}}},
        {"depth", NC_DOUBLE, 8, true,
         {{"long_name", "particle depth below sea surface"}, {"unit", "meters"},
          {"standard_name", "depth"}, {"positive", "up"}, {"axis", "Z"}}},
        {"k", NC_DOUBLE, 8, true, {{"long_name", "depth fractional index"}}},
        {"j", NC_DOUBLE, 8, true, {{"long_name", "latitude fractional index"}}},
        {"i", NC_DOUBLE, 8, true, {{"long_name", "longitude fractional index"}}},
        {"health", NC_DOUBLE, 8, true,
         {{"long_name", "health of the particle"}, {"units", "1e-9"},
          {"coordinates", "ocean_time lon lat depth"}}},
        {"age", NC_DOUBLE, 8, true,
         {{"long_name", "age of the particle"}, {"units", "seconds since emission"},
          {"coordinates", "ocean_time lon lat depth"}}},
        {"time", NC_DOUBLE, 8, true,
         {{"long_name", "emission time of the particle"},
          {"units", "seconds since 1968-05-23 00:00:00 GMT"}, {"calendar", "gregorian"},
          {"coordinates", "ocean_time lon lat depth"}}},
    };
    return v;
}

constexpr const char *RANDOM_KEY_SCHEME = "ordered-splitmix64-v2";

// The header for `kept` records with the data starting right after it: particle_time (8 bytes),
// then each variable's block (kept records) in definition order. With no records `particles` is
// the record (unlimited) dimension with no records, as the reference's size-0 dimension is.
std::string history_header(const wacomm_b200_history_meta &m, int backward, uint64_t seed,
                           size_t kept) {
    auto str = [](const char *s) { return std::string(s ? s : ""); };
    std::string out;
    for (int pass = 0; pass < 2; pass++) {  // the second pass knows the header's size
        const uint64_t base = pass ? out.size() : 0;
        Cdf5Header h;
        h.b = "CDF";
        h.b.push_back('\x05');
        h.u64(0);  // numrecs
        h.u32(TAG_DIMENSION);
        h.u64(2);
        h.name("particles");
        h.u64(kept);
        h.name("particle_time");
        h.u64(1);
        std::vector<std::pair<std::string, std::string>> text = {
            {"wacomm_git_revision", str(m.git_revision)},
            {"wacomm_compiler", str(m.compiler)},
            {"wacomm_cmake_options", str(m.cmake_options)},
            {"wacomm_configuration_file", str(m.configuration_file)},
            {"wacomm_configuration", str(m.configuration)},
            {"wacomm_random_key_scheme", RANDOM_KEY_SCHEME}};
        if (m.proj_version) text.push_back({"wacomm_proj_version", m.proj_version});
        text.push_back({"wacomm_restart_version", "3"});
        text.push_back({"tracking_direction", backward ? "backward" : "forward"});
        text.push_back({"ocean_model", str(m.ocean_model)});
        h.u32(TAG_ATTRIBUTE);
        h.u64(text.size() + 2);
        for (auto &a : text) h.text_att(a.first, a.second);
        h.double_att("checkpoint_time", m.checkpoint_time);
        h.uint64_att("random_seed", seed);
        const auto &vars = history_vars();
        h.u32(TAG_VARIABLE);
        h.u64(1 + vars.size());
        // particle_time[particle_time]
        h.name("particle_time");
        h.u64(1);
        h.u64(1);
        h.u32(TAG_ATTRIBUTE);
        h.u64(5);
        h.text_att("long_name", "time since initialization");
        h.text_att("units", "seconds since 1968-05-23 00:00:00 GMT");
        h.text_att("calendar", "gregorian");
        h.text_att("field", "time, scalar, series");
        h.text_att("_CoordinateAxisType", "Time");
        h.u32(NC_DOUBLE);
        h.u64(8);
        h.u64(base);
        uint64_t offset = base + 8, recordOffset = base + 8;
        for (const VarSpec &v : vars) {
            h.name(v.name);
            h.u64(v.twoD ? 2 : 1);
            h.u64(0);
            if (v.twoD) h.u64(1);
            h.u32(TAG_ATTRIBUTE);
            h.u64(v.atts.size());
            for (const TextAtt &a : v.atts) h.text_att(a.name, a.value);
            h.u32((uint32_t)v.type);
            if (kept) {  // fixed size: the whole block
                h.u64(pad4((size_t)v.bytes * kept));
                h.u64(offset);
                offset += pad4((size_t)v.bytes * kept);
            } else {  // record variable: one record's slice, records interleaved after the fixed data
                h.u64((uint64_t)v.bytes);
                h.u64(recordOffset);
                recordOffset += (uint64_t)v.bytes;
            }
        }
        out = h.b;
    }
    return out;
}

// ---- reader

struct CdfAtt {
    std::string name;
    int type = 0;
    uint64_t count = 0;
    std::string data;  // raw big-endian values
};

struct CdfVar {
    std::string name;
    std::vector<uint64_t> dims;
    std::vector<CdfAtt> atts;
    int type = 0;
    uint64_t vsize = 0, begin = 0;
};

struct CdfFile {
    int version = 0;
    uint64_t numrecs = 0;
    std::vector<std::pair<std::string, uint64_t>> dims;
    std::vector<CdfAtt> atts;
    std::vector<CdfVar> vars;
    std::vector<char> bytes;

    const CdfAtt *att(const std::string &n) const {
        for (const CdfAtt &a : atts)
            if (a.name == n) return &a;
        return nullptr;
    }
    const CdfVar *var(const std::string &n) const {
        for (const CdfVar &v : vars)
            if (v.name == n) return &v;
        return nullptr;
    }
    bool record(const CdfVar &v) const { return !v.dims.empty() && dims[v.dims[0]].second == 0; }
    uint64_t recsize() const {
        uint64_t s = 0;
        for (const CdfVar &v : vars)
            if (record(v)) s += v.vsize;
        return s;
    }
};

struct Reader {
    const std::vector<char> &b;
    size_t at = 0;
    bool ok = true;
    uint64_t take(int n) {
        if (at + (size_t)n > b.size()) {
            ok = false;
            return 0;
        }
        uint64_t v = 0;
        for (int i = 0; i < n; i++) v = (v << 8) | (uint8_t)b[at + i];
        at += (size_t)n;
        return v;
    }
    std::string str(uint64_t n) {
        if (!ok || n > b.size() || at + pad4(n) > b.size()) {
            ok = false;
            return "";
        }
        std::string s(b.data() + at, b.data() + at + n);
        at += pad4(n);
        return s;
    }
};

bool read_atts(Reader &r, int nonNeg, std::vector<CdfAtt> &atts) {
    const uint32_t tag = (uint32_t)r.take(4);
    const uint64_t n = r.take(nonNeg);
    if (!r.ok || (tag != TAG_ATTRIBUTE && !(tag == 0 && n == 0)) || n > r.b.size()) return false;
    for (uint64_t a = 0; a < n && r.ok; a++) {
        CdfAtt att;
        att.name = r.str(r.take(nonNeg));
        att.type = (int)r.take(4);
        att.count = r.take(nonNeg);
        const int size = type_size(att.type);
        if (!size || att.count > r.b.size()) return false;
        att.data = r.str(att.count * (uint64_t)size);
        atts.push_back(att);
    }
    return r.ok;
}

bool parse_cdf(CdfFile &f) {
    const std::vector<char> &b = f.bytes;
    if (b.size() < 8 || b[0] != 'C' || b[1] != 'D' || b[2] != 'F') return false;
    f.version = b[3];
    if (f.version != 1 && f.version != 2 && f.version != 5) return false;
    const int nonNeg = f.version == 5 ? 8 : 4, offsetBytes = f.version == 1 ? 4 : 8;
    Reader r{b, 4};
    f.numrecs = r.take(nonNeg);
    uint32_t tag = (uint32_t)r.take(4);
    uint64_t n = r.take(nonNeg);
    if (!r.ok || (tag != TAG_DIMENSION && !(tag == 0 && n == 0)) || n > b.size()) return false;
    for (uint64_t d = 0; d < n && r.ok; d++) {
        std::string name = r.str(r.take(nonNeg));
        f.dims.push_back({name, r.take(nonNeg)});
    }
    if (!read_atts(r, nonNeg, f.atts)) return false;
    tag = (uint32_t)r.take(4);
    n = r.take(nonNeg);
    if (!r.ok || (tag != TAG_VARIABLE && !(tag == 0 && n == 0)) || n > b.size()) return false;
    for (uint64_t v = 0; v < n && r.ok; v++) {
        CdfVar var;
        var.name = r.str(r.take(nonNeg));
        const uint64_t rank = r.take(nonNeg);
        if (rank > 64) return false;
        for (uint64_t d = 0; d < rank; d++) {
            var.dims.push_back(r.take(nonNeg));
            if (var.dims.back() >= f.dims.size()) return false;
        }
        if (!read_atts(r, nonNeg, var.atts)) return false;
        var.type = (int)r.take(4);
        var.vsize = r.take(nonNeg);
        var.begin = r.take(offsetBytes);
        if (!type_size(var.type)) return false;
        f.vars.push_back(var);
    }
    return r.ok;
}

// Element e of a raw big-endian value array of `type`, converted.
template <class T>
T element(const char *p, int type) {
    uint64_t u = 0;
    const int n = type_size(type);
    for (int i = 0; i < n; i++) u = (u << 8) | (uint8_t)p[i];
    switch (type) {
        case NC_BYTE: return (T)(int8_t)u;
        case NC_UBYTE: return (T)(uint8_t)u;
        case NC_SHORT: return (T)(int16_t)u;
        case NC_USHORT: return (T)(uint16_t)u;
        case NC_INT: return (T)(int32_t)u;
        case NC_UINT: return (T)(uint32_t)u;
        case NC_INT64: return (T)(int64_t)u;
        case NC_UINT64: return (T)u;
        case NC_FLOAT: {
            uint32_t w = (uint32_t)u;
            float f;
            memcpy(&f, &w, 4);
            return (T)f;
        }
        default: {
            double d;
            memcpy(&d, &u, 8);
            return (T)d;
        }
    }
}

// The first `count` values of the first column of a variable ([particles] or [particles][...]).
template <class T>
bool first_column(const CdfFile &f, const CdfVar &v, uint64_t count, std::vector<T> &out) {
    const int size = type_size(v.type);
    if (v.type == NC_CHAR || v.dims.empty()) return false;
    uint64_t inner = 1;
    for (size_t d = 1; d < v.dims.size(); d++) inner *= f.dims[v.dims[d]].second;
    if (inner == 0) return false;
    const bool rec = f.record(v);
    const uint64_t stride = rec ? f.recsize() : inner * (uint64_t)size;
    // the whole column must lie in the file before anything is sized from the header's counts
    if (count > 0 && (stride == 0 || v.begin > f.bytes.size() ||
                      (count - 1) > (f.bytes.size() - v.begin) / stride))
        return false;
    out.resize(count);
    for (uint64_t r = 0; r < count; r++) {
        const uint64_t at = v.begin + r * stride;
        if (at + (uint64_t)size > f.bytes.size()) return false;
        out[r] = element<T>(f.bytes.data() + at, v.type);
    }
    return true;
}

std::string att_text(const CdfAtt &a) { return a.type == NC_CHAR ? a.data : std::string(); }

}  // namespace

std::string history_header_for(const wacomm_b200_history_meta &m, int backward, uint64_t seed,
                               size_t kept) {
    return history_header(m, backward, seed, kept);
}

int history_netcdf_write(const char *path, const std::string &header, double particleTime,
                         const uint8_t *payload, size_t payloadBytes) {
    FILE *f = fopen(path, "wb");
    if (!f) return file_fail(std::string("Unable to write the NetCDF history ") + path);
    uint64_t bits;
    memcpy(&bits, &particleTime, 8);
    char be[8];
    for (int i = 0; i < 8; i++) be[i] = (char)(bits >> (56 - 8 * i));
    bool ok = fwrite(header.data(), 1, header.size(), f) == header.size();
    ok = ok && fwrite(be, 1, 8, f) == 8;
    ok = ok && (payloadBytes == 0 || fwrite(payload, 1, payloadBytes, f) == payloadBytes);
    ok = (fclose(f) == 0) && ok;
    if (!ok) return file_fail(std::string("Unable to write the NetCDF history ") + path);
    return WACOMM_B200_OK;
}

// Particles::loadFromNetCDF (Particles.cpp:373-480) on a classic file.
int history_netcdf_read(const char *path, const wacomm_b200_restart_expect &expect,
                        std::vector<wacomm_b200_particle> &records, double &checkpoint,
                        bool &hasCheckpoint) {
    records.clear();
    hasCheckpoint = false;
    CdfFile f;
    {
        FILE *fp = fopen(path, "rb");
        if (!fp) return file_fail(std::string("Unable to read the restart file ") + path);
        char chunk[1 << 16];
        size_t got;
        while ((got = fread(chunk, 1, sizeof(chunk), fp)) > 0)
            f.bytes.insert(f.bytes.end(), chunk, chunk + got);
        fclose(fp);
    }
    if (!parse_cdf(f))
        return file_fail(std::string(path) +
                         " is not a NetCDF classic file (CDF-1, CDF-2 or CDF-5); convert NetCDF-4 "
                         "restarts with nccopy -k cdf5");
    if (const CdfAtt *version = f.att("wacomm_restart_version")) {
        const std::string v = att_text(*version);
        if (v != "2" && v != "3") return file_fail("Unsupported restart version: " + v);
        if (v == "2" && expect.leeway)
            return file_fail("Restart version 2 does not contain drift object state required by "
                             "drift.model=leeway");
        const CdfAtt *direction = f.att("tracking_direction");
        if (!direction) return file_fail("Restart has no tracking_direction attribute");
        const std::string restartDirection = att_text(*direction);
        const std::string configured = expect.backward ? "backward" : "forward";
        if (restartDirection != configured)
            return file_fail("Restart tracking direction is " + restartDirection +
                             " but configuration direction is " + configured);
        if (const CdfAtt *c = f.att("checkpoint_time")) {
            if (c->type == NC_CHAR || c->count < 1) return file_fail("Invalid checkpoint_time");
            checkpoint = element<double>(c->data.data(), c->type);
            hasCheckpoint = true;
        }
        if (const CdfAtt *s = f.att("random_seed")) {
            if (s->type == NC_CHAR || s->count < 1) return file_fail("Invalid random_seed");
            if (element<uint64_t>(s->data.data(), s->type) != expect.random_seed)
                return file_fail("Restart random seed does not match the configured random seed");
        }
        if (const CdfAtt *s = f.att("wacomm_random_key_scheme")) {
            const std::string scheme = att_text(*s);
            if (scheme != RANDOM_KEY_SCHEME)
                return file_fail("Restart random-key scheme is " + scheme + " but this build uses " +
                                 RANDOM_KEY_SCHEME);
        }
        if (const CdfAtt *m = f.att("ocean_model")) {
            const std::string model = att_text(*m);
            const std::string configuredModel = expect.ocean_model ? expect.ocean_model : "";
            if (model != configuredModel)
                return file_fail("Restart ocean model is " + model +
                                 " but configuration ocean model is " + configuredModel);
        }
    }
    const CdfVar *id = f.var("id");
    if (!id || id->dims.empty()) return file_fail("Restart has no id variable");
    const uint64_t count = f.record(*id) ? f.numrecs : f.dims[id->dims[0]].second;
    std::vector<uint64_t> ids;
    std::vector<double> col[6];
    const char *names[6] = {"i", "j", "k", "health", "age", "time"};
    if (!first_column(f, *id, count, ids)) return file_fail("Unreadable id variable");
    for (int c = 0; c < 6; c++) {
        const CdfVar *v = f.var(names[c]);
        if (!v) return file_fail(std::string("Restart has no ") + names[c] + " variable");
        if (!first_column(f, *v, count, col[c]))
            return file_fail(std::string("Unreadable ") + names[c] + " variable");
    }
    std::vector<uint32_t> types(count, 0);
    std::vector<int32_t> sides(count, 0);
    if (const CdfVar *v = f.var("object_type"))
        if (!first_column(f, *v, count, types)) return file_fail("Unreadable object_type variable");
    if (const CdfVar *v = f.var("drift_side"))
        if (!first_column(f, *v, count, sides)) return file_fail("Unreadable drift_side variable");
    records.resize(count);
    for (uint64_t r = 0; r < count; r++) {
        wacomm_b200_particle &p = records[r];
        p = wacomm_b200_particle{};
        p.id = ids[r];
        p.i = col[0][r];
        p.j = col[1][r];
        p.k = col[2][r];
        p.health = col[3][r];
        p.age = col[4][r];
        p.time = col[5][r];
        p.driftObjectType = (uint16_t)types[r];
        p.driftSide = (int8_t)sides[r];
    }
    return WACOMM_B200_OK;
}

// ------------------------------------------------------------------ device side of the history

namespace {

__device__ __forceinline__ uint32_t be32(uint32_t v) { return __byte_perm(v, 0, 0x0123); }

__device__ __forceinline__ uint64_t be64(uint64_t v) {
    return ((uint64_t)be32((uint32_t)v) << 32) | be32((uint32_t)(v >> 32));
}

// The records Particles::netcdfRecords keeps (Particles.cpp:121-132): j >= 0, i >= 0, k <= 0 and
// a grid position (kji2deplatlon gives 1e37 off the grid or its valid levels).
__global__ void history_select_kernel(ParticleSoA S, int n, const double *dep, const double *lat,
                                      const double *lon, uint32_t *flags) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const bool inside = !(S.j[p] < 0 || S.i[p] < 0 || S.k[p] > 0);
        const bool located = !(dep[p] == 1e37 || lat[p] == 1e37 || lon[p] == 1e37);
        flags[p] = inside && located ? 1u : 0u;
    }
}

// Every variable's value of kept record p at its position q, big-endian, in the block layout of
// history_header: id, object_type, drift_side, lat, lon, depth, k, j, i, health, age, time.
__global__ void history_pack_kernel(ParticleSoA S, int n, const uint32_t *flags,
                                    const uint32_t *positions, const double *dep,
                                    const double *lat, const double *lon, size_t kept,
                                    uint8_t *payload) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        if (!flags[p]) continue;
        const size_t q = positions[p];
        uint64_t *id = reinterpret_cast<uint64_t *>(payload);
        uint32_t *type = reinterpret_cast<uint32_t *>(payload + 8 * kept);
        uint32_t *side = reinterpret_cast<uint32_t *>(payload + 12 * kept);
        uint64_t *reals = reinterpret_cast<uint64_t *>(payload + 16 * kept);
        id[q] = be64(S.id[p]);
        type[q] = be32((uint32_t)S.type[p]);
        side[q] = be32((uint32_t)(int32_t)S.side[p]);
        const double v[9] = {lat[p], lon[p], dep[p], S.k[p], S.j[p], S.i[p], S.health[p], S.age[p],
                             S.time[p]};
#pragma unroll
        for (int f = 0; f < 9; f++) reals[f * kept + q] = be64((uint64_t)__double_as_longlong(v[f]));
    }
}

int grid_for(int n) {
    const int blocks = (n + 255) / 256;
    return blocks < 148 * 16 ? (blocks > 0 ? blocks : 1) : 148 * 16;
}

}  // namespace

size_t history_payload_bytes(size_t kept) { return 88 * kept; }

cudaError_t history_select(const ParticleSoA &S, int n, const double *dep, const double *lat,
                           const double *lon, uint32_t *flags, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    history_select_kernel<<<grid_for(n), 256, 0, stream>>>(S, n, dep, lat, lon, flags);
    return cudaGetLastError();
}

cudaError_t history_pack(const ParticleSoA &S, int n, const uint32_t *flags,
                         const uint32_t *positions, const double *dep, const double *lat,
                         const double *lon, size_t kept, uint8_t *payload, cudaStream_t stream) {
    if (n <= 0 || kept == 0) return cudaSuccess;
    history_pack_kernel<<<grid_for(n), 256, 0, stream>>>(S, n, flags, positions, dep, lat, lon,
                                                         kept, payload);
    return cudaGetLastError();
}

}  // namespace wb

// ------------------------------------------------------------------ context-free file entries

// Exceptions (allocation, thread creation) end as an error status at the C boundary.
template <class Fn>
static int guarded(Fn fn) {
    try {
        return fn();
    } catch (const std::exception &e) {
        return wb::file_fail(std::string("file call failed: ") + e.what());
    }
}

extern "C" int wacomm_b200_text_write(const char *path, const wacomm_b200_particle *records,
                                      size_t n) {
    if (!path || (n && !records)) return wb::file_fail("null path or records");
    return guarded([&] { return wb::history_text_write(path, records, n); });
}

extern "C" int wacomm_b200_text_read(const char *path, wacomm_b200_particle *records,
                                     size_t capacity, size_t *n) {
    if (!path || !n) return wb::file_fail("null path or count");
    std::vector<wacomm_b200_particle> got;
    int rc = guarded([&] { return wb::history_text_read(path, got); });
    if (rc) return rc;
    *n = got.size();
    if (!records) return WACOMM_B200_OK;
    if (capacity < got.size())
        return wb::file_fail("capacity " + std::to_string(capacity) + " for " +
                             std::to_string(got.size()) + " records");
    if (!got.empty()) memcpy(records, got.data(), got.size() * sizeof(wacomm_b200_particle));
    return WACOMM_B200_OK;
}

extern "C" int wacomm_b200_netcdf_read(const char *path, const wacomm_b200_restart_expect *expect,
                                       wacomm_b200_particle *records, size_t capacity, size_t *n,
                                       double *checkpoint_time, int *has_checkpoint) {
    if (!path || !expect || !n) return wb::file_fail("null path, expectation or count");
    std::vector<wacomm_b200_particle> got;
    double checkpoint = 0;
    bool has = false;
    int rc = guarded([&] { return wb::history_netcdf_read(path, *expect, got, checkpoint, has); });
    if (rc) return rc;
    *n = got.size();
    if (checkpoint_time) *checkpoint_time = has ? checkpoint : 0.0;
    if (has_checkpoint) *has_checkpoint = has ? 1 : 0;
    if (!records) return WACOMM_B200_OK;
    if (capacity < got.size())
        return wb::file_fail("capacity " + std::to_string(capacity) + " for " +
                             std::to_string(got.size()) + " records");
    if (!got.empty()) memcpy(records, got.data(), got.size() * sizeof(wacomm_b200_particle));
    return WACOMM_B200_OK;
}

extern "C" const char *wacomm_b200_file_error(void) { return wb::fileError.c_str(); }
