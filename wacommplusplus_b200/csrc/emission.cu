// Device-side particle emission and geographic positions.
//
// Emission replaces the host loop of Sources::emit (Sources.cpp:233-249) over
// Source::emissionTimes / Source::emit (Source.cpp:16-45, SourceEmission.hpp:38-79): every
// source's release times for the interval are described on the device as an indexed sequence,
// the releases are merged in time order across sources exactly as std::stable_sort orders the
// source-major list (equal times keep source order), given ids last+1, last+2, ... in that order,
// optionally displaced by the seeded source offsets, given the configured drift object and side,
// and written straight into the resident particle arrays.
//
// Geographic positions restate OceanModelAdapter::kji2deplatlon (OceanModelAdapter.cpp:271-327)
// per record on the device.
//
// Compiled with -fmad=false: release times (start + (n + 1/2) * spacing) and the bilinear sums
// round exactly as the reference's unfused host arithmetic.
#include <cfloat>

#include "engine.h"
#include "move_kernels.cuh"

namespace wb {

namespace {

constexpr long long SOURCE_POSITION_INTERVAL = ENSEMBLE_INTERVAL + 2;  // SourceEmission.hpp:18
constexpr long long SIDE_INTERVAL = ENSEMBLE_INTERVAL + 1;             // DriftModel.hpp:111
constexpr long long MAX_RELEASES = (long long)1 << 31;  // per source and per emission
constexpr int ERR_SCHEDULE = 2, ERR_COUNT = 4;

// Release times of one source in one interval: time(n) for n in [0, count), non-decreasing in n.
struct Schedule {
    int mode;          // WACOMM_B200_EMISSION_*
    long long first;   // uniform_rate: reference index of the first release
    long long count;
    double start;      // uniform_rate: source start (seconds)
    double spacing;    // uniform_rate: 3600 / rate
    double fixed;      // batch modes: the common release time
};

__device__ __forceinline__ double uniform_time(const Schedule &s, long long index) {
    return s.start + ((double)index + 0.5) * s.spacing;  // SourceEmission.hpp:73
}

__device__ __forceinline__ double release_time(const Schedule &s, long long n) {
    if (s.mode == WACOMM_B200_EMISSION_UNIFORM_RATE) return uniform_time(s, s.first + n);
    return s.fixed;
}

// Releases of s strictly before t, or at or before t when at_or_before.
__device__ long long releases_before(const Schedule &s, double t, bool at_or_before) {
    if (s.count == 0) return 0;
    if (s.mode != WACOMM_B200_EMISSION_UNIFORM_RATE)
        return (at_or_before ? s.fixed <= t : s.fixed < t) ? s.count : 0;
    long long lo = 0, hi = s.count;  // first index not counted
    while (lo < hi) {
        long long mid = lo + (hi - lo) / 2;
        double tm = release_time(s, mid);
        if (at_or_before ? tm <= t : tm < t) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// First reference index in [lo, hi] whose time is >= bound (times non-decreasing); hi + 1 when
// none.
__device__ long long first_at_or_after(const Schedule &s, long long lo, long long hi, double bound) {
    long long a = lo, b = hi + 1;
    while (a < b) {
        long long mid = a + (b - a) / 2;
        if (uniform_time(s, mid) < bound) a = mid + 1;
        else b = mid;
    }
    return a;
}

// Source::emissionTimes + sourceEmissionTimes (Source.cpp:16-23, SourceEmission.hpp:38-79) as a
// schedule; returns 0 or an error bit (the reference throws where this returns ERR_SCHEDULE).
__device__ int make_schedule(const wacomm_b200_source &src, double julianStart,
                             double intervalStart, double intervalEnd, Schedule &s) {
    s = Schedule{src.emission_mode, 0, 0, 0.0, 0.0, 0.0};
    if (src.mode != 1) return 0;
    const double sourceStart = src.start < 0 ? julianStart * 86400.0 : src.start * 86400.0;
    const double sourceEnd = src.end < 0 ? -1 : src.end * 86400.0;
    const double value = src.emission_value;
    if (!isfinite(value) || value < 0 || !isfinite(sourceStart) || !isfinite(intervalStart) ||
        !isfinite(intervalEnd) || intervalEnd <= intervalStart)
        return ERR_SCHEDULE;
    if (value == 0) return 0;
    if (src.emission_mode == WACOMM_B200_EMISSION_SINGLE_PULSE) {
        if (floor(value) != value) return ERR_SCHEDULE;
        if (value >= (double)MAX_RELEASES) return ERR_COUNT;
        if (sourceStart >= intervalStart && sourceStart < intervalEnd) {
            s.count = (long long)value;
            s.fixed = sourceStart;
        }
        return 0;
    }
    if (src.emission_mode == WACOMM_B200_EMISSION_FORCING_INTERVAL_BATCH) {
        if (floor(value) != value) return ERR_SCHEDULE;
        if (value >= (double)MAX_RELEASES) return ERR_COUNT;
        // whole seconds decide membership of the closed window [start, end]
        const long long record = llround(intervalStart);
        if (record >= llround(sourceStart) && (sourceEnd < 0 || record <= llround(sourceEnd))) {
            s.count = (long long)value;
            s.fixed = intervalStart;
        }
        return 0;
    }
    if (src.emission_mode != WACOMM_B200_EMISSION_UNIFORM_RATE) return ERR_SCHEDULE;
    const double activeStart = intervalStart < sourceStart ? sourceStart : intervalStart;
    const double activeEnd =
        sourceEnd < 0 ? intervalEnd : (sourceEnd < intervalEnd ? sourceEnd : intervalEnd);
    if (activeEnd <= activeStart) return 0;
    const double spacing = 3600.0 / value;
    const double firstD = ceil((activeStart - sourceStart) / spacing - 0.5);
    const double lastD = (activeEnd - sourceStart) / spacing + 0.5;
    if (!(lastD < 4.0e18) || lastD - (firstD > 0 ? firstD : 0) > (double)MAX_RELEASES)
        return ERR_COUNT;
    const long long first = firstD > 0 ? (long long)firstD : 0;
    s.start = sourceStart;
    s.spacing = spacing;
    // The reference loop from `first` skips times before activeStart and stops at the first time
    // at or after activeEnd; both ends are found by bisection on its own time expression.
    const long long skipEnd = first + 64;
    const long long begin = first_at_or_after(s, first, skipEnd, activeStart);
    if (begin > skipEnd) return ERR_COUNT;
    long long hi = (long long)lastD + 64;
    if (hi < begin) hi = begin;
    const long long end = first_at_or_after(s, begin, hi, activeEnd);
    if (end > hi) return ERR_COUNT;
    s.first = begin;
    s.count = end - begin;
    return 0;
}

struct Plan {
    unsigned long long total;
    int err;
};

__global__ void schedule_kernel(const wacomm_b200_source *sources, int n, double julianStart,
                                double intervalStart, double intervalEnd, Schedule *out,
                                unsigned long long *counts, Plan *plan) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    Schedule sc;
    const int e = make_schedule(sources[s], julianStart, intervalStart, intervalEnd, sc);
    if (e) {
        atomicOr(&plan->err, e);
        sc.count = 0;
    }
    out[s] = sc;
    counts[s] = (unsigned long long)sc.count;
}

// Exclusive prefix of the per-source counts in one block of 256 threads (sources are few).
__global__ void offsets_kernel(const unsigned long long *counts, int n, unsigned long long *offsets,
                               Plan *plan) {
    __shared__ unsigned long long warpTotal[8];
    __shared__ unsigned long long carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += 256) {
        const int s = base + threadIdx.x;
        const unsigned long long c = s < n ? counts[s] : 0;
        unsigned long long x = c;  // inclusive scan within the warp
        for (int d = 1; d < 32; d <<= 1) {
            unsigned long long y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) warpTotal[warp] = x;
        __syncthreads();
        unsigned long long before = carry;
        for (int w = 0; w < warp; w++) before += warpTotal[w];
        if (s < n) offsets[s] = before + x - c;
        __syncthreads();
        if (threadIdx.x == 255) carry = before + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        offsets[n] = carry;
        plan->total = carry;
        if (carry >= (unsigned long long)MAX_RELEASES) plan->err |= ERR_COUNT;
    }
}

// One thread per release. Its merged rank is its index within its source plus the releases of
// earlier sources at or before its time and of later sources strictly before it: the position
// std::stable_sort by time gives it in the source-major list.
__global__ void emit_kernel(const wacomm_b200_source *sources, const Schedule *schedules,
                            int nSources, const unsigned long long *offsets,
                            unsigned long long total, const wacomm_b200_config *cfgp,
                            uint64_t firstId, ParticleSoA S, size_t base) {
    const wacomm_b200_config &cfg = *cfgp;
    for (unsigned long long e = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; e < total;
         e += (unsigned long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nSources - 1;  // the last source whose offset is <= e (it is non-empty)
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (offsets[mid] <= e) lo = mid;
            else hi = mid - 1;
        }
        const int src = lo;
        const long long n = (long long)(e - offsets[src]);
        const double t = release_time(schedules[src], n);
        unsigned long long rank = (unsigned long long)n;
        for (int other = 0; other < nSources; other++)
            if (other != src)
                rank += (unsigned long long)releases_before(schedules[other], t, other < src);
        const uint64_t id = firstId + rank;
        const wacomm_b200_source &so = sources[src];
        double k = so.k, j = so.j, i = so.i;
        if (cfg.randomSources) {  // Source.cpp:32-36, keyed on the new record's id
            k = so.k + 0.25 * full_normal(cfg.randomSeed, id, SOURCE_POSITION_INTERVAL, 0, 0);
            j = so.j + 0.25 * full_normal(cfg.randomSeed, id, SOURCE_POSITION_INTERVAL, 0, 1);
            i = so.i + 0.25 * full_normal(cfg.randomSeed, id, SOURCE_POSITION_INTERVAL, 0, 2);
        }
        int side = cfg.driftSide;
        if (cfg.leewayRandomSide)  // sampleDriftSide, DriftModel.hpp:147-154
            side = prefix_uniform(key_prefix(cfg.randomSeed, id, SIDE_INTERVAL, 0), 0) <
                           cfg.leewayRightSideProbability
                       ? 1
                       : -1;
        const size_t slot = base + rank;
        S.id[slot] = id;
        S.k[slot] = k;
        S.j[slot] = j;
        S.i[slot] = i;
        S.health[slot] = 1.0;  // Particle.cpp:30-44: health0 = 1, age 0
        S.age[slot] = 0.0;
        S.time[slot] = t;
        S.type[slot] = cfg.driftObjectType;
        S.side[slot] = (int8_t)side;
    }
}

// kji2deplatlon (OceanModelAdapter.cpp:271-327); 1e37 off the grid or its valid levels.
__global__ void geo_kernel(ParticleSoA S, int n, int eta, int xi, int sW, const double *lon,
                           const double *lat, const double *h, const double *sWValues, double *dep,
                           double *latOut, double *lonOut) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const double k = S.k[p], j = S.j[p], i = S.i[p];
        const double kc = ceil(k);
        const int kI = to_index<SEM_HOST>(kc), jI = to_index<SEM_HOST>(floor(j)),
                  iI = to_index<SEM_HOST>(floor(i));
        const double kF = kc - k, jF = j - jI, iF = i - iI;
        if (!valid_cell(jI, iI, eta, xi) || kI > 0 || kI <= -sW + 1) {
            dep[p] = latOut[p] = lonOut[p] = 1e37;
            continue;
        }
        const size_t c00 = (size_t)jI * xi + iI, c10 = c00 + xi, c11 = c10 + 1, c01 = c00 + 1;
        // each term is (value * weightI) * weightJ, summed left to right
        lonOut[p] = lon[c00] * (1.0 - iF) * (1.0 - jF) + lon[c10] * (1.0 - iF) * jF +
                    lon[c11] * iF * jF + lon[c01] * iF * (1.0 - jF);
        latOut[p] = lat[c00] * (1.0 - iF) * (1.0 - jF) + lat[c10] * (1.0 - iF) * jF +
                    lat[c11] * iF * jF + lat[c01] * iF * (1.0 - jF);
        const double hh = h[c00] * (1.0 - iF) * (1.0 - jF) + h[c10] * (1.0 - iF) * jF +
                          h[c11] * iF * jF + h[c01] * iF * (1.0 - jF);
        const double sUp = sWValues[kI + sW - 1], sLo = sWValues[kI - 1 + sW - 1];
        const double aDep = fabs(fabs(hh * sLo) - fabs(hh * sUp));
        dep[p] = -(hh * fabs(sUp) + fabs(kF * aDep));
    }
}

struct ScratchView {
    Plan *plan;
    Schedule *schedules;
    unsigned long long *counts, *offsets;
};

ScratchView scratch_view(void *scratch, int n) {
    ScratchView v;
    v.plan = static_cast<Plan *>(scratch);
    v.schedules = reinterpret_cast<Schedule *>(v.plan + 1);
    v.counts = reinterpret_cast<unsigned long long *>(v.schedules + n);
    v.offsets = v.counts + n;
    return v;
}

}  // namespace

size_t emission_scratch_bytes(int nSources) {
    return sizeof(Plan) + (size_t)nSources * sizeof(Schedule) +
           (size_t)(2 * nSources + 1) * sizeof(unsigned long long);
}

cudaError_t emission_plan(const wacomm_b200_source *sources, int nSources, double julianStart,
                          double intervalStart, double intervalEnd, void *scratch,
                          unsigned long long *totalHost, int *errHost, cudaStream_t stream) {
    ScratchView v = scratch_view(scratch, nSources);
    cudaError_t e = cudaMemsetAsync(v.plan, 0, sizeof(Plan), stream);
    if (e != cudaSuccess) return e;
    schedule_kernel<<<(nSources + 127) / 128, 128, 0, stream>>>(
        sources, nSources, julianStart, intervalStart, intervalEnd, v.schedules, v.counts, v.plan);
    offsets_kernel<<<1, 256, 0, stream>>>(v.counts, nSources, v.offsets, v.plan);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    Plan plan;
    if ((e = cudaMemcpyAsync(&plan, v.plan, sizeof(Plan), cudaMemcpyDeviceToHost, stream)) !=
        cudaSuccess)
        return e;
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
    *totalHost = plan.total;
    *errHost = plan.err;
    return cudaSuccess;
}

cudaError_t emission_fill(const wacomm_b200_source *sources, int nSources, const void *scratch,
                          unsigned long long total, const wacomm_b200_config *cfgDevice,
                          uint64_t firstId, const ParticleSoA &S, size_t base, cudaStream_t stream) {
    if (total == 0) return cudaSuccess;
    ScratchView v = scratch_view(const_cast<void *>(scratch), nSources);
    unsigned long long blocks = (total + 255) / 256;
    if (blocks > 148ull * 16) blocks = 148ull * 16;
    emit_kernel<<<(unsigned)blocks, 256, 0, stream>>>(sources, v.schedules, nSources, v.offsets,
                                                     total, cfgDevice, firstId, S, base);
    return cudaGetLastError();
}

cudaError_t geo_positions(const ParticleSoA &S, int n, int eta, int xi, int sW, const double *lon,
                          const double *lat, const double *h, const double *sWValues, double *dep,
                          double *latOut, double *lonOut, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    int blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    geo_kernel<<<blocks, 256, 0, stream>>>(S, n, eta, xi, sW, lon, lat, h, sWValues, dep, latOut,
                                           lonOut);
    return cudaGetLastError();
}

}  // namespace wb
