// The engine context behind the C ABI (include/wacomm_b200.h).
//
// It replaces the per-interval staging of Wacomm::run (Wacomm.cpp:386-610): instead of
// allocating, uploading the whole forcing window and the particles, launching and freeing on
// every interval, the context keeps the grid, every forcing record and the particle set
// resident in device memory, packs the bracketing pair once per interval, orders the work by
// forcing cell and moves all particles in one launch (or a few chunk launches), counting the
// concentration in the same kernel.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "engine.h"
#include "move_kernels.cuh"

using namespace wb;

namespace {

struct FrameSlot {
    float *zeta = nullptr, *u = nullptr, *v = nullptr, *w = nullptr, *akt = nullptr;
    float *windU = nullptr, *windV = nullptr, *stokesU = nullptr, *stokesV = nullptr;
    bool loaded = false;
    bool pending = false;           // an asynchronous upload the compute stream has not waited on
    cudaEvent_t ready = nullptr;    // recorded on the copy stream after an asynchronous upload
};

struct SoABuffers {
    ParticleSoA s{};
    size_t cap = 0;
};

constexpr size_t MAX_PARTICLES = (size_t)1 << 31;  // uint32 work indices

struct EnvField {
    float *u = nullptr, *v = nullptr;
};

}  // namespace

struct wacomm_b200_context {
    int device = 0;
    cudaStream_t stream = nullptr, h2d = nullptr, d2h = nullptr;
    std::string error;
    wacomm_b200_options opt{};
    wacomm_b200_config cfg{};
    wacomm_b200_config *dCfg = nullptr;  // device copy (drift branch of the FP32 step)
    bool hasConfig = false;

    int eta = 0, xi = 0, sRho = 0, sW = 0;
    bool hasGrid = false;
    double *dMask = nullptr, *dLon = nullptr, *dLat = nullptr, *dH = nullptr, *dDepth = nullptr;
    bool hasMask = false;
    double2 *dMetric = nullptr;
    float2 *dInvMetric = nullptr;
    float *dDepthF = nullptr;
    int metricSemantics = -1;

    std::vector<double> times;
    std::vector<FrameSlot> slots;

    void *dNodes = nullptr;
    size_t nodesBytes = 0;
    void *dCells = nullptr, *dCellSurface = nullptr;
    size_t cellsBytes = 0, cellSurfaceBytes = 0;
    bool pairCells = false;
    SurfPair *dSurf = nullptr;
    EnvPair *dEnv = nullptr;
    int pairT0 = -1, pairT1 = -1, pairStorage = -1;
    bool pairEnv = false;

    size_t n = 0;
    SoABuffers S, T;
    uint32_t *dKeys = nullptr, *dOrder = nullptr, *dFlags = nullptr, *dPositions = nullptr;
    // The last sorts' orders, the sequence the next sorts walk: for consecutive entries b, e of
    // seqBounds, dSeq[b, e) is a permutation of [0, e - b) (the work order of the records b..e-1).
    // Empty: nothing valid. {0, n}: the resident population sorted as one; the slab bounds of
    // move_interval_host: one permutation per slab. Any permutation gives the same sort; walking
    // the previous one keeps the histogram atomics from piling up where particles gather.
    uint32_t *dSeq = nullptr;
    std::vector<size_t> seqBounds;
    // Intervals since the resident population was last sorted by cell, for a sort cadence
    // (options.sort_by_cell = N > 1: sort every N-th interval, the others take the last order).
    // Large after the records were replaced, appended or compacted: the next interval sorts.
    int sortedAgo = 1 << 30;
    bool mayReuseOrder = false;  // set around the resident whole-population interval only
    size_t workCap = 0;
    uint32_t *dHist = nullptr, *dOffsets = nullptr;
    size_t binsCap = 0;
    uint32_t *dScanTemp = nullptr;
    size_t scanTempCap = 0;
    // The second compute lane of the host-buffer path: its stream and sort scratch, swapped in for
    // the slabs it runs (LaneSwap).
    cudaStream_t stream2 = nullptr;
    uint32_t *dHist2 = nullptr, *dOffsets2 = nullptr, *dScanTemp2 = nullptr;
    size_t binsCap2 = 0, scanTempCap2 = 0;
    cudaEvent_t evLaneStart = nullptr, evLaneDone = nullptr;
    uint32_t *dCount = nullptr;  // scratch word (compaction result)

    wacomm_b200_particle *dAos = nullptr;
    size_t aosCap = 0;

    uint32_t *dConc = nullptr;
    int concTimes = 0;
    // Concentration times counted since the last reset: the float grid masks land in these only,
    // as the solver masks each time it evaluates (Wacomm.cpp:722-737).
    std::vector<uint8_t> concEvaluated;

    wacomm_b200_source *dSources = nullptr;  // emission: the sources of the last call
    size_t sourcesCap = 0;
    unsigned char *dEmitScratch = nullptr;
    size_t emitScratchCap = 0;

    // learned surrogate (surrogate.cu)
    uint8_t *dSurrogate = nullptr;  // packed weights
    bool hasSurrogate = false;
    __half *dZ = nullptr;           // per-cell-level layer-1 sums [cell-levels][256]
    void *dCorners = nullptr;       // per-cell-level corner records (forcing, metric, gate)
    size_t zCap = 0;                // cell-levels held
    int zT0 = -1, zT1 = -1;         // forcing pair z was computed for
    int zSemantics = -1;            // metric rules of the corner records
    int *dDry = nullptr;            // dry-node prefix sums
    size_t dryCap = 0;
    double dryShore = NAN;
    bool dryValid = false;
    uint32_t *dFallback = nullptr;  // fallback list
    size_t fallbackCap = 0;
    float4 *dSurrRows = nullptr;  // surrogate layer-4 sums and row tags per work item
    size_t surrRowsCap = 0;
    unsigned long long *dSurrCounts = nullptr;  // [0]: fallback count (low 32 bits), [1]: run count
    cudaEvent_t evCell0 = nullptr, evCell1 = nullptr, evStep0 = nullptr, evStep1 = nullptr;
    bool surrTimed = false;  // the events of the last eager surrogate interval can be read
    bool surrRan = false;    // dSurrCounts holds the counts of a surrogate interval (eager or captured)
    float surrMaxError = INFINITY;  // wacomm_b200_set_surrogate_error_limit
    int smCount = 148;

    double *dGeoLon = nullptr, *dGeoLat = nullptr, *dSWValues = nullptr;  // kji2deplatlon grid
    bool hasGeo = false;
    double *dGeoOut = nullptr;  // [3][n] depth, lat, lon
    // A captured run of intervals (wacomm_b200_graph_capture) and the buffer layout it was
    // captured against.
    cudaGraphExec_t graphExec = nullptr;
    std::vector<uint64_t> graphLayout;
    int graphLaunches = 0;
    std::vector<size_t> graphSeqBounds;  // the sort sequence a launch of the graph leaves behind
    bool capturing = false;
    // ROMS grid (wacomm_b200_set_roms_grid): rho/u/v masks as bytes in one allocation, the
    // angle's (cos, sin) per rho node (null: earth-relative), and staging for raw records.
    uint8_t *dRomsMask = nullptr;
    double2 *dRomsRot = nullptr;
    bool hasRoms = false;
    float *dRomsRaw = nullptr;
    size_t romsRawCap = 0;
    // Wind (0) and Stokes (1) fields regridded to the rho nodes and the forcing times, [T][eta][xi]
    // each; a frame's own uploaded fields take precedence over these.
    EnvField env[2];
    size_t geoOutCap = 0;

    unsigned long long *dSteps = nullptr;  // [0]: the last interval or run, [1]: running total
    int *dErr = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evMove0 = nullptr, evMove1 = nullptr;
    cudaEvent_t evComputeMark = nullptr;  // orders asynchronous frame copies after enqueued kernels
    // Kernel times of eager intervals (wacomm_b200_kernel_times): a ring of event marks around
    // each interval's dominant kernels, so that intervals enqueued back to back are timed without
    // a host wait. Plain step: [move start, move end]; surrogate: [step kernel start, step kernel
    // end, walk or post kernel end, fallback step end].
    struct TimedInterval {
        cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
        int marks = 0;
    };
    std::vector<TimedInterval> timing;
    size_t timingNext = 0, timingCount = 0;
    TimedInterval *timingCur = nullptr;
    bool moveTimed = false;
    float lastMs = 0;
    int lastLaunches = 0;
    double lastSteps = 0;
};

namespace {

int fail(wacomm_b200_context *ctx, int code, const char *fmt, ...) {
    char buffer[512];
    va_list args;
    va_start(args, fmt);
    vsnprintf(buffer, sizeof(buffer), fmt, args);
    va_end(args);
    if (ctx) ctx->error = buffer;
    return code;
}

#define CUDA_TRY(ctx, expr)                                                                  \
    do {                                                                                     \
        cudaError_t _e = (expr);                                                             \
        if (_e != cudaSuccess)                                                               \
            return fail(ctx, WACOMM_B200_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(_e)); \
    } while (0)

template <class T>
int grow(wacomm_b200_context *ctx, T *&ptr, size_t &cap, size_t need) {
    if (need <= cap && ptr) return WACOMM_B200_OK;
    size_t bytes = std::max<size_t>(need, 1) * sizeof(T);
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    CUDA_TRY(ctx, cudaMalloc((void **)&ptr, bytes));
    cap = std::max<size_t>(need, 1);
    return WACOMM_B200_OK;
}

constexpr size_t TIMING_RING = 256;

// Opens the timing record of an eager interval (none while capturing).
int timing_begin(wacomm_b200_context *ctx) {
    ctx->timingCur = nullptr;
    if (ctx->capturing) return WACOMM_B200_OK;
    if (ctx->timing.empty()) ctx->timing.resize(TIMING_RING);
    wacomm_b200_context::TimedInterval &t = ctx->timing[ctx->timingNext];
    for (cudaEvent_t &e : t.ev)
        if (!e) CUDA_TRY(ctx, cudaEventCreate(&e));
    t.marks = 0;
    ctx->timingCur = &t;
    ctx->timingNext = (ctx->timingNext + 1) % TIMING_RING;
    ctx->timingCount = std::min(ctx->timingCount + 1, TIMING_RING);
    return WACOMM_B200_OK;
}

// Next mark of the open timing record, on the compute stream.
int timing_mark(wacomm_b200_context *ctx) {
    wacomm_b200_context::TimedInterval *t = ctx->timingCur;
    if (!t || t->marks >= 4) return WACOMM_B200_OK;
    CUDA_TRY(ctx, cudaEventRecord(t->ev[t->marks], ctx->stream));
    t->marks++;
    return WACOMM_B200_OK;
}

void free_soa(SoABuffers &b) {
    cudaFree(b.s.id);
    cudaFree(b.s.k);
    cudaFree(b.s.j);
    cudaFree(b.s.i);
    cudaFree(b.s.health);
    cudaFree(b.s.age);
    cudaFree(b.s.time);
    cudaFree(b.s.type);
    cudaFree(b.s.side);
    cudaFree(b.s.elapsed);
    b = SoABuffers{};
}

int alloc_soa(wacomm_b200_context *ctx, SoABuffers &b, size_t cap) {
    free_soa(b);
    size_t c = std::max<size_t>(cap, 1);
    CUDA_TRY(ctx, cudaMalloc(&b.s.id, c * sizeof(uint64_t)));
    CUDA_TRY(ctx, cudaMalloc(&b.s.k, c * sizeof(double)));
    CUDA_TRY(ctx, cudaMalloc(&b.s.j, c * sizeof(double)));
    CUDA_TRY(ctx, cudaMalloc(&b.s.i, c * sizeof(double)));
    CUDA_TRY(ctx, cudaMalloc(&b.s.health, c * sizeof(double)));
    CUDA_TRY(ctx, cudaMalloc(&b.s.age, c * sizeof(double)));
    CUDA_TRY(ctx, cudaMalloc(&b.s.time, c * sizeof(double)));
    CUDA_TRY(ctx, cudaMalloc(&b.s.type, c * sizeof(uint16_t)));
    CUDA_TRY(ctx, cudaMalloc(&b.s.side, c * sizeof(int8_t)));
    CUDA_TRY(ctx, cudaMalloc(&b.s.elapsed, c * sizeof(double)));
    b.cap = c;
    return WACOMM_B200_OK;
}

ParticleSoA offset_soa(const ParticleSoA &s, size_t off) {
    ParticleSoA r = s;
    r.id += off;
    r.k += off;
    r.j += off;
    r.i += off;
    r.health += off;
    r.age += off;
    r.time += off;
    r.type += off;
    r.side += off;
    r.elapsed += off;
    return r;
}

// Grows the resident particle arrays to hold `need` records, keeping the first `keep`.
int reserve_particles(wacomm_b200_context *ctx, size_t need, size_t keep) {
    if (need <= ctx->S.cap && ctx->S.s.id) return WACOMM_B200_OK;
    size_t cap = std::max(need, ctx->S.cap + ctx->S.cap / 2);
    SoABuffers fresh;
    int rc = alloc_soa(ctx, fresh, cap);
    if (rc) return rc;
    if (keep) {
        const ParticleSoA &a = ctx->S.s, &b = fresh.s;
        CUDA_TRY(ctx, cudaMemcpyAsync(b.id, a.id, keep * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        CUDA_TRY(ctx, cudaMemcpyAsync(b.k, a.k, keep * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        CUDA_TRY(ctx, cudaMemcpyAsync(b.j, a.j, keep * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        CUDA_TRY(ctx, cudaMemcpyAsync(b.i, a.i, keep * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        CUDA_TRY(ctx, cudaMemcpyAsync(b.health, a.health, keep * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        CUDA_TRY(ctx, cudaMemcpyAsync(b.age, a.age, keep * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        CUDA_TRY(ctx, cudaMemcpyAsync(b.time, a.time, keep * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        CUDA_TRY(ctx, cudaMemcpyAsync(b.type, a.type, keep * 2, cudaMemcpyDeviceToDevice, ctx->stream));
        CUDA_TRY(ctx, cudaMemcpyAsync(b.side, a.side, keep * 1, cudaMemcpyDeviceToDevice, ctx->stream));
        CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    }
    free_soa(ctx->S);
    ctx->S = fresh;
    return WACOMM_B200_OK;
}

int reserve_work(wacomm_b200_context *ctx, size_t n) {
    if (n <= ctx->workCap && ctx->dKeys) return WACOMM_B200_OK;
    size_t cap = std::max(n, ctx->workCap + ctx->workCap / 2);
    size_t c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0;
    int rc;
    ctx->seqBounds.clear();
    if ((rc = grow(ctx, ctx->dKeys, c1, cap))) return rc;
    if ((rc = grow(ctx, ctx->dOrder, c2, cap))) return rc;
    if ((rc = grow(ctx, ctx->dFlags, c3, cap))) return rc;
    if ((rc = grow(ctx, ctx->dPositions, c4, cap))) return rc;
    if ((rc = grow(ctx, ctx->dSeq, c5, cap))) return rc;
    ctx->workCap = cap;
    return WACOMM_B200_OK;
}

int reserve_scan(wacomm_b200_context *ctx, size_t n) {
    size_t words = scan_temp_words(n);
    return grow(ctx, ctx->dScanTemp, ctx->scanTempCap, words);
}

int check_ready(wacomm_b200_context *ctx) {
    if (!ctx->hasConfig) return fail(ctx, WACOMM_B200_ERR_STATE, "set_config has not been called");
    if (!ctx->hasGrid) return fail(ctx, WACOMM_B200_ERR_STATE, "set_grid has not been called");
    if (ctx->times.empty()) return fail(ctx, WACOMM_B200_ERR_STATE, "set_times has not been called");
    return WACOMM_B200_OK;
}

int validate_options(wacomm_b200_context *ctx, const wacomm_b200_options &o) {
    if (o.semantics != WACOMM_B200_SEMANTICS_HOST && o.semantics != WACOMM_B200_SEMANTICS_DEVICE)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "semantics %d out of range", o.semantics);
    if (o.arithmetic != WACOMM_B200_ARITH_REFERENCE && o.arithmetic != WACOMM_B200_ARITH_FP32)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "arithmetic %d out of range", o.arithmetic);
    if (o.storage < WACOMM_B200_STORAGE_FP32 || o.storage > WACOMM_B200_STORAGE_BF16)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "storage %d out of range", o.storage);
    if (o.arithmetic == WACOMM_B200_ARITH_REFERENCE && o.storage != WACOMM_B200_STORAGE_FP32)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT,
                    "reference arithmetic reads the forcing exactly and needs FP32 storage");
    if (o.sort_by_cell < 0 || o.sort_by_cell > 64)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "sort_by_cell %d out of [0, 64]", o.sort_by_cell);
    if (o.rng != WACOMM_B200_RNG_REFERENCE && o.rng != WACOMM_B200_RNG_PHILOX)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "rng %d out of range", o.rng);
    if (o.block_size < 32 || o.block_size > 256 || o.block_size % 32)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "block_size %d: need a multiple of 32 in [32, 256]",
                    o.block_size);
    if (o.substeps_per_launch < 0)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "substeps_per_launch must be >= 0");
    if (o.launch_shape < WACOMM_B200_LAUNCH_SHAPE_AUTO || o.launch_shape > 3)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "launch_shape %d out of [-1, 3]", o.launch_shape);
    if (o.particles_per_thread < 1 || o.particles_per_thread > 16)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "particles_per_thread %d out of [1, 16]",
                    o.particles_per_thread);
    if (o.surrogate != 0 && o.surrogate != 1)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "surrogate %d: 0 or 1", o.surrogate);
    if (o.surrogate && o.arithmetic != WACOMM_B200_ARITH_FP32)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT,
                    "the surrogate hands uncovered particles to the FP32 step: needs FP32 arithmetic");
    return WACOMM_B200_OK;
}

int ensure_metric(wacomm_b200_context *ctx) {
    if (ctx->metricSemantics == ctx->opt.semantics) return WACOMM_B200_OK;
    CUDA_TRY(ctx, build_metric(ctx->opt.semantics, ctx->eta, ctx->xi, ctx->dLon, ctx->dLat,
                               ctx->dMetric, ctx->dInvMetric, ctx->stream));
    ctx->metricSemantics = ctx->opt.semantics;
    return WACOMM_B200_OK;
}

void release_frames(wacomm_b200_context *ctx) {
    for (FrameSlot &s : ctx->slots) {
        cudaFree(s.zeta);
        cudaFree(s.u);
        cudaFree(s.v);
        cudaFree(s.w);
        cudaFree(s.akt);
        cudaFree(s.windU);
        cudaFree(s.windV);
        cudaFree(s.stokesU);
        cudaFree(s.stokesV);
        if (s.ready) cudaEventDestroy(s.ready);
        s = FrameSlot{};
    }
    ctx->pairT0 = ctx->pairT1 = -1;
    ctx->zT0 = ctx->zT1 = -1;
}

// Forcing record t: the slot's own fields, with the wind and Stokes pairs taken from the regridded
// environment where the record was uploaded without them.
FrameDevice frame_of(const wacomm_b200_context *ctx, int t) {
    const FrameSlot &s = ctx->slots[t];
    FrameDevice f{s.zeta, s.u, s.v, s.w, s.akt, s.windU, s.windV, s.stokesU, s.stokesV};
    const size_t at = (size_t)t * ctx->eta * ctx->xi;
    if (!s.windU && !s.windV && ctx->env[0].u) {
        f.windU = ctx->env[0].u + at;
        f.windV = ctx->env[0].v + at;
    }
    if (!s.stokesU && ctx->env[1].u) {
        f.stokesU = ctx->env[1].u + at;
        f.stokesV = ctx->env[1].v + at;
    }
    return f;
}

void release_roms(wacomm_b200_context *ctx) {
    cudaFree(ctx->dRomsMask);
    cudaFree(ctx->dRomsRot);
    cudaFree(ctx->dRomsRaw);
    ctx->dRomsMask = nullptr;
    ctx->dRomsRot = nullptr;
    ctx->dRomsRaw = nullptr;
    ctx->romsRawCap = 0;
    ctx->hasRoms = false;
}

void release_environment(wacomm_b200_context *ctx) {
    for (EnvField &e : ctx->env) {
        cudaFree(e.u);
        cudaFree(e.v);
        e = EnvField{};
    }
}

// Device buffers of the packed forcing pair (node records, environment pair, cell-column records).
int reserve_pair_buffers(wacomm_b200_context *ctx, bool env, bool cells) {
    size_t plane = (size_t)ctx->eta * ctx->xi;
    size_t need = plane * ctx->sW * node_record_bytes(ctx->opt.storage);
    if (need > ctx->nodesBytes) {
        cudaFree(ctx->dNodes);
        ctx->dNodes = nullptr;
        ctx->nodesBytes = 0;
        CUDA_TRY(ctx, cudaMalloc(&ctx->dNodes, need));
        ctx->nodesBytes = need;
    }
    if (env && !ctx->dEnv) CUDA_TRY(ctx, cudaMalloc(&ctx->dEnv, plane * sizeof(EnvPair)));
    if (cells) {
        size_t cneed = plane * ctx->sW * cell_record_bytes(ctx->opt.storage);
        if (cneed > ctx->cellsBytes) {
            cudaFree(ctx->dCells);
            ctx->dCells = nullptr;
            ctx->cellsBytes = 0;
            CUDA_TRY(ctx, cudaMalloc(&ctx->dCells, cneed));
            ctx->cellsBytes = cneed;
        }
        size_t sneed = plane * cell_surface_bytes();
        if (sneed > ctx->cellSurfaceBytes) {
            cudaFree(ctx->dCellSurface);
            ctx->dCellSurface = nullptr;
            ctx->cellSurfaceBytes = 0;
            CUDA_TRY(ctx, cudaMalloc(&ctx->dCellSurface, sneed));
            ctx->cellSurfaceBytes = sneed;
        }
    }
    return WACOMM_B200_OK;
}

int ensure_pair(wacomm_b200_context *ctx, int t0, int t1, int &launches) {
    const FrameDevice a = frame_of(ctx, t0), b = frame_of(ctx, t1);
    bool env = a.windU || a.windV || a.stokesU || b.windU || b.windV || b.stokesU;
    bool cells = ctx->opt.arithmetic == WACOMM_B200_ARITH_FP32;
    if (ctx->pairT0 == t0 && ctx->pairT1 == t1 && ctx->pairStorage == ctx->opt.storage &&
        ctx->pairEnv == env && (!cells || ctx->pairCells))
        return WACOMM_B200_OK;
    int rc = reserve_pair_buffers(ctx, env, cells);
    if (rc) return rc;
    CUDA_TRY(ctx, pack_pair(ctx->opt.storage, ctx->eta, ctx->xi, ctx->sW, a, b,
                            ctx->dH, ctx->dNodes, ctx->dSurf, env ? ctx->dEnv : nullptr,
                            ctx->stream));
    launches += 2;
    if (cells) {
        CUDA_TRY(ctx, pack_cells(ctx->opt.storage, ctx->eta, ctx->xi, ctx->sW, a, b, ctx->dH,
                                 ctx->dCells, ctx->dCellSurface, ctx->stream));
        launches += 2;
    }
    ctx->pairT0 = t0;
    ctx->pairT1 = t1;
    ctx->pairStorage = ctx->opt.storage;
    ctx->pairEnv = env;
    ctx->pairCells = cells;
    return WACOMM_B200_OK;
}

PackedArgs packed_args(wacomm_b200_context *ctx) {
    PackedArgs A;
    A.eta = ctx->eta;
    A.xi = ctx->xi;
    A.sW = ctx->sW;
    A.sRho = ctx->sRho;
    A.nodes = ctx->dNodes;
    A.surf = ctx->dSurf;
    A.env = ctx->pairEnv ? ctx->dEnv : nullptr;
    const FrameDevice a = frame_of(ctx, ctx->pairT0);
    A.hasWindU = ctx->pairEnv && a.windU;
    A.hasWindV = ctx->pairEnv && a.windV;
    A.hasStokes = ctx->pairEnv && a.stokesU && a.stokesV;
    A.lonRad = ctx->dLon;
    A.latRad = ctx->dLat;
    A.depthIntervals = ctx->dDepth;
    A.metric = ctx->dMetric;
    A.invMetric = ctx->dInvMetric;
    A.depthIntervalsF = ctx->dDepthF;
    A.cfgDevice = ctx->dCfg;
    A.cells = ctx->dCells;
    A.cellSurface = ctx->dCellSurface;
    return A;
}

// Histogram, offsets and scan scratch of the cell sort of `count` records.
int reserve_sort(wacomm_b200_context *ctx, size_t count) {
    size_t bins = (size_t)ctx->eta * ctx->xi + 1;
    if (ctx->binsCap < bins + 2 || !ctx->dHist || !ctx->dOffsets) {
        cudaFree(ctx->dHist);
        cudaFree(ctx->dOffsets);
        ctx->dHist = ctx->dOffsets = nullptr;
        ctx->binsCap = 0;
        CUDA_TRY(ctx, cudaMalloc(&ctx->dHist, (bins + 2) * sizeof(uint32_t)));
        CUDA_TRY(ctx, cudaMalloc(&ctx->dOffsets, (bins + 2) * sizeof(uint32_t)));
        ctx->binsCap = bins + 2;
    }
    return reserve_scan(ctx, std::max(bins, count));
}

// Orders `count` records by cell into order[]. A sort of the whole resident set walks the records
// in the previous full sort's order (when that is still a permutation of the slots) and keeps its
// own result for the next one; a sort of a slab walks its slots in order.
// Cell sort of `count` records: walks them in seqIn (a permutation of [0, count), or null: slot
// order) and copies the resulting order to seqOut (or not, if null).
int sort_work(wacomm_b200_context *ctx, const ParticleSoA &S, size_t count, uint32_t *keys,
              uint32_t *order, const uint32_t *seqIn, uint32_t *seqOut, int &launches) {
    size_t bins = (size_t)ctx->eta * ctx->xi + 1;
    int rc;
    if ((rc = reserve_sort(ctx, count))) return rc;
    CUDA_TRY(ctx, sort_by_cell(S.j, S.i, (int)count, ctx->eta, ctx->xi, seqIn, keys, ctx->dHist,
                               ctx->dOffsets, ctx->dScanTemp, order, ctx->stream));
    size_t blocks = (bins + 8191) / 8192;
    launches += 3 + (blocks > 1 ? 2 : 0);
    if (seqOut)
        CUDA_TRY(ctx, cudaMemcpyAsync(seqOut, order, count * sizeof(uint32_t),
                                      cudaMemcpyDeviceToDevice, ctx->stream));
    return WACOMM_B200_OK;
}

// Moves `count` resident records starting at `offset` over the interval (sort, chunks, count).
// The first sort walks seqIn (null: slot order); every sort leaves its order in seqOut, which the
// later chunks walk.
int run_interval(wacomm_b200_context *ctx, const IntervalParams &base, size_t offset, size_t count,
                 uint32_t *keys, uint32_t *order, const uint32_t *seqIn, uint32_t *seqOut,
                 int &launches) {
    if (count == 0) return WACOMM_B200_OK;
    ParticleSoA S = offset_soa(ctx->S.s, offset);
    PackedArgs A = packed_args(ctx);
    IntervalParams P = base;
    P.rng = ctx->opt.rng;
    MoveLaunch L;
    L.count = (int)count;
    L.order = nullptr;
    L.perThread = ctx->opt.particles_per_thread;
    int concTime = base.t0 + base.direction;
    bool count_here = ctx->opt.fuse_concentration && ctx->dConc && concTime >= 0 &&
                      concTime < ctx->concTimes;
    L.conc = count_here ? ctx->dConc : nullptr;
    if (count_here) ctx->concEvaluated[concTime] = 1;
    L.concTimeIndex = concTime;
    L.concTimes = ctx->concTimes;
    L.steps = ctx->dSteps;
    L.err = ctx->dErr;
    double chunk = ctx->opt.substeps_per_launch > 0 ? ctx->opt.substeps_per_launch * ctx->cfg.dti : 0;
    int nChunks = 1;
    if (chunk > 0 && base.length > 0) nChunks = (int)std::ceil(base.length / chunk);
    if (nChunks < 1) nChunks = 1;
    for (int c = 0; c < nChunks; c++) {
        // a sort cadence of N > 1: between sorts the work takes the last sort's order (any
        // permutation is a valid work order; the cell locality of a recent one is kept)
        const bool reuse = c == 0 && ctx->mayReuseOrder && seqIn && ctx->opt.sort_by_cell > 1 &&
                           ctx->sortedAgo + 1 < ctx->opt.sort_by_cell;
        if (reuse) {
            L.order = seqIn;
            ctx->sortedAgo++;
        } else if (ctx->opt.sort_by_cell) {
            int rc = sort_work(ctx, S, count, keys, order, c == 0 ? seqIn : seqOut, seqOut,
                               launches);
            if (rc) return rc;
            L.order = order;
            if (c == 0) ctx->sortedAgo = 0;
        }
        if (!ctx->moveTimed && !ctx->capturing) {
            CUDA_TRY(ctx, cudaEventRecord(ctx->evMove0, ctx->stream));
            ctx->moveTimed = true;
        }
        if (c == 0) {
            int rc = timing_begin(ctx);
            if (!rc) rc = timing_mark(ctx);
            if (rc) return rc;
        }
        P.firstChunk = c == 0;
        P.lastChunk = c == nChunks - 1;
        P.chunkEnd = P.lastChunk ? INFINITY : (c + 1) * chunk;
        cudaError_t e;
        if (ctx->opt.arithmetic == WACOMM_B200_ARITH_REFERENCE)
            e = move_ref_dispatch(ctx->opt.semantics, ctx->cfg, P, A, S, L, ctx->opt.block_size,
                                  ctx->stream);
        else
            e = move_f32_dispatch(ctx->opt.semantics, ctx->opt.storage, ctx->opt.launch_shape,
                                  ctx->cfg, P, A, S, L, ctx->stream);
        if (e != cudaSuccess)
            return fail(ctx, WACOMM_B200_ERR_CUDA, "move launch: %s", cudaGetErrorString(e));
        launches++;
        if (!ctx->capturing) CUDA_TRY(ctx, cudaEventRecord(ctx->evMove1, ctx->stream));
    }
    return timing_mark(ctx);
}

int prepare_interval(wacomm_b200_context *ctx, int time_index, IntervalParams &P, int &launches) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (time_index < 0 || time_index >= (int)ctx->times.size())
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "time_index %d out of [0, %zu)", time_index,
                    ctx->times.size());
    make_interval(ctx->cfg, ctx->times.data(), (int)ctx->times.size(), time_index, ctx->sW,
                  ctx->opt.semantics, P);
    if (P.skip) return WACOMM_B200_OK;
    if (!ctx->slots[P.t0].loaded || !ctx->slots[P.t1].loaded)
        return fail(ctx, WACOMM_B200_ERR_STATE, "forcing records %d and %d must be uploaded", P.t0,
                    P.t1);
    for (int t : {P.t0, P.t1}) {
        FrameSlot &slot = ctx->slots[t];
        if (slot.pending) {
            CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, slot.ready, 0));
            slot.pending = false;
        }
    }
    if ((rc = ensure_metric(ctx))) return rc;
    if ((rc = ensure_pair(ctx, P.t0, P.t1, launches))) return rc;
    return WACOMM_B200_OK;
}

int run_surrogate(wacomm_b200_context *ctx, const IntervalParams &P, int &launches);

// Buffers and tables a surrogate interval uses, sized (and the dry-node table built) before the
// interval, so that a captured run allocates nothing: the dry-node prefix sums of the current
// shore limit, the per-cell-level layer-1 sums and corner records, the fallback list and the rows.
int reserve_surrogate(wacomm_b200_context *ctx, int *launches = nullptr) {
    int rc;
    const size_t dryNeed = (size_t)(ctx->eta + 1) * (ctx->xi + 1);
    if (!ctx->dryValid || !(ctx->dryShore == ctx->cfg.shoreLimit)) {
        if ((rc = grow(ctx, ctx->dDry, ctx->dryCap, dryNeed))) return rc;
        CUDA_TRY(ctx, surrogate_dry_prefix(ctx->hasMask ? ctx->dMask : nullptr, ctx->dH,
                                           ctx->cfg.shoreLimit, ctx->eta, ctx->xi, ctx->dDry,
                                           ctx->stream));
        if (launches) *launches += 2;
        ctx->dryShore = ctx->cfg.shoreLimit;
        ctx->dryValid = true;
    }
    const long long nCL = surrogate_cell_levels(ctx->eta, ctx->xi, ctx->sW);
    if ((size_t)nCL > ctx->zCap) {
        cudaFree(ctx->dZ);
        cudaFree(ctx->dCorners);
        ctx->dZ = nullptr;
        ctx->dCorners = nullptr;
        ctx->zCap = 0;
        ctx->zT0 = ctx->zT1 = -1;
        CUDA_TRY(ctx, cudaMalloc(&ctx->dZ, (size_t)nCL * 256 * sizeof(__half)));
        CUDA_TRY(ctx, cudaMalloc(&ctx->dCorners, (size_t)nCL * surrogate_corner_bytes()));
        ctx->zCap = (size_t)nCL;
    }
    if (ctx->n) {
        if ((rc = grow(ctx, ctx->dFallback, ctx->fallbackCap, ctx->n))) return rc;
        if ((rc = grow(ctx, ctx->dSurrRows, ctx->surrRowsCap, ctx->n))) return rc;
    }
    return WACOMM_B200_OK;
}

// The work of one interval on the compute stream (pair packing, sort, move, fused count).
int enqueue_interval(wacomm_b200_context *ctx, int time_index, int &launches) {
    IntervalParams P;
    int rc = prepare_interval(ctx, time_index, P, launches);
    if (rc) return rc;
    ctx->surrTimed = false;
    if (P.skip || !ctx->n) return WACOMM_B200_OK;
    if (ctx->opt.surrogate) return run_surrogate(ctx, P, launches);
    if ((rc = reserve_work(ctx, ctx->n))) return rc;
    const std::vector<size_t> whole{0, ctx->n};
    const uint32_t *seqIn = ctx->seqBounds == whole ? ctx->dSeq : nullptr;
    ctx->seqBounds.clear();
    ctx->mayReuseOrder = true;
    rc = run_interval(ctx, P, 0, ctx->n, ctx->dKeys, ctx->dOrder, seqIn, ctx->dSeq, launches);
    ctx->mayReuseOrder = false;
    if (rc) return rc;
    if (ctx->opt.sort_by_cell) ctx->seqBounds = whole;
    return WACOMM_B200_OK;
}

// Surrogate interval: per-cell layer 1 for the forcing pair, cell sort, the tensor-core step, then
// the plain FP32 step over the particles the surrogate handed back.
int run_surrogate(wacomm_b200_context *ctx, const IntervalParams &P, int &launches) {
    if (!ctx->hasSurrogate)
        return fail(ctx, WACOMM_B200_ERR_STATE, "the surrogate option needs set_surrogate weights");
    const size_t count = ctx->n;
    if (count == 0) return WACOMM_B200_OK;
    int rc;
    const FrameDevice a = frame_of(ctx, P.t0), b = frame_of(ctx, P.t1);
    if ((rc = reserve_surrogate(ctx, &launches))) return rc;
    // layer 1 per cell-level
    CUDA_TRY(ctx, cudaEventRecord(ctx->evCell0, ctx->stream));
    if (ctx->zT0 != P.t0 || ctx->zT1 != P.t1 || ctx->zSemantics != ctx->metricSemantics) {
        CUDA_TRY(ctx, surrogate_cells(ctx->eta, ctx->xi, ctx->sW, ctx->sRho, a, b,
                                      ctx->dH, ctx->dDepth, ctx->dMetric, ctx->dSurrogate, ctx->dZ,
                                      ctx->dCorners, ctx->dErr, ctx->smCount, ctx->stream));
        launches++;
        ctx->zT0 = P.t0;
        ctx->zT1 = P.t1;
        ctx->zSemantics = ctx->metricSemantics;
    }
    CUDA_TRY(ctx, cudaEventRecord(ctx->evCell1, ctx->stream));
    // Work in slot order, unsorted: the per-cell data the step kernel gathers (FP16 layer-1 sums
    // and corner records) stays in L2, while the particle state is read and written coalesced.
    if ((rc = reserve_work(ctx, count))) return rc;
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->dSurrCounts, 0, 2 * sizeof(unsigned long long), ctx->stream));
    MoveLaunch L;
    L.count = (int)count;
    L.order = nullptr;
    const int concTime = P.t0 + P.direction;
    const bool countHere = ctx->opt.fuse_concentration && ctx->dConc && concTime >= 0 &&
                           concTime < ctx->concTimes;
    L.conc = countHere ? ctx->dConc : nullptr;
    if (countHere) ctx->concEvaluated[concTime] = 1;
    L.concTimeIndex = concTime;
    L.concTimes = ctx->concTimes;
    L.steps = ctx->dSteps;
    L.err = ctx->dErr;
    SurrogateStep st;
    st.eta = ctx->eta;
    st.xi = ctx->xi;
    st.sW = ctx->sW;
    st.sRho = ctx->sRho;
    st.start = P.start;
    st.length = P.length;
    st.cfg = ctx->cfg;
    // Diffusive forward intervals keep the surrogate's displacement and add the plain stochastic
    // operator per substep (the walk kernel); backward, restart-clipped, empty and jibing intervals
    // go to the plain step whole.
    const bool diffuse = ctx->cfg.random && (P.direction > 0 || ctx->cfg.backwardDiffusion);
    st.fallbackAll = P.direction < 0 || P.elapsed0 != 0 || P.length <= 0 ||
                     ctx->cfg.leewayJibeProbabilityHourly > 0;
    IntervalParams Q = P;
    Q.rng = ctx->opt.rng;
    Q.firstChunk = 1;
    Q.lastChunk = 1;
    Q.chunkEnd = INFINITY;
    const PackedArgs A = packed_args(ctx);
    st.walk = diffuse ? 1 : 0;
    st.maxError = ctx->surrMaxError;
    st.semantics = ctx->opt.semantics;
    st.storage = ctx->opt.storage;
    st.interval = &Q;
    st.cells = A.cells;
    st.cellSurface = A.cellSurface;
    st.invMetric = A.invMetric;
    st.depthF = A.depthIntervalsF;
    if (diffuse && ctx->opt.sort_by_cell) {
        // the walk takes its particles in cell order; the sort walks the previous order (with a
        // sort cadence N > 1, the intervals between sorts take that order as it is)
        const std::vector<size_t> whole{0, ctx->n};
        const uint32_t *seqIn = ctx->seqBounds == whole ? ctx->dSeq : nullptr;
        if (seqIn && ctx->opt.sort_by_cell > 1 && ctx->sortedAgo + 1 < ctx->opt.sort_by_cell) {
            ctx->sortedAgo++;
            st.walkOrder = seqIn;
        } else {
            ctx->seqBounds.clear();
            if ((rc = sort_work(ctx, ctx->S.s, count, ctx->dKeys, ctx->dOrder, seqIn, ctx->dSeq,
                                launches)))
                return rc;
            ctx->seqBounds = whole;
            ctx->sortedAgo = 0;
            st.walkOrder = ctx->dOrder;
        }
    }
    st.dry = ctx->dDry;
    st.z = ctx->dZ;
    st.corners = ctx->dCorners;
    st.weights = ctx->dSurrogate;
    st.fallback = ctx->dFallback;
    st.fallbackCount = reinterpret_cast<uint32_t *>(ctx->dSurrCounts);
    st.runCount = ctx->dSurrCounts + 1;
    st.rows = ctx->dSurrRows;
    CUDA_TRY(ctx, cudaEventRecord(ctx->evMove0, ctx->stream));
    CUDA_TRY(ctx, cudaEventRecord(ctx->evStep0, ctx->stream));
    ctx->moveTimed = true;
    if ((rc = timing_begin(ctx)) || (rc = timing_mark(ctx))) return rc;
    st.midEvent = ctx->timingCur ? ctx->timingCur->ev[1] : nullptr;
    if (ctx->timingCur) ctx->timingCur->marks = 2;  // ev[1] is recorded between the two kernels
    CUDA_TRY(ctx, surrogate_step(st, ctx->S.s, L, ctx->smCount, ctx->stream));
    launches += 2;
    CUDA_TRY(ctx, cudaEventRecord(ctx->evStep1, ctx->stream));
    if ((rc = timing_mark(ctx))) return rc;
    ctx->surrTimed = !ctx->capturing;
    ctx->surrRan = true;
    // The plain FP32 step over the fallback list, whose length the kernels above left on the
    // device: the launch covers every particle and the blocks past the list exit at once, so the
    // host never waits for the count and the interval can be captured.
    MoveLaunch F = L;
    F.count = (int)count;
    F.order = ctx->dFallback;
    F.countDevice = reinterpret_cast<const uint32_t *>(ctx->dSurrCounts);
    cudaError_t e = move_f32_dispatch(ctx->opt.semantics, ctx->opt.storage, ctx->opt.launch_shape,
                                      ctx->cfg, Q, A, ctx->S.s, F, ctx->stream);
    if (e != cudaSuccess)
        return fail(ctx, WACOMM_B200_ERR_CUDA, "fallback move launch: %s", cudaGetErrorString(e));
    launches++;
    CUDA_TRY(ctx, cudaEventRecord(ctx->evMove1, ctx->stream));
    return timing_mark(ctx);
}

int check_errors(wacomm_b200_context *ctx) {
    int flags = 0;
    CUDA_TRY(ctx, cudaMemcpy(&flags, ctx->dErr, sizeof(int), cudaMemcpyDeviceToHost));
    if (flags & ERR_DRIFT_OBJECT) {
        CUDA_TRY(ctx, cudaMemset(ctx->dErr, 0, sizeof(int)));
        return fail(ctx, WACOMM_B200_ERR_DRIFT_OBJECT,
                    "a particle names a drift object outside the catalogue (ids 0-22)");
    }
    if (flags & ERR_SURROGATE_WAIT) {
        CUDA_TRY(ctx, cudaMemset(ctx->dErr, 0, sizeof(int)));
        return fail(ctx, WACOMM_B200_ERR_CUDA,
                    "a surrogate kernel gave up waiting on a tensor-core or copy barrier");
    }
    return WACOMM_B200_OK;
}

}  // namespace

extern "C" {

const char *wacomm_b200_version(void) { return "wacomm_b200 1.0 (sm_100a)"; }

int wacomm_b200_device_count(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return count;
}

int wacomm_b200_default_options(wacomm_b200_options *out) {
    if (!out) return WACOMM_B200_ERR_ARGUMENT;
    out->semantics = WACOMM_B200_SEMANTICS_HOST;
    out->arithmetic = WACOMM_B200_ARITH_FP32;
    out->storage = WACOMM_B200_STORAGE_FP32;
    out->rng = WACOMM_B200_RNG_REFERENCE;
    out->block_size = 256;
    out->substeps_per_launch = 0;
    out->sort_by_cell = 1;
    out->fuse_concentration = 1;
    out->launch_shape = WACOMM_B200_LAUNCH_SHAPE_AUTO;
    out->surrogate = 0;
    out->particles_per_thread = 1;
    return WACOMM_B200_OK;
}

int wacomm_b200_context_create(int device, wacomm_b200_context **out) {
    if (!out) return WACOMM_B200_ERR_ARGUMENT;
    *out = nullptr;
    int count = wacomm_b200_device_count();
    if (device < 0 || device >= count) return WACOMM_B200_ERR_ARGUMENT;
    wacomm_b200_context *ctx = new wacomm_b200_context();
    ctx->device = device;
    wacomm_b200_default_options(&ctx->opt);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->h2d, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->d2h, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->evLaneStart, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->evLaneDone, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev1);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->evComputeMark, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->evMove0);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->evMove1);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->dSteps, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(ctx->dSteps, 0, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&ctx->dErr, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&ctx->dCount, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(ctx->dErr, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->evCell0);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->evCell1);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->evStep0);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->evStep1);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->dSurrCounts, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->smCount, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        wacomm_b200_context_destroy(ctx);
        return WACOMM_B200_ERR_CUDA;
    }
    *out = ctx;
    return WACOMM_B200_OK;
}

int wacomm_b200_context_destroy(wacomm_b200_context *ctx) {
    if (!ctx) return WACOMM_B200_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->h2d) cudaStreamSynchronize(ctx->h2d);
    release_frames(ctx);
    cudaFree(ctx->dMask);
    cudaFree(ctx->dLon);
    cudaFree(ctx->dLat);
    cudaFree(ctx->dH);
    cudaFree(ctx->dDepth);
    cudaFree(ctx->dMetric);
    cudaFree(ctx->dInvMetric);
    cudaFree(ctx->dDepthF);
    cudaFree(ctx->dNodes);
    cudaFree(ctx->dCells);
    cudaFree(ctx->dCellSurface);
    cudaFree(ctx->dSurf);
    cudaFree(ctx->dEnv);
    free_soa(ctx->S);
    free_soa(ctx->T);
    cudaFree(ctx->dKeys);
    cudaFree(ctx->dOrder);
    cudaFree(ctx->dSeq);
    cudaFree(ctx->dFlags);
    cudaFree(ctx->dPositions);
    cudaFree(ctx->dHist);
    cudaFree(ctx->dOffsets);
    cudaFree(ctx->dScanTemp);
    cudaFree(ctx->dHist2);
    cudaFree(ctx->dOffsets2);
    cudaFree(ctx->dScanTemp2);
    cudaFree(ctx->dCount);
    cudaFree(ctx->dAos);
    cudaFree(ctx->dConc);
    cudaFree(ctx->dSurrogate);
    cudaFree(ctx->dZ);
    cudaFree(ctx->dCorners);
    cudaFree(ctx->dDry);
    cudaFree(ctx->dFallback);
    cudaFree(ctx->dSurrRows);
    cudaFree(ctx->dSurrCounts);
    if (ctx->evCell0) cudaEventDestroy(ctx->evCell0);
    if (ctx->evCell1) cudaEventDestroy(ctx->evCell1);
    if (ctx->evStep0) cudaEventDestroy(ctx->evStep0);
    if (ctx->evStep1) cudaEventDestroy(ctx->evStep1);
    cudaFree(ctx->dSources);
    cudaFree(ctx->dEmitScratch);
    cudaFree(ctx->dGeoLon);
    cudaFree(ctx->dGeoLat);
    cudaFree(ctx->dSWValues);
    cudaFree(ctx->dGeoOut);
    release_environment(ctx);
    release_roms(ctx);
    if (ctx->graphExec) cudaGraphExecDestroy(ctx->graphExec);
    cudaFree(ctx->dSteps);
    cudaFree(ctx->dErr);
    cudaFree(ctx->dCfg);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->evComputeMark) cudaEventDestroy(ctx->evComputeMark);
    if (ctx->evMove0) cudaEventDestroy(ctx->evMove0);
    if (ctx->evMove1) cudaEventDestroy(ctx->evMove1);
    for (auto &t : ctx->timing)
        for (cudaEvent_t e : t.ev)
            if (e) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->h2d) cudaStreamDestroy(ctx->h2d);
    if (ctx->d2h) cudaStreamDestroy(ctx->d2h);
    if (ctx->stream2) cudaStreamDestroy(ctx->stream2);
    if (ctx->evLaneStart) cudaEventDestroy(ctx->evLaneStart);
    if (ctx->evLaneDone) cudaEventDestroy(ctx->evLaneDone);
    delete ctx;
    return WACOMM_B200_OK;
}

const char *wacomm_b200_last_error(const wacomm_b200_context *ctx) {
    return ctx ? ctx->error.c_str() : "null context";
}

int wacomm_b200_set_options(wacomm_b200_context *ctx, const wacomm_b200_options *options) {
    if (!ctx || !options) return WACOMM_B200_ERR_ARGUMENT;
    int rc = validate_options(ctx, *options);
    if (rc) return rc;
    ctx->opt = *options;
    return WACOMM_B200_OK;
}

int wacomm_b200_get_options(const wacomm_b200_context *ctx, wacomm_b200_options *out) {
    if (!ctx || !out) return WACOMM_B200_ERR_ARGUMENT;
    *out = ctx->opt;
    return WACOMM_B200_OK;
}

int wacomm_b200_set_config(wacomm_b200_context *ctx, const wacomm_b200_config *config) {
    if (!ctx || !config) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "null config");
    if (config->trackingDirection != 1 && config->trackingDirection != -1)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "trackingDirection must be 1 or -1");
    if (!(config->dti > 0)) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "dti must be > 0");
    if (config->observationalCalibrationRegionCount > 16)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "more than 16 calibration regions");
    cudaSetDevice(ctx->device);
    if (!ctx->dCfg) CUDA_TRY(ctx, cudaMalloc(&ctx->dCfg, sizeof(wacomm_b200_config)));
    // kernels of earlier intervals may still read the previous copy
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(ctx, cudaMemcpy(ctx->dCfg, config, sizeof(wacomm_b200_config), cudaMemcpyHostToDevice));
    ctx->cfg = *config;
    ctx->hasConfig = true;
    return WACOMM_B200_OK;
}

int wacomm_b200_set_grid(wacomm_b200_context *ctx, int eta, int xi, int s_rho, int s_w,
                         const double *mask, const double *lon_rad, const double *lat_rad,
                         const double *h, const double *depth_intervals) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (eta < 2 || xi < 2 || s_rho < 1 || s_w != s_rho + 1)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "grid %dx%d with s_rho=%d s_w=%d: need eta,xi>=2, "
                    "s_rho>=1, s_w=s_rho+1", eta, xi, s_rho, s_w);
    if ((size_t)eta * xi >= ((size_t)1 << 31) - 2)
        return fail(ctx, WACOMM_B200_ERR_CAPACITY, "grid of %zu cells exceeds 2^31-2",
                    (size_t)eta * xi);
    if (!lon_rad || !lat_rad || !h || !depth_intervals)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "null grid array");
    cudaSetDevice(ctx->device);
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->h2d));
    size_t plane = (size_t)eta * xi;
    cudaFree(ctx->dMask);
    cudaFree(ctx->dLon);
    cudaFree(ctx->dLat);
    cudaFree(ctx->dH);
    cudaFree(ctx->dDepth);
    cudaFree(ctx->dMetric);
    cudaFree(ctx->dInvMetric);
    cudaFree(ctx->dDepthF);
    cudaFree(ctx->dSurf);
    ctx->dMask = ctx->dLon = ctx->dLat = ctx->dH = ctx->dDepth = nullptr;
    ctx->dMetric = nullptr;
    ctx->dInvMetric = nullptr;
    ctx->dDepthF = nullptr;
    ctx->dSurf = nullptr;
    cudaFree(ctx->dEnv);
    ctx->dEnv = nullptr;
    ctx->hasGrid = false;
    cudaFree(ctx->dGeoLon);
    cudaFree(ctx->dGeoLat);
    cudaFree(ctx->dSWValues);
    ctx->dGeoLon = ctx->dGeoLat = ctx->dSWValues = nullptr;
    ctx->hasGeo = false;
    release_environment(ctx);
    release_roms(ctx);
    CUDA_TRY(ctx, cudaMalloc(&ctx->dLon, plane * sizeof(double)));
    CUDA_TRY(ctx, cudaMalloc(&ctx->dLat, plane * sizeof(double)));
    CUDA_TRY(ctx, cudaMalloc(&ctx->dH, plane * sizeof(double)));
    CUDA_TRY(ctx, cudaMalloc(&ctx->dDepth, (size_t)(s_w - 1) * sizeof(double)));
    CUDA_TRY(ctx, cudaMalloc(&ctx->dMetric, plane * sizeof(double2)));
    CUDA_TRY(ctx, cudaMalloc(&ctx->dInvMetric, plane * sizeof(float2)));
    CUDA_TRY(ctx, cudaMalloc(&ctx->dDepthF, (size_t)(s_w - 1) * sizeof(float)));
    CUDA_TRY(ctx, cudaMalloc(&ctx->dSurf, plane * sizeof(SurfPair)));
    CUDA_TRY(ctx, cudaMemcpy(ctx->dLon, lon_rad, plane * sizeof(double), cudaMemcpyHostToDevice));
    CUDA_TRY(ctx, cudaMemcpy(ctx->dLat, lat_rad, plane * sizeof(double), cudaMemcpyHostToDevice));
    CUDA_TRY(ctx, cudaMemcpy(ctx->dH, h, plane * sizeof(double), cudaMemcpyHostToDevice));
    CUDA_TRY(ctx, cudaMemcpy(ctx->dDepth, depth_intervals, (size_t)(s_w - 1) * sizeof(double),
                             cudaMemcpyHostToDevice));
    {
        std::vector<float> depthF(depth_intervals, depth_intervals + (s_w - 1));
        CUDA_TRY(ctx, cudaMemcpy(ctx->dDepthF, depthF.data(), depthF.size() * sizeof(float),
                                 cudaMemcpyHostToDevice));
    }
    ctx->hasMask = mask != nullptr;
    if (mask) {
        CUDA_TRY(ctx, cudaMalloc(&ctx->dMask, plane * sizeof(double)));
        CUDA_TRY(ctx, cudaMemcpy(ctx->dMask, mask, plane * sizeof(double), cudaMemcpyHostToDevice));
    }
    ctx->eta = eta;
    ctx->xi = xi;
    ctx->sRho = s_rho;
    ctx->sW = s_w;
    ctx->metricSemantics = -1;
    ctx->pairT0 = ctx->pairT1 = -1;
    ctx->zT0 = ctx->zT1 = -1;
    ctx->dryValid = false;
    ctx->hasGrid = true;
    // Forcing records of another grid no longer fit: release them.
    release_frames(ctx);
    return WACOMM_B200_OK;
}

int wacomm_b200_set_times(wacomm_b200_context *ctx, int n_times, const double *ocean_time) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (n_times < 1 || !ocean_time) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "need >= 1 time");
    cudaSetDevice(ctx->device);
    if (ctx->env[0].u || ctx->env[1].u) {
        // regridded fields were aligned to the previous times
        if (ctx->times.size() != (size_t)n_times ||
            !std::equal(ctx->times.begin(), ctx->times.end(), ocean_time)) {
            CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
            release_environment(ctx);
        }
    }
    ctx->times.assign(ocean_time, ocean_time + n_times);
    if ((int)ctx->slots.size() < n_times) ctx->slots.resize(n_times);
    ctx->pairT0 = ctx->pairT1 = -1;
    ctx->zT0 = ctx->zT1 = -1;
    return WACOMM_B200_OK;
}

}  // extern "C"

namespace {

// Copies forcing record t from host arrays into its device slot on the copy stream. Synchronous:
// the compute stream is drained first and the copies are waited for. Asynchronous: the copy
// stream waits for the work enqueued so far on the compute stream (which may still read the
// slot), and the slot's ready event is recorded for the next interval to wait on.
// With copyOcean false the ocean fields' device arrays are only allocated (their values come from
// a kernel afterwards).
int stage_frame(wacomm_b200_context *ctx, int t, const float *zeta, const float *u, const float *v,
                const float *w, const float *akt, const float *wind_u10, const float *wind_v10,
                const float *stokes_u, const float *stokes_v, bool async, bool copyOcean = true) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (!ctx->hasGrid) return fail(ctx, WACOMM_B200_ERR_STATE, "set_grid has not been called");
    if (t < 0 || t >= (int)ctx->times.size())
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "frame %d out of [0, %zu)", t, ctx->times.size());
    if (!zeta || !u || !v || !w || !akt) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "null field");
    if ((stokes_u == nullptr) != (stokes_v == nullptr))
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "stokes_u and stokes_v come together");
    cudaSetDevice(ctx->device);
    size_t plane = (size_t)ctx->eta * ctx->xi;
    FrameSlot &s = ctx->slots[t];
    auto put = [&](float *&dst, const float *src, size_t count) -> int {
        if (!src) {
            if (dst) {
                CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
                CUDA_TRY(ctx, cudaStreamSynchronize(ctx->h2d));
                cudaFree(dst);
            }
            dst = nullptr;
            return WACOMM_B200_OK;
        }
        if (!dst) CUDA_TRY(ctx, cudaMalloc(&dst, count * sizeof(float)));
        CUDA_TRY(ctx, cudaMemcpyAsync(dst, src, count * sizeof(float), cudaMemcpyHostToDevice,
                                      ctx->h2d));
        return WACOMM_B200_OK;
    };
    if (async) {
        if (!s.ready) CUDA_TRY(ctx, cudaEventCreateWithFlags(&s.ready, cudaEventDisableTiming));
        // kernels already enqueued may read this slot (through the pair packing): copy after them
        CUDA_TRY(ctx, cudaEventRecord(ctx->evComputeMark, ctx->stream));
        CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->h2d, ctx->evComputeMark, 0));
    } else {
        // The pair cache may reference this slot: finish kernels that read it first.
        CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    }
    auto ocean = [&](float *&dst, const float *src, size_t count) -> int {
        if (copyOcean) return put(dst, src, count);
        if (!dst) CUDA_TRY(ctx, cudaMalloc(&dst, count * sizeof(float)));
        return WACOMM_B200_OK;
    };
    int rc;
    if ((rc = ocean(s.zeta, zeta, plane))) return rc;
    if ((rc = ocean(s.u, u, plane * ctx->sRho))) return rc;
    if ((rc = ocean(s.v, v, plane * ctx->sRho))) return rc;
    if ((rc = ocean(s.w, w, plane * ctx->sW))) return rc;
    if ((rc = ocean(s.akt, akt, plane * ctx->sW))) return rc;
    if ((rc = put(s.windU, wind_u10, plane))) return rc;
    if ((rc = put(s.windV, wind_v10, plane))) return rc;
    if ((rc = put(s.stokesU, stokes_u, plane))) return rc;
    if ((rc = put(s.stokesV, stokes_v, plane))) return rc;
    if (async) {
        CUDA_TRY(ctx, cudaEventRecord(s.ready, ctx->h2d));
        s.pending = true;
    } else {
        CUDA_TRY(ctx, cudaStreamSynchronize(ctx->h2d));
        s.pending = false;
    }
    s.loaded = true;
    if (ctx->pairT0 == t || ctx->pairT1 == t) ctx->pairT0 = ctx->pairT1 = -1;
    if (ctx->zT0 == t || ctx->zT1 == t) ctx->zT0 = ctx->zT1 = -1;
    return WACOMM_B200_OK;
}

}  // namespace

extern "C" {

int wacomm_b200_upload_frame(wacomm_b200_context *ctx, int t, const float *zeta, const float *u,
                             const float *v, const float *w, const float *akt,
                             const float *wind_u10, const float *wind_v10, const float *stokes_u,
                             const float *stokes_v) {
    return stage_frame(ctx, t, zeta, u, v, w, akt, wind_u10, wind_v10, stokes_u, stokes_v, false);
}

int wacomm_b200_upload_frame_async(wacomm_b200_context *ctx, int t, const float *zeta,
                                   const float *u, const float *v, const float *w,
                                   const float *akt, const float *wind_u10,
                                   const float *wind_v10, const float *stokes_u,
                                   const float *stokes_v) {
    return stage_frame(ctx, t, zeta, u, v, w, akt, wind_u10, wind_v10, stokes_u, stokes_v, true);
}

int wacomm_b200_set_particles(wacomm_b200_context *ctx, const wacomm_b200_particle *host,
                              size_t n) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    ctx->n = 0;
    ctx->sortedAgo = 1 << 30;
    return wacomm_b200_append_particles(ctx, host, n);
}

int wacomm_b200_append_particles(wacomm_b200_context *ctx, const wacomm_b200_particle *host,
                                 size_t n) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (n == 0) return WACOMM_B200_OK;
    if (!host) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "null particles");
    ctx->sortedAgo = 1 << 30;
    if (ctx->n + n >= MAX_PARTICLES)
        return fail(ctx, WACOMM_B200_ERR_CAPACITY, "more than 2^31 particles");
    cudaSetDevice(ctx->device);
    int rc;
    if ((rc = reserve_particles(ctx, ctx->n + n, ctx->n))) return rc;
    if ((rc = grow(ctx, ctx->dAos, ctx->aosCap, n))) return rc;
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->dAos, host, n * sizeof(wacomm_b200_particle),
                                  cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, aos_to_soa(ctx->dAos, (int)n, offset_soa(ctx->S.s, ctx->n), ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->n += n;
    return WACOMM_B200_OK;
}

int wacomm_b200_get_particles(wacomm_b200_context *ctx, wacomm_b200_particle *out, size_t n) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (n < ctx->n) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "buffer of %zu for %zu records", n, ctx->n);
    if (ctx->n == 0) return WACOMM_B200_OK;
    if (!out) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "null output");
    cudaSetDevice(ctx->device);
    int rc;
    if ((rc = grow(ctx, ctx->dAos, ctx->aosCap, ctx->n))) return rc;
    CUDA_TRY(ctx, soa_to_aos(ctx->S.s, (int)ctx->n, ctx->dAos, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(out, ctx->dAos, ctx->n * sizeof(wacomm_b200_particle),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return check_errors(ctx);
}

int wacomm_b200_particle_count(const wacomm_b200_context *ctx, size_t *out) {
    if (!ctx || !out) return WACOMM_B200_ERR_ARGUMENT;
    *out = ctx->n;
    return WACOMM_B200_OK;
}

int wacomm_b200_move_interval(wacomm_b200_context *ctx, int time_index) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    cudaSetDevice(ctx->device);
    int launches = 0;
    ctx->moveTimed = false;
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->dSteps, 0, sizeof(unsigned long long), ctx->stream));
    CUDA_TRY(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    int rc = enqueue_interval(ctx, time_index, launches);
    if (rc) return rc;
    CUDA_TRY(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    CUDA_TRY(ctx, accumulate_steps(ctx->dSteps, ctx->dSteps + 1, ctx->stream));
    ctx->lastLaunches = launches;
    return WACOMM_B200_OK;
}

}  // extern "C"

namespace {

// Runs the enclosed slab work on the second compute lane: its stream and sort scratch take the
// place of the main ones until the guard ends.
struct LaneSwap {
    wacomm_b200_context *ctx;
    bool active;
    LaneSwap(wacomm_b200_context *c, bool second) : ctx(c), active(second) { swap(); }
    ~LaneSwap() { swap(); }
    void swap() {
        if (!active) return;
        std::swap(ctx->stream, ctx->stream2);
        std::swap(ctx->dHist, ctx->dHist2);
        std::swap(ctx->dOffsets, ctx->dOffsets2);
        std::swap(ctx->binsCap, ctx->binsCap2);
        std::swap(ctx->dScanTemp, ctx->dScanTemp2);
        std::swap(ctx->scanTempCap, ctx->scanTempCap2);
    }
};

}  // namespace

extern "C" {

int wacomm_b200_move_interval_host(wacomm_b200_context *ctx, int time_index,
                                   wacomm_b200_particle *particles, size_t n) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (n && !particles) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "null particles");
    if (n >= MAX_PARTICLES) return fail(ctx, WACOMM_B200_ERR_CAPACITY, "more than 2^31 particles");
    cudaSetDevice(ctx->device);
    IntervalParams P;
    int launches = 0;
    ctx->moveTimed = false;
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->dSteps, 0, sizeof(unsigned long long), ctx->stream));
    int rc = prepare_interval(ctx, time_index, P, launches);
    if (rc) return rc;
    if ((rc = reserve_particles(ctx, n, 0))) return rc;
    if ((rc = reserve_work(ctx, n))) return rc;
    if ((rc = grow(ctx, ctx->dAos, ctx->aosCap, n))) return rc;
    ctx->n = n;
    // Slabs: the upload of slab s+1 and the download of slab s-1 overlap the move of slab s. Only
    // the first upload and the last download are exposed, so the end slabs are small (1/32 of the
    // records) and the slabs double from there (1/16, 1/8) up to pieces of at most 4 M records in
    // the middle: a slab's move (about 3 ns per record) outlasts the copy of a neighbour twice its
    // size (about 1.2 ns per record each way over PCIe), so the compute never waits for a copy.
    std::vector<size_t> bounds{0};
    if (n >= ((size_t)4 << 20)) {
        const size_t e = n / 32, ramp = 7 * e, rest = n - 2 * ramp;
        const size_t pieces = (rest + ((size_t)4 << 20) - 1) / ((size_t)4 << 20);
        bounds.push_back(e);
        bounds.push_back(3 * e);
        bounds.push_back(ramp);
        for (size_t q = 1; q < pieces; q++) bounds.push_back(ramp + rest * q / pieces);
        bounds.push_back(n - ramp);
        bounds.push_back(n - 3 * e);
        bounds.push_back(n - e);
        bounds.push_back(n);
    } else {
        const size_t pieces = n >= ((size_t)2 << 20) ? 2 : 1;
        for (size_t q = 1; q <= pieces; q++) bounds.push_back(n * q / pieces);
    }
    const int slabs = (int)bounds.size() - 1;
    std::vector<cudaEvent_t> up(slabs), done(slabs);
    for (int s = 0; s < slabs; s++) {
        cudaEventCreateWithFlags(&up[s], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&done[s], cudaEventDisableTiming);
    }
    // each slab's sort walks that slab's previous order when the last call had the same slabs
    const bool sorts = !P.skip && ctx->opt.sort_by_cell;
    const bool walk = sorts && ctx->seqBounds == bounds;
    if (sorts) ctx->seqBounds.clear();
    CUDA_TRY(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    // Slab s runs on compute lane s % 2 (LaneSwap), the last two on the main lane: the next
    // slab's conversion, sort and move fill the SMs that the previous slab's move releases in its
    // last wave. The second lane starts after the work enqueued so far on the main stream (the
    // forcing pair of the interval).
    CUDA_TRY(ctx, cudaEventRecord(ctx->evLaneStart, ctx->stream));
    CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream2, ctx->evLaneStart, 0));
    for (int s = 0; s < slabs; s++) {
        size_t off = bounds[s], cnt = bounds[s + 1] - bounds[s];
        if (cnt == 0) continue;
        CUDA_TRY(ctx, cudaMemcpyAsync(ctx->dAos + off, particles + off,
                                      cnt * sizeof(wacomm_b200_particle), cudaMemcpyHostToDevice,
                                      ctx->h2d));
        CUDA_TRY(ctx, cudaEventRecord(up[s], ctx->h2d));
    }
    for (int s = 0; s < slabs; s++) {
        size_t off = bounds[s], cnt = bounds[s + 1] - bounds[s];
        if (cnt == 0) continue;
        // the ramp-down slabs (the last three) run on the main lane after both lanes are done,
        // in order, so that each download overlaps the next slab's move
        if (s == slabs - 3 && s > 0) {
            CUDA_TRY(ctx, cudaEventRecord(ctx->evLaneDone, ctx->stream2));
            CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, ctx->evLaneDone, 0));
        }
        LaneSwap lane(ctx, (s & 1) != 0 && s < slabs - 3);
        CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, up[s], 0));
        ParticleSoA S = offset_soa(ctx->S.s, off);
        CUDA_TRY(ctx, aos_to_soa(ctx->dAos + off, (int)cnt, S, ctx->stream));
        launches++;
        if (!P.skip) {
            if ((rc = run_interval(ctx, P, off, cnt, ctx->dKeys + off, ctx->dOrder + off,
                                   walk ? ctx->dSeq + off : nullptr, ctx->dSeq + off, launches)))
                return rc;
        }
        CUDA_TRY(ctx, soa_to_aos(S, (int)cnt, ctx->dAos + off, ctx->stream));
        launches++;
        CUDA_TRY(ctx, cudaEventRecord(done[s], ctx->stream));
        CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->d2h, done[s], 0));
        CUDA_TRY(ctx, cudaMemcpyAsync(particles + off, ctx->dAos + off,
                                      cnt * sizeof(wacomm_b200_particle), cudaMemcpyDeviceToHost,
                                      ctx->d2h));
    }
    if (sorts) ctx->seqBounds = bounds;
    CUDA_TRY(ctx, cudaEventRecord(ctx->evLaneDone, ctx->stream2));
    CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, ctx->evLaneDone, 0));
    CUDA_TRY(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    CUDA_TRY(ctx, accumulate_steps(ctx->dSteps, ctx->dSteps + 1, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->d2h));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    for (int s = 0; s < slabs; s++) {
        cudaEventDestroy(up[s]);
        cudaEventDestroy(done[s]);
    }
    ctx->lastLaunches = launches;
    return check_errors(ctx);
}

int wacomm_b200_remove_dead(wacomm_b200_context *ctx) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (ctx->n == 0) return WACOMM_B200_OK;
    ctx->sortedAgo = 1 << 30;
    cudaSetDevice(ctx->device);
    int rc;
    if ((rc = reserve_work(ctx, ctx->n))) return rc;
    if ((rc = reserve_scan(ctx, ctx->n))) return rc;
    if (ctx->T.cap < ctx->n && (rc = alloc_soa(ctx, ctx->T, ctx->S.cap))) return rc;
    CUDA_TRY(ctx, compact_alive(ctx->S.s, (int)ctx->n, ctx->T.s, ctx->dFlags, ctx->dPositions,
                                ctx->dScanTemp, ctx->dCount, ctx->stream));
    uint32_t kept = 0;
    CUDA_TRY(ctx, cudaMemcpyAsync(&kept, ctx->dCount, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    std::swap(ctx->S, ctx->T);
    ctx->n = kept;
    return WACOMM_B200_OK;
}

int wacomm_b200_emit(wacomm_b200_context *ctx, const wacomm_b200_source *sources, int n_sources,
                     double julian_start, double interval_start, double interval_end,
                     size_t *emitted) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (emitted) *emitted = 0;
    ctx->sortedAgo = 1 << 30;
    if (n_sources < 0 || (n_sources > 0 && !sources))
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "%d sources at %p", n_sources, (const void *)sources);
    if (!ctx->hasConfig) return fail(ctx, WACOMM_B200_ERR_STATE, "set_config has not been called");
    if (n_sources == 0) return WACOMM_B200_OK;
    cudaSetDevice(ctx->device);
    int rc;
    if ((rc = grow(ctx, ctx->dSources, ctx->sourcesCap, (size_t)n_sources))) return rc;
    if ((rc = grow(ctx, ctx->dEmitScratch, ctx->emitScratchCap, emission_scratch_bytes(n_sources))))
        return rc;
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->dSources, sources, n_sources * sizeof(wacomm_b200_source),
                                  cudaMemcpyHostToDevice, ctx->stream));
    uint64_t firstId = 0;  // Source.cpp:27: the last record's id + 1, or 0
    if (ctx->n) {
        CUDA_TRY(ctx, cudaMemcpyAsync(&firstId, ctx->S.s.id + ctx->n - 1, sizeof(uint64_t),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    }
    unsigned long long total = 0;
    int err = 0;
    CUDA_TRY(ctx, emission_plan(ctx->dSources, n_sources, julian_start, interval_start,
                                interval_end, ctx->dEmitScratch, &total, &err, ctx->stream));
    if (ctx->n) firstId += 1;
    if (err & 2) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "invalid source emission schedule");
    if (err & 4 || ctx->n + total >= MAX_PARTICLES)
        return fail(ctx, WACOMM_B200_ERR_CAPACITY, "emission of %llu records beyond 2^31", total);
    if (total == 0) return WACOMM_B200_OK;
    if ((rc = reserve_particles(ctx, ctx->n + total, ctx->n))) return rc;
    CUDA_TRY(ctx, emission_fill(ctx->dSources, n_sources, ctx->dEmitScratch, total, ctx->dCfg,
                                firstId, ctx->S.s, ctx->n, ctx->stream));
    ctx->n += total;
    if (emitted) *emitted = total;
    return WACOMM_B200_OK;
}

int wacomm_b200_set_geo_grid(wacomm_b200_context *ctx, const double *lon, const double *lat,
                             const double *s_w_values) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (!ctx->hasGrid) return fail(ctx, WACOMM_B200_ERR_STATE, "set_grid has not been called");
    if (!lon || !lat || !s_w_values) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "null geo array");
    cudaSetDevice(ctx->device);
    size_t plane = (size_t)ctx->eta * ctx->xi;
    if (!ctx->dGeoLon) {
        CUDA_TRY(ctx, cudaMalloc(&ctx->dGeoLon, plane * sizeof(double)));
        CUDA_TRY(ctx, cudaMalloc(&ctx->dGeoLat, plane * sizeof(double)));
        CUDA_TRY(ctx, cudaMalloc(&ctx->dSWValues, (size_t)ctx->sW * sizeof(double)));
    }
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->dGeoLon, lon, plane * sizeof(double), cudaMemcpyHostToDevice,
                                  ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->dGeoLat, lat, plane * sizeof(double), cudaMemcpyHostToDevice,
                                  ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->dSWValues, s_w_values, (size_t)ctx->sW * sizeof(double),
                                  cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->hasGeo = true;
    return WACOMM_B200_OK;
}

int wacomm_b200_geo_positions(wacomm_b200_context *ctx, double *depth, double *lat, double *lon,
                              size_t n) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (!ctx->hasGeo) return fail(ctx, WACOMM_B200_ERR_STATE, "set_geo_grid has not been called");
    if (n < ctx->n) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "buffers of %zu for %zu records", n, ctx->n);
    if (ctx->n == 0) return WACOMM_B200_OK;
    if (!depth || !lat || !lon) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "null output");
    cudaSetDevice(ctx->device);
    int rc;
    if ((rc = grow(ctx, ctx->dGeoOut, ctx->geoOutCap, 3 * ctx->n))) return rc;
    double *dDep = ctx->dGeoOut, *dLat = dDep + ctx->n, *dLon = dLat + ctx->n;
    CUDA_TRY(ctx, geo_positions(ctx->S.s, (int)ctx->n, ctx->eta, ctx->xi, ctx->sW, ctx->dGeoLon,
                                ctx->dGeoLat, ctx->dH, ctx->dSWValues, dDep, dLat, dLon, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(depth, dDep, ctx->n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(lat, dLat, ctx->n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(lon, dLon, ctx->n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return WACOMM_B200_OK;
}

static int save_text_impl(wacomm_b200_context *ctx, const char *path);
static int save_netcdf_impl(wacomm_b200_context *ctx, const char *path,
                            const wacomm_b200_history_meta *meta, size_t *written);

// The host buffers of the writers are as large as the resident records: an allocation failure
// ends as an error status, not an exception through the C boundary.
int wacomm_b200_save_text(wacomm_b200_context *ctx, const char *path) {
    if (!ctx || !path) return WACOMM_B200_ERR_ARGUMENT;
    try {
        return save_text_impl(ctx, path);
    } catch (const std::exception &e) {
        return fail(ctx, WACOMM_B200_ERR_IO, "text restart: %s", e.what());
    }
}

int wacomm_b200_save_netcdf(wacomm_b200_context *ctx, const char *path,
                            const wacomm_b200_history_meta *meta, size_t *written) {
    if (!ctx || !path || !meta) return WACOMM_B200_ERR_ARGUMENT;
    try {
        return save_netcdf_impl(ctx, path, meta, written);
    } catch (const std::exception &e) {
        return fail(ctx, WACOMM_B200_ERR_IO, "NetCDF history: %s", e.what());
    }
}

static int save_text_impl(wacomm_b200_context *ctx, const char *path) {
    cudaSetDevice(ctx->device);
    std::vector<wacomm_b200_particle> host(ctx->n);
    if (ctx->n) {
        int rc;
        if ((rc = grow(ctx, ctx->dAos, ctx->aosCap, ctx->n))) return rc;
        CUDA_TRY(ctx, soa_to_aos(ctx->S.s, (int)ctx->n, ctx->dAos, ctx->stream));
        CUDA_TRY(ctx, cudaMemcpyAsync(host.data(), ctx->dAos, ctx->n * sizeof(wacomm_b200_particle),
                                      cudaMemcpyDeviceToHost, ctx->stream));
        CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    }
    if (history_text_write(path, host.data(), host.size()))
        return fail(ctx, WACOMM_B200_ERR_IO, "%s", wacomm_b200_file_error());
    return WACOMM_B200_OK;
}

static int save_netcdf_impl(wacomm_b200_context *ctx, const char *path,
                            const wacomm_b200_history_meta *meta, size_t *written) {
    if (written) *written = 0;
    if (!ctx->hasConfig) return fail(ctx, WACOMM_B200_ERR_STATE, "set_config has not been called");
    if (!ctx->hasGeo) return fail(ctx, WACOMM_B200_ERR_STATE, "set_geo_grid has not been called");
    cudaSetDevice(ctx->device);
    const size_t n = ctx->n;
    size_t kept = 0;
    std::vector<uint8_t> payload;
    if (n) {
        int rc;
        if ((rc = grow(ctx, ctx->dGeoOut, ctx->geoOutCap, 3 * n))) return rc;
        if ((rc = reserve_work(ctx, n))) return rc;
        if ((rc = reserve_scan(ctx, n))) return rc;
        double *dDep = ctx->dGeoOut, *dLat = dDep + n, *dLon = dLat + n;
        CUDA_TRY(ctx, geo_positions(ctx->S.s, (int)n, ctx->eta, ctx->xi, ctx->sW, ctx->dGeoLon,
                                    ctx->dGeoLat, ctx->dH, ctx->dSWValues, dDep, dLat, dLon,
                                    ctx->stream));
        CUDA_TRY(ctx, history_select(ctx->S.s, (int)n, dDep, dLat, dLon, ctx->dFlags, ctx->stream));
        CUDA_TRY(ctx, exclusive_scan(ctx->dFlags, ctx->dPositions, n, ctx->dCount, ctx->dScanTemp,
                                     ctx->stream));
        uint32_t total = 0;
        CUDA_TRY(ctx, cudaMemcpyAsync(&total, ctx->dCount, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                      ctx->stream));
        CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        kept = total;
        if (kept) {
            uint8_t *dPayload = nullptr;
            const size_t bytes = history_payload_bytes(kept);
            CUDA_TRY(ctx, cudaMallocAsync((void **)&dPayload, bytes, ctx->stream));
            payload.resize(bytes);
            cudaError_t e = history_pack(ctx->S.s, (int)n, ctx->dFlags, ctx->dPositions, dDep, dLat,
                                         dLon, kept, dPayload, ctx->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(payload.data(), dPayload, bytes, cudaMemcpyDeviceToHost,
                                    ctx->stream);
            cudaError_t f = cudaFreeAsync(dPayload, ctx->stream);
            if (e == cudaSuccess) e = f;
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess)
                return fail(ctx, WACOMM_B200_ERR_CUDA, "history payload: %s", cudaGetErrorString(e));
        }
    }
    const std::string header = history_header_for(*meta, ctx->cfg.trackingDirection < 0,
                                                  ctx->cfg.randomSeed, kept);
    if (history_netcdf_write(path, header, meta->checkpoint_time, payload.data(), payload.size()))
        return fail(ctx, WACOMM_B200_ERR_IO, "%s", wacomm_b200_file_error());
    if (written) *written = kept;
    return check_errors(ctx);
}

int wacomm_b200_concentration_reset(wacomm_b200_context *ctx, int n_conc_times) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (!ctx->hasGrid) return fail(ctx, WACOMM_B200_ERR_STATE, "set_grid has not been called");
    if (n_conc_times < 1) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "need >= 1 concentration time");
    cudaSetDevice(ctx->device);
    size_t cells = (size_t)n_conc_times * ctx->sRho * ctx->eta * ctx->xi;
    if (ctx->concTimes != n_conc_times) {
        cudaFree(ctx->dConc);
        ctx->dConc = nullptr;
        ctx->concTimes = 0;
        CUDA_TRY(ctx, cudaMalloc(&ctx->dConc, cells * sizeof(uint32_t)));
        ctx->concTimes = n_conc_times;
    }
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->dConc, 0, cells * sizeof(uint32_t), ctx->stream));
    ctx->concEvaluated.assign((size_t)n_conc_times, 0);
    return WACOMM_B200_OK;
}

int wacomm_b200_concentration_count(wacomm_b200_context *ctx, int conc_time_index) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (!ctx->dConc) return fail(ctx, WACOMM_B200_ERR_STATE, "concentration_reset has not been called");
    if (conc_time_index < 0 || conc_time_index >= ctx->concTimes)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "concentration time %d out of range", conc_time_index);
    cudaSetDevice(ctx->device);
    CUDA_TRY(ctx, count_concentration(ctx->S.s, (int)ctx->n, conc_time_index, ctx->sRho, ctx->eta,
                                      ctx->xi, ctx->dConc, ctx->stream));
    ctx->concEvaluated[conc_time_index] = 1;
    return WACOMM_B200_OK;
}

int wacomm_b200_concentration_get(wacomm_b200_context *ctx, uint32_t *out, size_t n) {
    if (!ctx || !out) return WACOMM_B200_ERR_ARGUMENT;
    size_t cells = (size_t)ctx->concTimes * ctx->sRho * ctx->eta * ctx->xi;
    if (!ctx->dConc) return fail(ctx, WACOMM_B200_ERR_STATE, "concentration_reset has not been called");
    if (n < cells) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "buffer of %zu for %zu cells", n, cells);
    cudaSetDevice(ctx->device);
    CUDA_TRY(ctx, cudaMemcpyAsync(out, ctx->dConc, cells * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return WACOMM_B200_OK;
}

int wacomm_b200_concentration_device(wacomm_b200_context *ctx, void **device_ptr, size_t *cells) {
    if (!ctx || !device_ptr || !cells) return WACOMM_B200_ERR_ARGUMENT;
    if (!ctx->dConc) return fail(ctx, WACOMM_B200_ERR_STATE, "concentration_reset has not been called");
    *device_ptr = ctx->dConc;
    *cells = (size_t)ctx->concTimes * ctx->sRho * ctx->eta * ctx->xi;
    return WACOMM_B200_OK;
}

int wacomm_b200_concentration_get_float(wacomm_b200_context *ctx, float *out, size_t n,
                                        int mask_land) {
    if (!ctx || !out) return WACOMM_B200_ERR_ARGUMENT;
    size_t cells = (size_t)ctx->concTimes * ctx->sRho * ctx->eta * ctx->xi;
    if (!ctx->dConc) return fail(ctx, WACOMM_B200_ERR_STATE, "concentration_reset has not been called");
    if (n < cells) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "buffer of %zu for %zu cells", n, cells);
    if (mask_land && !ctx->hasMask) return fail(ctx, WACOMM_B200_ERR_STATE, "no mask was given");
    cudaSetDevice(ctx->device);
    float *dOut = nullptr;
    CUDA_TRY(ctx, cudaMallocAsync((void **)&dOut, cells * sizeof(float), ctx->stream));
    // one time at a time: land is masked only in the times counted since the last reset
    const size_t perTime = (size_t)ctx->sRho * ctx->eta * ctx->xi;
    cudaError_t e = cudaSuccess;
    for (int t = 0; t < ctx->concTimes && e == cudaSuccess; t++) {
        const bool mask = mask_land && ctx->concEvaluated[t];
        e = concentration_to_float(ctx->dConc + t * perTime, perTime, 1, ctx->sRho, ctx->eta,
                                   ctx->xi, mask ? ctx->dMask : nullptr, dOut + t * perTime,
                                   ctx->stream);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, dOut, cells * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
    cudaFreeAsync(dOut, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return fail(ctx, WACOMM_B200_ERR_CUDA, "%s", cudaGetErrorString(e));
    return WACOMM_B200_OK;
}

int wacomm_b200_synchronize(wacomm_b200_context *ctx) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    cudaSetDevice(ctx->device);
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->h2d));
    return check_errors(ctx);
}

int wacomm_b200_set_surrogate(wacomm_b200_context *ctx, const float *parameters, size_t count) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (!parameters) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "null surrogate parameters");
    if (count != surrogate_parameter_count())
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "surrogate needs %zu parameters, got %zu",
                    surrogate_parameter_count(), count);
    cudaSetDevice(ctx->device);
    std::vector<uint8_t> image(surrogate_packed_bytes());
    surrogate_pack(parameters, image.data());
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (!ctx->dSurrogate) CUDA_TRY(ctx, cudaMalloc(&ctx->dSurrogate, image.size()));
    CUDA_TRY(ctx, cudaMemcpy(ctx->dSurrogate, image.data(), image.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(ctx, surrogate_prepare());
    ctx->hasSurrogate = true;
    ctx->zT0 = ctx->zT1 = -1;
    return WACOMM_B200_OK;
}

int wacomm_b200_set_surrogate_error_limit(wacomm_b200_context *ctx, double metres) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (!(metres > 0))
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "error limit %g: must be > 0 (infinity: off)",
                    metres);
    ctx->surrMaxError = (float)metres;
    return WACOMM_B200_OK;
}

int wacomm_b200_last_surrogate_stats(const wacomm_b200_context *ctx, size_t *run, size_t *fallback,
                                     float *cell_ms, float *step_ms) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    unsigned long long counts[2] = {0, 0};
    float c = 0.f, s = 0.f;
    if (ctx->surrRan) {
        cudaSetDevice(ctx->device);
        wacomm_b200_context *m = const_cast<wacomm_b200_context *>(ctx);
        CUDA_TRY(m, cudaStreamSynchronize(ctx->stream));
        CUDA_TRY(m, cudaMemcpy(counts, ctx->dSurrCounts, sizeof(counts), cudaMemcpyDeviceToHost));
        if (ctx->surrTimed) {
            if (cudaEventElapsedTime(&c, ctx->evCell0, ctx->evCell1) != cudaSuccess) c = 0.f;
            if (cudaEventElapsedTime(&s, ctx->evStep0, ctx->evStep1) != cudaSuccess) s = 0.f;
        }
    }
    if (run) *run = (size_t)counts[1];
    if (fallback) *fallback = (size_t)(counts[0] & 0xffffffffull);
    if (cell_ms) *cell_ms = c;
    if (step_ms) *step_ms = s;
    return WACOMM_B200_OK;
}

int wacomm_b200_kernel_times(wacomm_b200_context *ctx, float *ms, int capacity, int *count) {
    if (!ctx || !count || (capacity > 0 && !ms)) return WACOMM_B200_ERR_ARGUMENT;
    cudaSetDevice(ctx->device);
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    const size_t n = std::min(ctx->timingCount, (size_t)std::max(capacity, 0));
    const size_t first = (ctx->timingNext + TIMING_RING - ctx->timingCount) % TIMING_RING;
    const size_t skip = ctx->timingCount - n;  // the oldest records that do not fit
    for (size_t q = 0; q < n; q++) {
        const wacomm_b200_context::TimedInterval &t = ctx->timing[(first + skip + q) % TIMING_RING];
        if (t.marks > 0) CUDA_TRY(ctx, cudaEventSynchronize(t.ev[t.marks - 1]));
        for (int m = 0; m < 3; m++) {
            float v = 0.f;
            if (m + 1 < t.marks) CUDA_TRY(ctx, cudaEventElapsedTime(&v, t.ev[m], t.ev[m + 1]));
            ms[3 * q + m] = v;
        }
    }
    *count = (int)n;
    ctx->timingCount = 0;
    ctx->timingCur = nullptr;
    return WACOMM_B200_OK;
}

int wacomm_b200_last_interval_stats(const wacomm_b200_context *ctx, float *device_ms,
                                    float *move_ms, int *kernel_launches, double *particle_steps) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    wacomm_b200_context *c = const_cast<wacomm_b200_context *>(ctx);
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaEventSynchronize(c->ev1));
    float ms = 0, mm = 0;
    CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    if (c->moveTimed) CUDA_TRY(c, cudaEventElapsedTime(&mm, c->evMove0, c->evMove1));
    unsigned long long steps = 0;
    CUDA_TRY(c, cudaMemcpy(&steps, c->dSteps, sizeof(steps), cudaMemcpyDeviceToHost));
    if (device_ms) *device_ms = ms;
    if (move_ms) *move_ms = mm;
    if (kernel_launches) *kernel_launches = c->lastLaunches;
    if (particle_steps) *particle_steps = (double)steps;
    return WACOMM_B200_OK;
}

int wacomm_b200_stream(const wacomm_b200_context *ctx, void **out) {
    if (!ctx || !out) return WACOMM_B200_ERR_ARGUMENT;
    *out = (void *)ctx->stream;
    return WACOMM_B200_OK;
}

}  // extern "C"

namespace {

// Source longitudes and target longitudes farther than this from the grid's reference longitude
// are refused (the reference steps them by 360 degrees in an unbounded loop).
constexpr double LONGITUDE_REACH = 3600.0;

double near_longitude_host(double value, double reference) {
    while (value - reference > 180) value -= 360;
    while (value - reference < -180) value += 360;
    return value;
}

int cell_bin_host(double v, double minimum, double maximum, int bins) {
    if (maximum == minimum) return 0;
    return std::max(0, std::min(bins - 1, (int)((v - minimum) / (maximum - minimum) * bins)));
}

// Device buffers of one call, freed on every return path.
struct Scratch {
    std::vector<void *> held;
    ~Scratch() {
        for (void *p : held) cudaFree(p);
    }
    template <class T> cudaError_t get(T *&p, size_t count) {
        p = nullptr;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) held.push_back(p);
        return e;
    }
};

// Rectilinear source checks of bilinearGeographic (EnvironmentalRegridder.cpp:243-258) and the
// axis checks of bracket (:14-19); fills the unwrapped axes.
const char *geographic_axes(int eta, int xi, const double *lon, const double *lat,
                            std::vector<double> &ax, std::vector<double> &ay) {
    ax.assign(xi, 0.0);
    ay.assign(eta, 0.0);
    for (int i = 0; i < xi; i++) ax[i] = lon[i];
    for (int j = 0; j < eta; j++) ay[j] = lat[(size_t)j * xi];
    for (int j = 0; j < eta; j++)
        for (int i = 0; i < xi; i++) {
            double x = lon[(size_t)j * xi + i], y = lat[(size_t)j * xi + i];
            if (!std::isfinite(x) || !std::isfinite(y) || std::abs(x - ax[i]) > 1.e-10 ||
                std::abs(y - ay[j]) > 1.e-10)
                return "bilinear geographic regridding requires a finite rectilinear source grid";
        }
    for (int i = 1; i < xi; i++) {
        if (!(std::abs(ax[i] - ax[i - 1]) <= LONGITUDE_REACH))
            return "source longitudes lie more than 3600 degrees apart";
        while (ax[i] - ax[i - 1] > 180) ax[i] -= 360;
        while (ax[i] - ax[i - 1] < -180) ax[i] += 360;
    }
    if (std::abs(ax.back() - ax.front()) > 360 + 1.e-10)
        return "the source longitude axis spans more than one revolution";
    for (const std::vector<double> *axis : {&ax, &ay}) {
        const std::vector<double> &a = *axis;
        bool rising = a.back() > a.front();
        for (size_t i = 1; i < a.size(); i++)
            if ((rising && a[i] <= a[i - 1]) || (!rising && a[i] >= a[i - 1]))
                return "a source axis is not strictly monotonic";
    }
    return nullptr;
}

struct CellIndexHost {
    std::vector<double4> box;
    std::vector<int> binStart, binCells;
    double minX = 0, maxX = 0, minY = 0, maxY = 0, reference = 0;
    int binsX = 1, binsY = 1;
};

// CurvilinearCellIndex (EnvironmentalRegridder.cpp:170-236) with cyclic longitudes: per-cell
// boxes on the branch of lon(0,0), bins about as many as cells with the aspect of the grid's box,
// and every cell listed, in index order, in each bin its box touches.
const char *build_cell_index(int eta, int xi, const double *lon, const double *lat,
                             CellIndexHost &ix) {
    const double reference = lon[0];
    if (!std::isfinite(reference)) return "curvilinear source coordinates must be finite";
    for (size_t n = 0; n < (size_t)eta * xi; n++) {
        if (!std::isfinite(lon[n]) || !std::isfinite(lat[n]))
            return "curvilinear source coordinates must be finite";
        if (!(std::abs(lon[n] - reference) <= LONGITUDE_REACH))
            return "source longitudes lie more than 3600 degrees apart";
    }
    const size_t cells = (size_t)(eta - 1) * (xi - 1);
    ix.box.resize(cells);
    for (int j = 0; j + 1 < eta; j++)
        for (int i = 0; i + 1 < xi; i++) {
            auto L = [&](int jj, int ii) { return lon[(size_t)jj * xi + ii]; };
            auto A = [&](int jj, int ii) { return lat[(size_t)jj * xi + ii]; };
            double x00 = L(j, i), x10 = near_longitude_host(L(j, i + 1), x00);
            double x01 = near_longitude_host(L(j + 1, i), x00);
            double x11 = near_longitude_host(L(j + 1, i + 1), x00);
            double y00 = A(j, i), y10 = A(j, i + 1), y01 = A(j + 1, i), y11 = A(j + 1, i + 1);
            double center = .25 * (x00 + x10 + x01 + x11);
            double shift = 360 * std::round((reference - center) / 360);
            ix.box[(size_t)j * (xi - 1) + i] =
                make_double4(std::min(std::min(x00, x10), std::min(x01, x11)) + shift,
                             std::max(std::max(x00, x10), std::max(x01, x11)) + shift,
                             std::min(std::min(y00, y10), std::min(y01, y11)),
                             std::max(std::max(y00, y10), std::max(y01, y11)));
        }
    ix.minX = ix.box[0].x;
    ix.maxX = ix.box[0].y;
    ix.minY = ix.box[0].z;
    ix.maxY = ix.box[0].w;
    for (const double4 &b : ix.box) {
        ix.minX = std::min(ix.minX, b.x);
        ix.maxX = std::max(ix.maxX, b.y);
        ix.minY = std::min(ix.minY, b.z);
        ix.maxY = std::max(ix.maxY, b.w);
    }
    double width = std::max(ix.maxX - ix.minX, 1.e-12), height = std::max(ix.maxY - ix.minY, 1.e-12);
    double scale = std::sqrt((double)cells);
    ix.binsX = std::max(1, (int)std::round(scale * std::sqrt(width / height)));
    ix.binsY = std::max(1, (int)std::round(scale * std::sqrt(height / width)));
    ix.binsX = std::min(ix.binsX, (int)cells);
    ix.binsY = std::min(ix.binsY, (int)cells);
    const size_t bins = (size_t)ix.binsX * ix.binsY;
    std::vector<size_t> start(bins + 1, 0);
    auto span = [&](const double4 &b, int &i0, int &i1, int &j0, int &j1) {
        i0 = cell_bin_host(b.x, ix.minX, ix.maxX, ix.binsX);
        i1 = cell_bin_host(b.y, ix.minX, ix.maxX, ix.binsX);
        j0 = cell_bin_host(b.z, ix.minY, ix.maxY, ix.binsY);
        j1 = cell_bin_host(b.w, ix.minY, ix.maxY, ix.binsY);
    };
    int i0, i1, j0, j1;
    for (const double4 &b : ix.box) {
        span(b, i0, i1, j0, j1);
        for (int jj = j0; jj <= j1; jj++)
            for (int ii = i0; ii <= i1; ii++) start[(size_t)jj * ix.binsX + ii + 1]++;
    }
    for (size_t b = 0; b < bins; b++) start[b + 1] += start[b];
    if (start[bins] >= ((size_t)1 << 31) || bins >= ((size_t)1 << 31) - 1)
        return "the source grid's cell index exceeds 2^31 entries";
    ix.binCells.assign(start[bins], 0);
    std::vector<size_t> fill(start.begin(), start.end() - 1);
    for (size_t c = 0; c < cells; c++) {
        span(ix.box[c], i0, i1, j0, j1);
        for (int jj = j0; jj <= j1; jj++)
            for (int ii = i0; ii <= i1; ii++) ix.binCells[fill[(size_t)jj * ix.binsX + ii]++] = (int)c;
    }
    ix.binStart.assign(start.begin(), start.end());
    ix.reference = reference;
    return nullptr;
}

// Source records for each forcing time: an equal time (1e-6 s) copies the record, a time strictly
// between two records blends them with timeWeight (NumericalHelpers.hpp:30-33).
const char *align_times(int nSrc, const double *src, const std::vector<double> &dst,
                        std::vector<RegridTime> &out) {
    for (int k = 0; k < nSrc; k++)
        if (!std::isfinite(src[k]) || (k && !(src[k] > src[k - 1])))
            return "source times must be finite and strictly increasing";
    out.clear();
    for (double t : dst) {
        int k0 = -1, k1 = -1;
        for (int k = 0; k < nSrc && k0 < 0; k++)
            if (std::abs(t - src[k]) <= 1.e-6) k0 = k1 = k;
        for (int k = 0; k + 1 < nSrc && k0 < 0; k++)
            if (t > src[k] && t < src[k + 1]) {
                k0 = k;
                k1 = k + 1;
            }
        if (k0 < 0) return "a forcing time lies outside the source times; extrapolation is prohibited";
        double alpha = 0.0;
        if (k1 != k0)
            alpha = std::max(0.0, std::min(1.0, (t - src[k0]) / (src[k1] - src[k0])));
        out.push_back(RegridTime{k0, k1, alpha});
    }
    return nullptr;
}

}  // namespace

extern "C" {

int wacomm_b200_regrid_environment(wacomm_b200_context *ctx, int field, int method, int src_eta,
                                   int src_xi, const double *src_lon, const double *src_lat,
                                   int src_times, const double *times, const float *u,
                                   const float *v) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (field != WACOMM_B200_FIELD_WIND && field != WACOMM_B200_FIELD_STOKES)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "field %d: wind (0) or Stokes (1)", field);
    if (method != WACOMM_B200_REGRID_BILINEAR_GEOGRAPHIC &&
        method != WACOMM_B200_REGRID_BILINEAR_CURVILINEAR_GEOGRAPHIC)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "regridding method %d out of range", method);
    if (!ctx->hasGrid || !ctx->hasGeo || ctx->times.empty())
        return fail(ctx, WACOMM_B200_ERR_STATE,
                    "regridding needs set_grid, set_geo_grid (the target nodes) and set_times");
    if (src_eta < 2 || src_xi < 2 || src_times < 1)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT,
                    "source grid %dx%d with %d records: need at least 2x2 and one record", src_eta,
                    src_xi, src_times);
    if (!src_lon || !src_lat || !times || !u || !v)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "null source array");
    const size_t srcPlane = (size_t)src_eta * src_xi;
    if (srcPlane >= ((size_t)1 << 31) - 1)
        return fail(ctx, WACOMM_B200_ERR_CAPACITY, "source grid of %zu nodes exceeds 2^31", srcPlane);
    const bool curvilinear = method == WACOMM_B200_REGRID_BILINEAR_CURVILINEAR_GEOGRAPHIC;
    std::vector<RegridTime> plan;
    if (const char *why = align_times(src_times, times, ctx->times, plan))
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "%s", why);
    std::vector<double> ax, ay;
    CellIndexHost ix;
    const char *why = curvilinear ? build_cell_index(src_eta, src_xi, src_lon, src_lat, ix)
                                  : geographic_axes(src_eta, src_xi, src_lon, src_lat, ax, ay);
    if (why) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "%s", why);

    cudaSetDevice(ctx->device);
    // intervals already enqueued may read the previous fields
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    const size_t plane = (size_t)ctx->eta * ctx->xi, T = ctx->times.size();
    EnvField &out = ctx->env[field];
    if (!out.u) {
        CUDA_TRY(ctx, cudaMalloc(&out.u, T * plane * sizeof(float)));
        CUDA_TRY(ctx, cudaMalloc(&out.v, T * plane * sizeof(float)));
    }
    Scratch scratch;
    float *dSrc;
    RegridPlan *dPlan;
    RegridTime *dTimes;
    int *dErr;
    const size_t values = srcPlane * (size_t)src_times;
    CUDA_TRY(ctx, scratch.get(dSrc, 2 * values));
    CUDA_TRY(ctx, scratch.get(dPlan, plane));
    CUDA_TRY(ctx, scratch.get(dTimes, T));
    CUDA_TRY(ctx, scratch.get(dErr, 1));
    CUDA_TRY(ctx, cudaMemcpyAsync(dSrc, u, values * sizeof(float), cudaMemcpyHostToDevice,
                                  ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(dSrc + values, v, values * sizeof(float), cudaMemcpyHostToDevice,
                                  ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(dTimes, plan.data(), T * sizeof(RegridTime),
                                  cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaMemsetAsync(dErr, 0, sizeof(int), ctx->stream));
    CUDA_TRY(ctx, regrid_check_finite(dSrc, (long long)(2 * values), dErr, ctx->stream));
    if (curvilinear) {
        double *dLon, *dLat;
        double4 *dBox;
        int *dStart, *dCells;
        CUDA_TRY(ctx, scratch.get(dLon, srcPlane));
        CUDA_TRY(ctx, scratch.get(dLat, srcPlane));
        CUDA_TRY(ctx, scratch.get(dBox, ix.box.size()));
        CUDA_TRY(ctx, scratch.get(dStart, ix.binStart.size()));
        CUDA_TRY(ctx, scratch.get(dCells, ix.binCells.size()));
        CUDA_TRY(ctx, cudaMemcpyAsync(dLon, src_lon, srcPlane * sizeof(double),
                                      cudaMemcpyHostToDevice, ctx->stream));
        CUDA_TRY(ctx, cudaMemcpyAsync(dLat, src_lat, srcPlane * sizeof(double),
                                      cudaMemcpyHostToDevice, ctx->stream));
        CUDA_TRY(ctx, cudaMemcpyAsync(dBox, ix.box.data(), ix.box.size() * sizeof(double4),
                                      cudaMemcpyHostToDevice, ctx->stream));
        CUDA_TRY(ctx, cudaMemcpyAsync(dStart, ix.binStart.data(), ix.binStart.size() * sizeof(int),
                                      cudaMemcpyHostToDevice, ctx->stream));
        if (!ix.binCells.empty())
            CUDA_TRY(ctx, cudaMemcpyAsync(dCells, ix.binCells.data(),
                                          ix.binCells.size() * sizeof(int), cudaMemcpyHostToDevice,
                                          ctx->stream));
        RegridCurvilinear C{dLon, dLat, dBox, dStart, dCells, ix.minX, ix.maxX, ix.minY, ix.maxY,
                            ix.reference, ix.binsX, ix.binsY, src_xi, src_eta};
        CUDA_TRY(ctx, regrid_plan_curvilinear(C, (long long)plane, ctx->dGeoLon, ctx->dGeoLat,
                                              dPlan, dErr, ctx->stream));
    } else {
        double *dAx, *dAy;
        CUDA_TRY(ctx, scratch.get(dAx, ax.size()));
        CUDA_TRY(ctx, scratch.get(dAy, ay.size()));
        CUDA_TRY(ctx, cudaMemcpyAsync(dAx, ax.data(), ax.size() * sizeof(double),
                                      cudaMemcpyHostToDevice, ctx->stream));
        CUDA_TRY(ctx, cudaMemcpyAsync(dAy, ay.data(), ay.size() * sizeof(double),
                                      cudaMemcpyHostToDevice, ctx->stream));
        RegridGeographic G{dAx, dAy, src_xi, src_eta, ax.back() > ax.front(),
                           ay.back() > ay.front(), .5 * (ax.front() + ax.back())};
        CUDA_TRY(ctx, regrid_plan_geographic(G, (long long)plane, ctx->dGeoLon, ctx->dGeoLat,
                                             dPlan, dErr, ctx->stream));
    }
    CUDA_TRY(ctx, regrid_apply(curvilinear, dPlan, (long long)plane, src_xi, (long long)srcPlane,
                               dSrc, dSrc + values, dTimes, (int)T, out.u, out.v, ctx->stream));
    int err = 0;
    CUDA_TRY(ctx, cudaMemcpyAsync(&err, dErr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->pairT0 = ctx->pairT1 = -1;
    ctx->zT0 = ctx->zT1 = -1;
    if (err) {
        cudaFree(out.u);
        cudaFree(out.v);
        out = EnvField{};
        const char *what = (err & REGRID_ERR_FIELD)    ? "the source field holds a non-finite value"
                           : (err & REGRID_ERR_TARGET) ? "a target coordinate is not finite or "
                                                         "lies more than 3600 degrees away"
                           : (err & REGRID_ERR_FOLDED) ? "the curvilinear source holds a folded or "
                                                         "singular cell"
                                                       : "a target node lies outside the source "
                                                         "grid; extrapolation is prohibited";
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "%s", what);
    }
    return WACOMM_B200_OK;
}

int wacomm_b200_clear_environment(wacomm_b200_context *ctx, int field) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (field != WACOMM_B200_FIELD_WIND && field != WACOMM_B200_FIELD_STOKES)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "field %d: wind (0) or Stokes (1)", field);
    cudaSetDevice(ctx->device);
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->env[field].u);
    cudaFree(ctx->env[field].v);
    ctx->env[field] = EnvField{};
    ctx->pairT0 = ctx->pairT1 = -1;
    ctx->zT0 = ctx->zT1 = -1;
    return WACOMM_B200_OK;
}

int wacomm_b200_get_environment(wacomm_b200_context *ctx, int field, int t, float *u, float *v) {
    if (!ctx || !u || !v) return WACOMM_B200_ERR_ARGUMENT;
    if (field != WACOMM_B200_FIELD_WIND && field != WACOMM_B200_FIELD_STOKES)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "field %d: wind (0) or Stokes (1)", field);
    if (!ctx->env[field].u)
        return fail(ctx, WACOMM_B200_ERR_STATE, "no regridded field %d", field);
    if (t < 0 || t >= (int)ctx->times.size())
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "frame %d out of [0, %zu)", t, ctx->times.size());
    cudaSetDevice(ctx->device);
    const size_t plane = (size_t)ctx->eta * ctx->xi;
    CUDA_TRY(ctx, cudaMemcpyAsync(u, ctx->env[field].u + t * plane, plane * sizeof(float),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(v, ctx->env[field].v + t * plane, plane * sizeof(float),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return WACOMM_B200_OK;
}

}  // extern "C"

namespace {

// Everything a captured run reads by address or by value: buffer addresses and sizes, the particle
// count, the forcing times, the run configuration and options. A graph is launched only while this
// is unchanged.
std::vector<uint64_t> layout_of(const wacomm_b200_context *ctx) {
    std::vector<uint64_t> f;
    auto add = [&](const void *p) { f.push_back((uint64_t)(uintptr_t)p); };
    auto bytes = [&](const void *p, size_t n) {
        const unsigned char *b = (const unsigned char *)p;
        for (size_t o = 0; o < n; o += 8) {
            uint64_t w = 0;
            std::memcpy(&w, b + o, std::min<size_t>(8, n - o));
            f.push_back(w);
        }
    };
    const ParticleSoA &S = ctx->S.s;
    f.push_back(ctx->n);
    for (const void *p : {(const void *)S.id, (const void *)S.k, (const void *)S.j,
                          (const void *)S.i, (const void *)S.health, (const void *)S.age,
                          (const void *)S.time, (const void *)S.type, (const void *)S.side,
                          (const void *)S.elapsed})
        add(p);
    for (const void *p : {(const void *)ctx->dKeys, (const void *)ctx->dOrder,
                          (const void *)ctx->dSeq,
                          (const void *)ctx->dHist, (const void *)ctx->dOffsets,
                          (const void *)ctx->dScanTemp, (const void *)ctx->dNodes,
                          (const void *)ctx->dCells, (const void *)ctx->dCellSurface,
                          (const void *)ctx->dSurf, (const void *)ctx->dEnv,
                          (const void *)ctx->dConc, (const void *)ctx->dMetric,
                          (const void *)ctx->dInvMetric, (const void *)ctx->dLon,
                          (const void *)ctx->dLat, (const void *)ctx->dH, (const void *)ctx->dDepth,
                          (const void *)ctx->dDepthF, (const void *)ctx->dMask,
                          (const void *)ctx->dCfg, (const void *)ctx->dSteps,
                          (const void *)ctx->dErr})
        add(p);
    f.push_back((uint64_t)ctx->concTimes);
    for (const FrameSlot &s : ctx->slots)
        for (const void *p : {(const void *)s.zeta, (const void *)s.u, (const void *)s.v,
                              (const void *)s.w, (const void *)s.akt, (const void *)s.windU,
                              (const void *)s.windV, (const void *)s.stokesU,
                              (const void *)s.stokesV})
            add(p);
    for (const EnvField &e : ctx->env) {
        add(e.u);
        add(e.v);
    }
    bytes(ctx->times.data(), ctx->times.size() * sizeof(double));
    bytes(&ctx->cfg, sizeof ctx->cfg);
    bytes(&ctx->opt, sizeof ctx->opt);
    // the learned form's buffers and its trust limit
    for (const void *p : {(const void *)ctx->dSurrogate, (const void *)ctx->dZ,
                          (const void *)ctx->dCorners, (const void *)ctx->dDry,
                          (const void *)ctx->dFallback, (const void *)ctx->dSurrRows,
                          (const void *)ctx->dSurrCounts})
        add(p);
    bytes(&ctx->surrMaxError, sizeof ctx->surrMaxError);
    return f;
}

void release_graph(wacomm_b200_context *ctx) {
    if (ctx->graphExec) cudaGraphExecDestroy(ctx->graphExec);
    ctx->graphExec = nullptr;
    ctx->graphLayout.clear();
    ctx->graphLaunches = 0;
}

}  // namespace

extern "C" {

int wacomm_b200_graph_capture(wacomm_b200_context *ctx, int first_time_index, int n_intervals) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    int rc = check_ready(ctx);
    if (rc) return rc;
    const int T = (int)ctx->times.size(), dir = ctx->cfg.trackingDirection;
    const int last = first_time_index + dir * (n_intervals - 1);
    if (n_intervals < 1 || first_time_index < 0 || first_time_index >= T || last < 0 || last >= T)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "intervals %d..%d out of [0, %d)",
                    first_time_index, last, T);
    if (ctx->opt.surrogate && !ctx->hasSurrogate)
        return fail(ctx, WACOMM_B200_ERR_STATE, "the surrogate option needs set_surrogate weights");
    cudaSetDevice(ctx->device);
    release_graph(ctx);
    // Uploads in flight finish first (their ready events lie outside the capture), and every
    // buffer the intervals use is sized now: nothing may be allocated while capturing.
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->h2d));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    for (FrameSlot &s : ctx->slots) s.pending = false;
    const bool cells = ctx->opt.arithmetic == WACOMM_B200_ARITH_FP32;
    for (int n = 0, t = first_time_index; n < n_intervals; n++, t += dir) {
        IntervalParams P;
        make_interval(ctx->cfg, ctx->times.data(), T, t, ctx->sW, ctx->opt.semantics, P);
        if (P.skip) continue;
        if (!ctx->slots[P.t0].loaded || !ctx->slots[P.t1].loaded)
            return fail(ctx, WACOMM_B200_ERR_STATE, "forcing records %d and %d must be uploaded",
                        P.t0, P.t1);
        const FrameDevice a = frame_of(ctx, P.t0), b = frame_of(ctx, P.t1);
        bool env = a.windU || a.windV || a.stokesU || b.windU || b.windV || b.stokesU;
        if ((rc = reserve_pair_buffers(ctx, env, cells))) return rc;
    }
    if ((rc = ensure_metric(ctx))) return rc;
    if (ctx->n) {
        if ((rc = reserve_work(ctx, ctx->n))) return rc;
        if (ctx->opt.sort_by_cell && (rc = reserve_sort(ctx, ctx->n))) return rc;
    }
    if (ctx->opt.surrogate && (rc = reserve_surrogate(ctx))) return rc;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->pairT0 = ctx->pairT1 = -1;  // the graph packs its own pairs
    ctx->zT0 = ctx->zT1 = -1;        // and evaluates its own per-cell layer 1
    CUDA_TRY(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    ctx->capturing = true;
    // The captured sorts' sequence is written only at launch, and what dSeq holds when the graph
    // is launched is not known here: the first captured sort walks slot order.
    const std::vector<size_t> seqBefore = ctx->seqBounds;
    ctx->seqBounds.clear();
    int launches = 0;
    cudaError_t e = cudaMemsetAsync(ctx->dSteps, 0, sizeof(unsigned long long), ctx->stream);
    rc = e == cudaSuccess ? WACOMM_B200_OK
                          : fail(ctx, WACOMM_B200_ERR_CUDA, "%s", cudaGetErrorString(e));
    for (int n = 0, t = first_time_index; n < n_intervals && !rc; n++, t += dir)
        rc = enqueue_interval(ctx, t, launches);
    ctx->capturing = false;
    ctx->graphSeqBounds = ctx->seqBounds;
    ctx->seqBounds = seqBefore;
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(ctx->stream, &graph);
    ctx->pairT0 = ctx->pairT1 = -1;  // nothing captured has run yet
    ctx->zT0 = ctx->zT1 = -1;
    if (!rc && e != cudaSuccess)
        rc = fail(ctx, WACOMM_B200_ERR_CUDA, "capture: %s", cudaGetErrorString(e));
    if (!rc) {
        e = cudaGraphInstantiate(&ctx->graphExec, graph, 0);
        if (e != cudaSuccess) {
            ctx->graphExec = nullptr;
            rc = fail(ctx, WACOMM_B200_ERR_CUDA, "instantiate: %s", cudaGetErrorString(e));
        }
    }
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (rc) return rc;
    ctx->graphLayout = layout_of(ctx);
    ctx->graphLaunches = launches;
    return WACOMM_B200_OK;
}

int wacomm_b200_graph_launch(wacomm_b200_context *ctx) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (!ctx->graphExec) return fail(ctx, WACOMM_B200_ERR_STATE, "no captured graph");
    if (layout_of(ctx) != ctx->graphLayout)
        return fail(ctx, WACOMM_B200_ERR_STATE,
                    "particles, buffers, times, config or options changed since the capture");
    cudaSetDevice(ctx->device);
    for (FrameSlot &s : ctx->slots)
        if (s.pending) {
            CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, s.ready, 0));
            s.pending = false;
        }
    ctx->moveTimed = false;
    CUDA_TRY(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    CUDA_TRY(ctx, cudaGraphLaunch(ctx->graphExec, ctx->stream));
    ctx->seqBounds = ctx->graphSeqBounds;
    CUDA_TRY(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    CUDA_TRY(ctx, accumulate_steps(ctx->dSteps, ctx->dSteps + 1, ctx->stream));
    ctx->pairT0 = ctx->pairT1 = -1;
    ctx->zT0 = ctx->zT1 = -1;
    ctx->surrTimed = false;
    ctx->lastLaunches = ctx->graphLaunches;
    return WACOMM_B200_OK;
}

int wacomm_b200_graph_release(wacomm_b200_context *ctx) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    cudaSetDevice(ctx->device);
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    release_graph(ctx);
    return WACOMM_B200_OK;
}

int wacomm_b200_autotune(wacomm_b200_context *ctx, int time_index, int *best, float *best_ms) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (ctx->opt.surrogate)
        return fail(ctx, WACOMM_B200_ERR_STATE, "autotune times the plain step: surrogate is on");
    if (!ctx->n) return fail(ctx, WACOMM_B200_ERR_STATE, "no resident particles to time");
    int rc = check_ready(ctx);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    const bool fp32 = ctx->opt.arithmetic == WACOMM_B200_ARITH_FP32;
    const std::vector<int> candidates = fp32 ? std::vector<int>{0, 1, 2, 3}
                                             : std::vector<int>{64, 128, 192, 256};
    // snapshot: records (AoS), concentration, then one timed interval per candidate from it
    const size_t n = ctx->n;
    if ((rc = grow(ctx, ctx->dAos, ctx->aosCap, n))) return rc;
    CUDA_TRY(ctx, soa_to_aos(ctx->S.s, (int)n, ctx->dAos, ctx->stream));
    const size_t concBytes = ctx->dConc ? (size_t)ctx->concTimes * ctx->sRho * ctx->eta * ctx->xi *
                                              sizeof(uint32_t)
                                        : 0;
    uint32_t *concCopy = nullptr;
    if (concBytes) {
        CUDA_TRY(ctx, cudaMalloc(&concCopy, concBytes));
        cudaError_t e = cudaMemcpyAsync(concCopy, ctx->dConc, concBytes, cudaMemcpyDeviceToDevice,
                                        ctx->stream);
        if (e != cudaSuccess) {
            cudaFree(concCopy);
            return fail(ctx, WACOMM_B200_ERR_CUDA, "%s", cudaGetErrorString(e));
        }
    }
    const wacomm_b200_options saved = ctx->opt;
    auto restore = [&]() -> cudaError_t {
        cudaError_t e = aos_to_soa(ctx->dAos, (int)n, ctx->S.s, ctx->stream);
        if (e == cudaSuccess && concBytes)
            e = cudaMemcpyAsync(ctx->dConc, concCopy, concBytes, cudaMemcpyDeviceToDevice,
                                ctx->stream);
        return e;
    };
    int chosen = fp32 ? saved.launch_shape : saved.block_size;
    float chosenMs = INFINITY;
    for (int pass = 0; pass < 2 && !rc; pass++)  // the first pass warms every variant up
        for (int c : candidates) {
            if (fp32) ctx->opt.launch_shape = c;
            else ctx->opt.block_size = c;
            cudaError_t e = restore();
            if (e != cudaSuccess) {
                rc = fail(ctx, WACOMM_B200_ERR_CUDA, "%s", cudaGetErrorString(e));
                break;
            }
            if ((rc = wacomm_b200_move_interval(ctx, time_index))) break;
            float ms = 0;
            e = cudaEventSynchronize(ctx->ev1);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
            if (e != cudaSuccess) {
                rc = fail(ctx, WACOMM_B200_ERR_CUDA, "%s", cudaGetErrorString(e));
                break;
            }
            if (pass == 1 && ms < chosenMs) {
                chosenMs = ms;
                chosen = c;
            }
        }
    ctx->opt = saved;
    if (!rc) {
        if (fp32) ctx->opt.launch_shape = chosen;
        else ctx->opt.block_size = chosen;
    }
    // Work items per thread of the FP32 step, with the chosen shape: one interval each from the
    // snapshot, the fastest kept in options.particles_per_thread.
    if (!rc && fp32) {
        int per = saved.particles_per_thread;
        float bestPer = INFINITY;
        for (int pass = 0; pass < 2 && !rc; pass++)
            for (int c : {1, 2, 4}) {
                ctx->opt.particles_per_thread = c;
                cudaError_t e = restore();
                if (e != cudaSuccess) {
                    rc = fail(ctx, WACOMM_B200_ERR_CUDA, "%s", cudaGetErrorString(e));
                    break;
                }
                if ((rc = wacomm_b200_move_interval(ctx, time_index))) break;
                float ms = 0;
                e = cudaEventSynchronize(ctx->ev1);
                if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
                if (e != cudaSuccess) {
                    rc = fail(ctx, WACOMM_B200_ERR_CUDA, "%s", cudaGetErrorString(e));
                    break;
                }
                if (pass == 1 && ms < bestPer) {
                    bestPer = ms;
                    per = c;
                }
            }
        ctx->opt.particles_per_thread = per;
    }
    // The sort cadence, with the chosen shape: four intervals from the snapshot sorting every
    // 1, 2 or 4 of them; the fastest run sets options.sort_by_cell (when sorting is on and the
    // four intervals lie inside the forcing window).
    const int dir = ctx->cfg.trackingDirection, T = (int)ctx->times.size();
    const int runEnd = time_index + 4 * dir;
    if (!rc && saved.sort_by_cell && runEnd >= 0 && runEnd < T) {
        int cadence = saved.sort_by_cell;
        float bestRun = INFINITY;
        for (int pass = 0; pass < 2 && !rc; pass++)
            for (int cad : {1, 2, 4}) {
                ctx->opt.sort_by_cell = cad;
                cudaError_t e = restore();
                if (e != cudaSuccess) {
                    rc = fail(ctx, WACOMM_B200_ERR_CUDA, "%s", cudaGetErrorString(e));
                    break;
                }
                ctx->sortedAgo = 1 << 30;  // every run starts with a sort
                float total = 0;
                for (int q = 0; q < 4 && !rc; q++) {
                    if ((rc = wacomm_b200_move_interval(ctx, time_index + q * dir))) break;
                    float ms = 0;
                    e = cudaEventSynchronize(ctx->ev1);
                    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
                    if (e != cudaSuccess) rc = fail(ctx, WACOMM_B200_ERR_CUDA, "%s", cudaGetErrorString(e));
                    total += ms;
                }
                if (!rc && pass == 1 && total < bestRun) {
                    bestRun = total;
                    cadence = cad;
                }
            }
        ctx->opt.sort_by_cell = cadence;
        ctx->sortedAgo = 1 << 30;
    }
    cudaError_t e = restore();
    cudaError_t s = cudaStreamSynchronize(ctx->stream);
    cudaFree(concCopy);
    if (rc) return rc;
    if (e != cudaSuccess || s != cudaSuccess)
        return fail(ctx, WACOMM_B200_ERR_CUDA, "%s", cudaGetErrorString(e != cudaSuccess ? e : s));
    if (best) *best = chosen;
    if (best_ms) *best_ms = chosenMs;
    return WACOMM_B200_OK;
}

}  // extern "C"

extern "C" {

int wacomm_b200_set_roms_grid(wacomm_b200_context *ctx, const double *mask_u,
                              const double *mask_v, const double *angle) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (!ctx->hasGrid || !ctx->hasMask)
        return fail(ctx, WACOMM_B200_ERR_STATE, "set_grid with the rho mask comes first");
    if (!mask_u || !mask_v) return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "null mask");
    cudaSetDevice(ctx->device);
    const int eta = ctx->eta, xi = ctx->xi;
    const size_t plane = (size_t)eta * xi, planeU = (size_t)eta * (xi - 1),
                 planeV = (size_t)(eta - 1) * xi;
    std::vector<double> maskRho(plane);
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(ctx, cudaMemcpy(maskRho.data(), ctx->dMask, plane * sizeof(double),
                             cudaMemcpyDeviceToHost));
    // ROMSAdapter.cpp:139-160: masks of 0 and 1 only, a finite angle at every wet node
    std::vector<uint8_t> bytes(plane + planeU + planeV);
    auto take = [&](const double *m, size_t count, uint8_t *out) {
        for (size_t n = 0; n < count; n++) {
            if (m[n] != 0.0 && m[n] != 1.0) return false;
            out[n] = m[n] > 0.0;
        }
        return true;
    };
    if (!take(maskRho.data(), plane, bytes.data()) || !take(mask_u, planeU, bytes.data() + plane) ||
        !take(mask_v, planeV, bytes.data() + plane + planeU))
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "ROMS masks must hold 0 or 1 only");
    std::vector<double2> rot;
    if (angle) {
        rot.resize(plane);
        for (size_t n = 0; n < plane; n++) {
            if (maskRho[n] > 0.0 && !std::isfinite(angle[n]))
                return fail(ctx, WACOMM_B200_ERR_ARGUMENT,
                            "ROMS angle is non-finite at wet rho node %zu", n);
            // ROMSAdapter.cpp:276-280, with the host libm the reference uses
            rot[n] = maskRho[n] > 0.0 ? make_double2(std::cos(angle[n]), std::sin(angle[n]))
                                      : make_double2(1.0, 0.0);
        }
    }
    release_roms(ctx);
    CUDA_TRY(ctx, cudaMalloc(&ctx->dRomsMask, bytes.size()));
    CUDA_TRY(ctx, cudaMemcpy(ctx->dRomsMask, bytes.data(), bytes.size(), cudaMemcpyHostToDevice));
    if (angle) {
        CUDA_TRY(ctx, cudaMalloc(&ctx->dRomsRot, plane * sizeof(double2)));
        CUDA_TRY(ctx, cudaMemcpy(ctx->dRomsRot, rot.data(), plane * sizeof(double2),
                                 cudaMemcpyHostToDevice));
    }
    ctx->hasRoms = true;
    return WACOMM_B200_OK;
}

int wacomm_b200_upload_roms_frame(wacomm_b200_context *ctx, int t, const float *zeta,
                                  const float *u_faces, const float *v_faces, const float *w,
                                  const float *akt, const float *wind_u10,
                                  const float *wind_v10, const float *stokes_u,
                                  const float *stokes_v) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (!ctx->hasRoms) return fail(ctx, WACOMM_B200_ERR_STATE, "set_roms_grid has not been called");
    if (t < 0 || t >= (int)ctx->times.size())
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "frame %d out of [0, %zu)", t, ctx->times.size());
    if (!zeta || !u_faces || !v_faces || !w || !akt)
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "null field");
    // wind and Stokes as upload_frame takes them; the ocean fields follow
    int rc = stage_frame(ctx, t, zeta, zeta, zeta, zeta, zeta, wind_u10, wind_v10, stokes_u,
                         stokes_v, false, false);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    const int eta = ctx->eta, xi = ctx->xi, sRho = ctx->sRho, sW = ctx->sW;
    const size_t plane = (size_t)eta * xi, planeU = (size_t)eta * (xi - 1),
                 planeV = (size_t)(eta - 1) * xi;
    const size_t nU = sRho * planeU, nV = sRho * planeV, nW = sW * plane;
    const size_t raw = plane + nU + nV + 2 * nW;
    if ((rc = grow(ctx, ctx->dRomsRaw, ctx->romsRawCap, raw))) return rc;
    float *r = ctx->dRomsRaw;
    FrameSlot &s = ctx->slots[t];
    CUDA_TRY(ctx, cudaMemcpyAsync(r, zeta, plane * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(r + plane, u_faces, nU * sizeof(float), cudaMemcpyHostToDevice,
                                  ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(r + plane + nU, v_faces, nV * sizeof(float),
                                  cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(r + plane + nU + nV, w, nW * sizeof(float),
                                  cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(r + plane + nU + nV + nW, akt, nW * sizeof(float),
                                  cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->dErr, 0, sizeof(int), ctx->stream));
    RomsGrid G{ctx->dRomsMask, ctx->dRomsMask + plane, ctx->dRomsMask + plane + planeU,
               ctx->dRomsRot, eta, xi, sRho};
    RomsRecord R{r, r + plane, r + plane + nU, r + plane + nU + nV, r + plane + nU + nV + nW,
                 s.zeta, s.u, s.v, s.w, s.akt};
    CUDA_TRY(ctx, roms_record(G, R, ctx->dErr, ctx->stream));
    int err = 0;
    CUDA_TRY(ctx, cudaMemcpyAsync(&err, ctx->dErr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (err) {
        s.loaded = false;
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "%s",
                    (err & ROMS_ERR_FACE) ? "ROMS u or v is non-finite at a wet face"
                                          : "ROMS normalized velocity is outside finite float range");
    }
    return WACOMM_B200_OK;
}

}  // extern "C"

extern "C" {

int wacomm_b200_get_frame(wacomm_b200_context *ctx, int t, float *zeta, float *u, float *v,
                          float *w, float *akt) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    if (t < 0 || t >= (int)ctx->times.size())
        return fail(ctx, WACOMM_B200_ERR_ARGUMENT, "frame %d out of [0, %zu)", t, ctx->times.size());
    const FrameSlot &s = ctx->slots[t];
    if (!s.loaded) return fail(ctx, WACOMM_B200_ERR_STATE, "record %d is not loaded", t);
    cudaSetDevice(ctx->device);
    const size_t plane = (size_t)ctx->eta * ctx->xi;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->h2d));
    auto get = [&](float *dst, const float *src, size_t count) -> int {
        if (dst)
            CUDA_TRY(ctx, cudaMemcpyAsync(dst, src, count * sizeof(float), cudaMemcpyDeviceToHost,
                                          ctx->stream));
        return WACOMM_B200_OK;
    };
    int rc;
    if ((rc = get(zeta, s.zeta, plane))) return rc;
    if ((rc = get(u, s.u, plane * ctx->sRho))) return rc;
    if ((rc = get(v, s.v, plane * ctx->sRho))) return rc;
    if ((rc = get(w, s.w, plane * ctx->sW))) return rc;
    if ((rc = get(akt, s.akt, plane * ctx->sW))) return rc;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return WACOMM_B200_OK;
}

}  // extern "C"

extern "C" {

int wacomm_b200_particle_steps_total(wacomm_b200_context *ctx, int reset, double *total) {
    if (!ctx) return WACOMM_B200_ERR_ARGUMENT;
    cudaSetDevice(ctx->device);
    unsigned long long steps = 0;
    CUDA_TRY(ctx, cudaMemcpyAsync(&steps, ctx->dSteps + 1, sizeof(steps), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    if (reset) CUDA_TRY(ctx, cudaMemsetAsync(ctx->dSteps + 1, 0, sizeof(steps), ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (total) *total = (double)steps;
    return WACOMM_B200_OK;
}

}  // extern "C"
