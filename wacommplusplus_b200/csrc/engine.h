// Host-side declarations of the engine's kernel launchers (defined in the .cu units).
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "wacomm_b200.h"

namespace wb {

struct IntervalParams;
struct ParticleSoA;
struct MoveLaunch;
struct SurfPair;
struct EnvPair;

struct PackedArgs {
    int eta, xi, sW, sRho;
    const void *nodes;  // NodeRecord<storage>[sW][eta][xi]
    const SurfPair *surf;
    const EnvPair *env;
    bool hasWindU, hasWindV, hasStokes;
    const double *lonRad, *latRad, *depthIntervals;
    const double2 *metric;
    const float2 *invMetric;           // {1/xdist, 1/ydist} per cell (FP32 step)
    const float *depthIntervalsF;      // FP32 copy of depthIntervals (FP32 step)
    const wacomm_b200_config *cfgDevice;  // device copy of the run parameters (FP32 step, drift)
    const void *cells;                 // CellQuad<storage>[eta*xi][sW][2] (FP32 step)
    const void *cellSurface;           // CellSurface[eta*xi] (FP32 step)
};

// move_ref.cu (reference arithmetic, FP32 storage)
cudaError_t move_ref_dispatch(int semantics, const wacomm_b200_config &cfg,
                              const IntervalParams &P, const PackedArgs &A, const ParticleSoA &S,
                              const MoveLaunch &L, int blockSize, cudaStream_t stream);
// move_f32.cu (FP32 arithmetic, any storage)
cudaError_t move_f32_dispatch(int semantics, int storage, int shape, const wacomm_b200_config &cfg,
                              const IntervalParams &P, const PackedArgs &A, const ParticleSoA &S,
                              const MoveLaunch &L, cudaStream_t stream);

// support.cu ----------------------------------------------------------------------------

// Size in bytes of one node record of the packed pair.
size_t node_record_bytes(int storage);

struct FrameDevice {  // one forcing record in the reference layout (device)
    const float *zeta, *u, *v, *w, *akt;
    const float *windU, *windV, *stokesU, *stokesV;
};

cudaError_t pack_pair(int storage, int eta, int xi, int sW, const FrameDevice &f0,
                      const FrameDevice &f1, const double *h, void *nodes, SurfPair *surf,
                      EnvPair *env, cudaStream_t stream);

// Cell-column layout of the pair for the FP32 step (views.cuh): bytes per (cell, level) and per
// cell surface, and the packing kernel.
size_t cell_record_bytes(int storage);
size_t cell_surface_bytes();
cudaError_t pack_cells(int storage, int eta, int xi, int sW, const FrameDevice &f0,
                       const FrameDevice &f1, const double *h, void *cells, void *cellSurface,
                       cudaStream_t stream);

cudaError_t build_metric(int semantics, int eta, int xi, const double *lonRad,
                         const double *latRad, double2 *metric, float2 *invMetric,
                         cudaStream_t stream);

// Exclusive scan of n uint32 values; `temp` must hold scan_temp_words(n) words. The total is
// written to *total (device).
size_t scan_temp_words(size_t n);
cudaError_t exclusive_scan(const uint32_t *in, uint32_t *out, size_t n, uint32_t *total,
                           uint32_t *temp, cudaStream_t stream);

// Counting sort of particles by forcing cell: order[] receives particle slots grouped by cell.
// The records are visited in the sequence seq[n] (a permutation of the slots; null: slot order).
// keys/hist/offsets/temp are scratch: keys[n], hist[eta*xi+1], offsets[eta*xi+2].
cudaError_t sort_by_cell(const double *j, const double *i, int n, int eta, int xi,
                         const uint32_t *seq, uint32_t *keys, uint32_t *hist, uint32_t *offsets,
                         uint32_t *temp, uint32_t *order, cudaStream_t stream);

cudaError_t aos_to_soa(const wacomm_b200_particle *aos, int n, const ParticleSoA &S,
                       cudaStream_t stream);
cudaError_t soa_to_aos(const ParticleSoA &S, int n, wacomm_b200_particle *aos,
                       cudaStream_t stream);

// Stable removal of records with health <= 0: compacts S in place through `tmp` (a second SoA)
// and the scan scratch; writes the kept count to *kept (device).
cudaError_t compact_alive(const ParticleSoA &S, int n, const ParticleSoA &tmp, uint32_t *flags,
                          uint32_t *positions, uint32_t *temp, uint32_t *kept,
                          cudaStream_t stream);

// *total += *steps on the stream (the running particle-step count of a context).
cudaError_t accumulate_steps(const unsigned long long *steps, unsigned long long *total,
                             cudaStream_t stream);

cudaError_t count_concentration(const ParticleSoA &S, int n, int concTime, int sRho, int eta,
                                int xi, uint32_t *conc, cudaStream_t stream);

cudaError_t concentration_to_float(const uint32_t *conc, size_t n, int nTimes, int sRho, int eta,
                                   int xi, const double *mask, float *out, cudaStream_t stream);

// emission.cu ------------------------------------------------------------------------------

// Scratch for one emission of n sources (release schedules, counts, offsets, status).
size_t emission_scratch_bytes(int nSources);

// First pass: schedules, per-source counts and their offsets on the device; the total number of
// releases and an error word (bit 1: invalid schedule, bit 2: too many releases) are copied to
// the host (the call synchronizes the stream).
cudaError_t emission_plan(const wacomm_b200_source *sources, int nSources, double julianStart,
                          double intervalStart, double intervalEnd, void *scratch,
                          unsigned long long *totalHost, int *errHost, cudaStream_t stream);

// Second pass: writes the `total` releases in merged time order into S at slots base.. with ids
// firstId.. .
cudaError_t emission_fill(const wacomm_b200_source *sources, int nSources, const void *scratch,
                          unsigned long long total, const wacomm_b200_config *cfgDevice,
                          uint64_t firstId, const ParticleSoA &S, size_t base, cudaStream_t stream);

// kji2deplatlon of n records into device arrays.
cudaError_t geo_positions(const ParticleSoA &S, int n, int eta, int xi, int sW, const double *lon,
                          const double *lat, const double *h, const double *sWValues, double *dep,
                          double *latOut, double *lonOut, cudaStream_t stream);

// regrid.cu --------------------------------------------------------------------------------

// Error bits of the regridding kernels.
constexpr int REGRID_ERR_OUTSIDE = 1, REGRID_ERR_FIELD = 2, REGRID_ERR_FOLDED = 4,
              REGRID_ERR_TARGET = 8;

// A target's source cell (row-major index of its lower-left source node; -1: none) and weights.
struct RegridPlan {
    int node;
    double wx, wy;
};

// Rectilinear source: the longitude axis already unwrapped, `center` the midpoint of its ends.
struct RegridGeographic {
    const double *axisX, *axisY;
    int xi, eta;
    bool risingX, risingY;
    double center;
};

// Curvilinear source: coordinates [eta][xi], the per-cell boxes (minimumX, maximumX, minimumY,
// maximumY, shifted to the branch of `reference`) and the bins as offsets + cell lists.
struct RegridCurvilinear {
    const double *lon, *lat;
    const double4 *box;
    const int *binStart, *binCells;
    double minX, maxX, minY, maxY, reference;
    int binsX, binsY, xi, eta;
};

// A forcing time: source records k0 and k1 blended with weight alpha (k0 == k1: a copy).
struct RegridTime {
    int k0, k1;
    double alpha;
};

cudaError_t regrid_check_finite(const float *values, long long count, int *err,
                                cudaStream_t stream);
cudaError_t regrid_plan_geographic(const RegridGeographic &G, long long nTarget,
                                   const double *tLon, const double *tLat, RegridPlan *plan,
                                   int *err, cudaStream_t stream);
cudaError_t regrid_plan_curvilinear(const RegridCurvilinear &C, long long nTarget,
                                    const double *tLon, const double *tLat, RegridPlan *plan,
                                    int *err, cudaStream_t stream);
// outU/outV: nTimes planes of nTarget values each.
cudaError_t regrid_apply(bool curvilinear, const RegridPlan *plan, long long nTarget, int srcXi,
                         long long srcPlane, const float *srcU, const float *srcV,
                         const RegridTime *times, int nTimes, float *outU, float *outV,
                         cudaStream_t stream);

// roms.cu ----------------------------------------------------------------------------------

constexpr int ROMS_ERR_FACE = 1, ROMS_ERR_VELOCITY = 2;

// Grid part of the ROMS normalization: masks of rho nodes [eta][xi], u faces [eta][xi-1] and v
// faces [eta-1][xi] as 0/1 bytes; (cos, sin) of the grid angle per rho node, or null when the
// velocities are already east/north.
struct RomsGrid {
    const uint8_t *maskRho, *maskU, *maskV;
    const double2 *rotation;
    int eta, xi, sRho;
};

// One raw ROMS record (u [sRho][eta][xi-1], v [sRho][eta-1][xi], w/akt [sRho+1][eta][xi], zeta
// [eta][xi]) and the forcing record it becomes (u, v on the rho nodes).
struct RomsRecord {
    const float *zeta, *u, *v, *w, *akt;
    float *zetaOut, *uOut, *vOut, *wOut, *aktOut;
};

cudaError_t roms_record(const RomsGrid &G, const RomsRecord &R, int *err, cudaStream_t stream);

// surrogate.cu -----------------------------------------------------------------------------

// One surrogate interval: grid, interval, run parameters, the dry-node table, the per-cell layer-1
// sums and corner records, the packed weights and the fallback outputs.
struct SurrogateStep {
    int eta, xi, sW, sRho;
    double start, length;
    wacomm_b200_config cfg;
    int fallbackAll;
    const int *dry;
    const __half *z;
    const void *corners;  // per-cell-level corner records (surrogate_corner_bytes each)
    const uint8_t *weights;
    uint32_t *fallback, *fallbackCount;
    unsigned long long *runCount;
    float4 *rows;  // per work item (count): layer-4 sums and row tag, step kernel -> post kernel
    // Diffusive forward intervals: the surrogate's displacement spread over the substeps plus the
    // plain stochastic operator and closures of every substep (surrogate_walk_kernel), over the
    // cell-column pair of the FP32 step; otherwise the closed-form post kernel.
    int walk = 0;
    int semantics = 0, storage = 0;
    const IntervalParams *interval = nullptr;
    const void *cells = nullptr, *cellSurface = nullptr;
    const float2 *invMetric = nullptr;
    const float *depthF = nullptr;
    cudaEvent_t midEvent = nullptr;  // recorded between the step kernel and the post/walk kernel
    const uint32_t *walkOrder = nullptr;  // cell order of the walk kernel's work (null: slot order)
    float maxError = INFINITY;  // trust limit of the prediction, metres per interval (off: INFINITY)
};

// Kernel attributes of the tensor-core kernels (once per device; outside stream capture).
cudaError_t surrogate_prepare();
size_t surrogate_packed_bytes();
size_t surrogate_corner_bytes();
size_t surrogate_parameter_count();
// Packs the flat FP32 parameters (w1 [256][388], b1, w2 [256][256], b2, w3, b3, w4 [3][256], b4)
// into the device image: BF16 swizzled K-blocks of the GEMM weights, FP32 vectors.
void surrogate_pack(const float *flat, uint8_t *out);
long long surrogate_cell_levels(int eta, int xi, int sW);
cudaError_t surrogate_cells(int eta, int xi, int sW, int sRho, const FrameDevice &f0,
                            const FrameDevice &f1, const double *h, const double *depthIntervals,
                            const double2 *metric, const uint8_t *weights, __half *z, void *corners,
                            int *err, int smCount, cudaStream_t stream);
// The step kernel (layers 1-4 of every work item into s.rows) and the post kernel (displacement,
// closures, state, concentration, fallback list) or, for diffusive intervals, the walk kernel
// (displacement with the plain stochastic operator per substep): two launches.
cudaError_t surrogate_step(const SurrogateStep &s, const ParticleSoA &S, const MoveLaunch &L,
                           int smCount, cudaStream_t stream);
// Inclusive 2-D prefix sums [(eta+1)][(xi+1)] of nodes with mask 0 or h <= shore.
cudaError_t surrogate_dry_prefix(const double *mask, const double *h, double shore, int eta, int xi,
                                 int *pre, cudaStream_t stream);

// mlp_train.cu ----------------------------------------------------------------------------
size_t mlp_train_work_floats(int batch);
cudaError_t mlp_train_step(const float *stencil, const float *particle, const float *gate,
                           const float *target, int batch, float *params, float *grads, float *m,
                           float *v, float *work, float *loss, int step, float lr, bool update,
                           cudaStream_t stream);

// history.cu ------------------------------------------------------------------------------

// Text restart of n host records (Particles.cpp:28-55) / the records of a text restart
// (Particles.cpp:320-364); WACOMM_B200_ERR_IO with wacomm_b200_file_error() on failure.
int history_text_write(const char *path, const wacomm_b200_particle *records, size_t n);
int history_text_read(const char *path, std::vector<wacomm_b200_particle> &records);

// NetCDF history: the CDF-5 header for `kept` records, the file (header, particle_time, payload)
// and a restart read with the reference's checks.
std::string history_header_for(const wacomm_b200_history_meta &m, int backward, uint64_t seed,
                               size_t kept);
int history_netcdf_write(const char *path, const std::string &header, double particleTime,
                         const uint8_t *payload, size_t payloadBytes);
int history_netcdf_read(const char *path, const wacomm_b200_restart_expect &expect,
                        std::vector<wacomm_b200_particle> &records, double &checkpoint,
                        bool &hasCheckpoint);

// Device side: flags of the stored records (given kji2deplatlon's dep/lat/lon), and the payload of
// the `kept` records at their scan positions (88 bytes per record, big-endian, file order).
size_t history_payload_bytes(size_t kept);
cudaError_t history_select(const ParticleSoA &S, int n, const double *dep, const double *lat,
                           const double *lon, uint32_t *flags, cudaStream_t stream);
cudaError_t history_pack(const ParticleSoA &S, int n, const uint32_t *flags,
                         const uint32_t *positions, const double *dep, const double *lat,
                         const double *lon, size_t kept, uint8_t *payload, cudaStream_t stream);

// dropin.cu -------------------------------------------------------------------------------
int dropin_move(const wacomm_b200_config *config, wacomm_b200_particle *particles, int timeIndex,
                int oceanTime, int sW, int sRho, int eta, int xi, const double *times,
                const double *lonRad, const double *latRad, const double *depthIntervals,
                const double *h, const float *zeta, const float *u, const float *v,
                const float *w, const float *akt, const float *windU, const float *windV,
                const float *stokesU, const float *stokesV, int count, cudaStream_t stream);

}  // namespace wb
