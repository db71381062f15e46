/*
 * wacomm_b200 -- B200-native particle-move engine for WaComM++: the C ABI.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, returns an int status
 * (WACOMM_B200_OK = 0) and never exits the process; wacomm_b200_last_error() returns the
 * message of the last failure on a context. Host pointers are owned by the caller; device
 * memory is owned by the context. A context is bound to one CUDA device and is not
 * re-entrant: calls from several host threads must be serialized by the caller.
 *
 * The reference interfaces replaced here:
 *   - the CPU step Particle::move(config_data*, ...)            Particle.hpp:54-58, Particle.cpp:71-824
 *   - the GPU launcher cudaMoveParticle(...)                   cuda/kernel.h:7, kernel.cu:370-382
 *   - the per-interval device staging of Wacomm::run           Wacomm.cpp:386-610
 *   - dead-particle removal                                     Wacomm.cpp:711-713
 *   - Concentration::evaluate(...) and the land mask            Concentration.hpp:16-44, Wacomm.cpp:722-739
 *   - sourceEmissionTimes / Source::emit / Sources::emit        SourceEmission.hpp:38-79, Source.cpp:16-45,
 *                                                               Sources.cpp:233-249 (wacomm_b200_emit)
 *   - OceanModelAdapter::kji2deplatlon                          OceanModelAdapter.cpp:271-327
 *                                                               (wacomm_b200_geo_positions)
 *   - the record normalization of ROMSAdapter::process          OceanModelAdapters/ROMSAdapter.cpp:228-462
 *                                                               (wacomm_b200_upload_roms_frame)
 *   - EnvironmentalRegridder::bilinearGeographic /              EnvironmentalRegridder.cpp:239-334,
 *     bilinearCurvilinearGeographic of wind and Stokes fields   WacommPlusPlus.cpp:162-173
 *                                                               (wacomm_b200_regrid_environment)
 * The drop-in C++ launcher with the reference's exact signature is declared in
 * include/wacomm_b200_kernel.h.
 */
#ifndef WACOMM_B200_H
#define WACOMM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
#define WACOMM_B200_BOOL bool
extern "C" {
#else
#define WACOMM_B200_BOOL _Bool
#endif

/* ------------------------------------------------------------------ status codes */
#define WACOMM_B200_OK 0
#define WACOMM_B200_ERR_ARGUMENT 1     /* a null pointer, a size or an option out of range */
#define WACOMM_B200_ERR_CUDA 2         /* a CUDA runtime call failed */
#define WACOMM_B200_ERR_STATE 3        /* a call out of order (no grid, frame missing ...) */
#define WACOMM_B200_ERR_DRIFT_OBJECT 4 /* a particle names a drift object outside the catalogue */
#define WACOMM_B200_ERR_CAPACITY 5     /* a size above a documented maximum */
#define WACOMM_B200_ERR_IO 6           /* a file could not be opened, written, read or parsed, or a
                                          restart does not match the run (the message says which) */

/* ------------------------------------------------------------------ records */

/* Byte-for-byte the reference particle_data (Particle.hpp:31-41), 64 bytes. */
typedef struct wacomm_b200_particle {
    uint64_t id;
    double k, j, i;
    double health, age, time;
    uint16_t driftObjectType;
    int8_t driftSide;
} wacomm_b200_particle;

typedef struct wacomm_b200_calibration_region {
    double west, south, east, north;
    double windErrorStdDev, windErrorComponentCorrelation;
    double windErrorSpatialScale, windErrorTemporalScale;
} wacomm_b200_calibration_region;

/* Byte-for-byte the reference config_data (Config.hpp:36-72), 1248 bytes. */
typedef struct wacomm_b200_config {
    WACOMM_B200_BOOL random;
    WACOMM_B200_BOOL randomSources;
    double deltat, dti, survprob, tau0, sv, crid, sigma, shoreLimit;
    int upperClosure, lowerClosure, horizontalClosure;
    uint64_t randomSeed;
    int trackingDirection, backwardDiffusion, integrator;
    double restartCheckpoint;
    int driftModel;
    WACOMM_B200_BOOL leewayCoefficientEnsemble;
    double leewayResidualCorrelation;
    WACOMM_B200_BOOL leewayRandomSide;
    double leewayRightSideProbability, leewayJibeProbabilityHourly;
    double windErrorStdDev, windErrorComponentCorrelation;
    double windErrorSpatialScale, windErrorTemporalScale;
    uint32_t observationalCalibrationRegionCount;
    wacomm_b200_calibration_region observationalCalibrationRegions[16];
    uint16_t driftObjectType;
    int8_t driftSide;
    WACOMM_B200_BOOL hasWind;
    double windU10, windV10;
} wacomm_b200_config;

/* A release point (the fields of Source, Source.hpp:19-60). k, j, i are grid indices; start and
 * end are days as the reference stores them (start < 0: the run start; end < 0: no end); mode is
 * the source's own mode field, and only mode 1 emits (Source.cpp:18). */
#define WACOMM_B200_EMISSION_UNIFORM_RATE 0           /* emission_value particles per hour */
#define WACOMM_B200_EMISSION_FORCING_INTERVAL_BATCH 1 /* emission_value particles per record */
#define WACOMM_B200_EMISSION_SINGLE_PULSE 2           /* emission_value particles once, at start */

typedef struct wacomm_b200_source {
    double k, j, i;
    double start, end;
    double emission_value;
    int32_t emission_mode; /* WACOMM_B200_EMISSION_* */
    int32_t mode;
} wacomm_b200_source;

/* ------------------------------------------------------------------ engine options */

#define WACOMM_B200_SEMANTICS_HOST 0   /* Particle::move rules (Particle.cpp:71-824), the default */
#define WACOMM_B200_SEMANTICS_DEVICE 1 /* reference kernel rules (kernel.cu:153-368) */

#define WACOMM_B200_ARITH_REFERENCE 0  /* FP64 with the reference's float roundings (parity mode) */
#define WACOMM_B200_ARITH_FP32 1       /* FP32 interpolation, FP64 position and time weight */

#define WACOMM_B200_STORAGE_FP32 0     /* forcing pair stored as float */
#define WACOMM_B200_STORAGE_FP16 1     /* forcing pair stored as half (requires ARITH_FP32) */
#define WACOMM_B200_STORAGE_BF16 2     /* forcing pair stored as bfloat16 (requires ARITH_FP32) */

#define WACOMM_B200_RNG_REFERENCE 0    /* ordered-splitmix64-v2 draws, draw-for-draw with the reference */
#define WACOMM_B200_RNG_PHILOX 1       /* Philox4x32-10 keyed on (particle id, interval, step time) */

#define WACOMM_B200_LAUNCH_SHAPE_AUTO (-1) /* launch_shape by compiled form: 3 for the deterministic
                                              form without drift (96 registers, no spills), 2 for
                                              the others; the default */

typedef struct wacomm_b200_options {
    int semantics;            /* WACOMM_B200_SEMANTICS_* */
    int arithmetic;           /* WACOMM_B200_ARITH_* */
    int storage;              /* WACOMM_B200_STORAGE_* */
    int rng;                  /* WACOMM_B200_RNG_* */
    int block_size;           /* threads per block of the move kernel: 64..1024, multiple of 32 */
    int substeps_per_launch;  /* 0: one launch per interval; else launches of this many dti */
    int sort_by_cell;         /* N >= 1: order the work by forcing cell, sorting the resident
                                 population every N-th interval (the intervals between take the
                                 last sort's order); 1 (the default): every interval; 0: never;
                                 at most 64; wacomm_b200_autotune chooses 1, 2 or 4 */
    int fuse_concentration;   /* 1: count the concentration in the move kernel's epilogue */
    int launch_shape;         /* FP32 step: 0 = 256 threads, registers unbounded; 1 = 128 threads,
                                 3 blocks/SM; 2 = 256 threads, 2 blocks/SM; 3 = 128 threads,
                                 5 blocks/SM (fewer registers, more resident warps);
                                 WACOMM_B200_LAUNCH_SHAPE_AUTO (default): 3 or 2 by form */
    int surrogate;            /* 1: forward intervals by the learned surrogate
                                 (wacomm_b200_set_surrogate), with the plain stochastic operator
                                 per substep when the random walk is on; the rest by the FP32 step */
    int particles_per_thread; /* FP32 step: work items per thread, 1..16 (default 1): the grid
                                 shrinks by this factor and each block strides over it, taking
                                 consecutive blocks of work items in turn; results do not depend
                                 on it; wacomm_b200_autotune chooses 1, 2 or 4 */
} wacomm_b200_options;

/* ------------------------------------------------------------------ context */

typedef struct wacomm_b200_context wacomm_b200_context;

/* Library version string; usable without a GPU. */
const char *wacomm_b200_version(void);
/* Number of CUDA devices visible (0 when none); never fails. */
int wacomm_b200_device_count(void);

int wacomm_b200_context_create(int device, wacomm_b200_context **out);
int wacomm_b200_context_destroy(wacomm_b200_context *ctx);
const char *wacomm_b200_last_error(const wacomm_b200_context *ctx);

/* Fills *out with the defaults: host semantics, FP32 arithmetic and storage, reference RNG,
 * 256 threads, one launch per interval, cell sort on, fused concentration on, launch shape 2,
 * surrogate off. */
int wacomm_b200_default_options(wacomm_b200_options *out);
int wacomm_b200_set_options(wacomm_b200_context *ctx, const wacomm_b200_options *options);
int wacomm_b200_get_options(const wacomm_b200_context *ctx, wacomm_b200_options *out);

/* Run parameters (the reference's config_data, copied). */
int wacomm_b200_set_config(wacomm_b200_context *ctx, const wacomm_b200_config *config);

/* Static grid (the oceanmodel_data fields, OceanModelAdapter.hpp:20-34), host arrays [eta][xi];
 * depth_intervals has s_w-1 entries indexed kI+s_w-2 (WacommAdapter.cpp:101-103); s_w = s_rho+1.
 * mask may be NULL (used only by the concentration land mask). */
int wacomm_b200_set_grid(wacomm_b200_context *ctx, int eta, int xi, int s_rho, int s_w,
                         const double *mask, const double *lon_rad, const double *lat_rad,
                         const double *h, const double *depth_intervals);

/* Times of the forcing records (seconds; oceanTime). Allocates one device frame slot per time. */
int wacomm_b200_set_times(wacomm_b200_context *ctx, int n_times, const double *ocean_time);

/* Uploads forcing record t (host arrays in the reference layout: zeta [eta][xi],
 * u,v [s_rho][eta][xi], w,akt [s_w][eta][xi], level 0 at the bottom). wind/stokes are optional
 * [eta][xi] fields on the ocean grid and times (Wacomm.cpp:70-84); pass NULL when absent. Frames
 * persist on the device until overwritten, so each record crosses PCIe once. */
int wacomm_b200_upload_frame(wacomm_b200_context *ctx, int t, const float *zeta, const float *u,
                             const float *v, const float *w, const float *akt,
                             const float *wind_u10, const float *wind_v10, const float *stokes_u,
                             const float *stokes_v);

/* The same upload without waiting: the copies run on the context's copy stream, after the kernels
 * already enqueued on its compute stream (which may still read record t), and the next interval
 * that uses record t waits for them on the device. The host arrays must stay unchanged until the
 * copies have completed (wacomm_b200_synchronize); from page-locked memory the call returns at
 * once, so the next record crosses PCIe while the current interval computes (the reference
 * re-uploads its whole window each interval, Wacomm.cpp:424-477). */
int wacomm_b200_upload_frame_async(wacomm_b200_context *ctx, int t, const float *zeta,
                                   const float *u, const float *v, const float *w,
                                   const float *akt, const float *wind_u10,
                                   const float *wind_v10, const float *stokes_u,
                                   const float *stokes_v);

/* ROMS records as the model writes them, normalized on the device into forcing records: the
 * per-record part of ROMSAdapter::process (OceanModelAdapters/ROMSAdapter.cpp:228-306) with
 * uv2rho (:309-368) and wakt2wakt (:431-462). set_roms_grid takes the u-face mask [eta][xi-1], the
 * v-face mask [eta-1][xi] and the grid angle [eta][xi] in radians (NULL when u/v are already
 * east/north), on the grid of set_grid, whose mask is the rho mask (required); masks must hold 0
 * or 1 and the angle must be finite on wet nodes (the reference's checks, :139-160).
 * upload_roms_frame stages record t from u on u faces [s_rho][eta][xi-1], v on v faces
 * [s_rho][eta-1][xi], w and AKt [s_w][eta][xi] and zeta [eta][xi] (the adapter's own array
 * orders): zeta is zeroed on land and at fill values >= 1e36, u/v are averaged from the wet faces
 * to the rho nodes and rotated to east/north in double, w/AKt are zeroed on land. A non-finite u/v
 * on a wet face or a rotated velocity outside the float range is an error, as in the reference
 * (the record is then not loaded). Wind and Stokes as in upload_frame. Synchronous. The grid-only
 * part of process (h and zeta zeroed on land, lon/lat to radians, depth intervals) belongs to the
 * set_grid arguments. */
/* Copies the ocean fields of loaded record t back to host arrays in the upload_frame layout (any
 * pointer may be NULL): the processed input the reference saves with SaveInput
 * (WacommPlusPlus.cpp:204-216). */
int wacomm_b200_get_frame(wacomm_b200_context *ctx, int t, float *zeta, float *u, float *v,
                          float *w, float *akt);
int wacomm_b200_set_roms_grid(wacomm_b200_context *ctx, const double *mask_u,
                              const double *mask_v, const double *angle);
int wacomm_b200_upload_roms_frame(wacomm_b200_context *ctx, int t, const float *zeta,
                                  const float *u_faces, const float *v_faces, const float *w,
                                  const float *akt, const float *wind_u10,
                                  const float *wind_v10, const float *stokes_u,
                                  const float *stokes_v);

/* Particle records in and out (reference particle_data layout, host memory). set replaces the
 * resident set, append adds after it, get copies the resident records (in their order) into
 * out (capacity n), and count reports how many are resident. */
int wacomm_b200_set_particles(wacomm_b200_context *ctx, const wacomm_b200_particle *host,
                              size_t n);
int wacomm_b200_append_particles(wacomm_b200_context *ctx, const wacomm_b200_particle *host,
                                 size_t n);
int wacomm_b200_get_particles(wacomm_b200_context *ctx, wacomm_b200_particle *out, size_t n);
int wacomm_b200_particle_count(const wacomm_b200_context *ctx, size_t *out);

/* Moves every resident particle over the forcing interval that starts at record time_index in
 * the configured tracking direction (Particle.cpp:109-120), asynchronously on the context's
 * stream. When fuse_concentration is on, alive particles are also counted into the
 * concentration grid at time index time_index + direction (Wacomm.cpp:713-722). */
int wacomm_b200_move_interval(wacomm_b200_context *ctx, int time_index);

/* A run of n_intervals intervals from first_time_index on, in the tracking direction, recorded
 * once as a CUDA graph (pair packing, cell sort, move and fused count of every interval) and
 * launched as one unit by wacomm_b200_graph_launch; the solver's per-interval loop
 * (Wacomm.cpp:386-739) becomes one host call. Every buffer is sized before the capture. The graph
 * holds the particle count, the buffer addresses, the forcing times, the config and the options
 * of the capture: new record values (upload_frame into existing slots, set_particles with the
 * same count, a new batch of scenarios) are picked up by the next launch, while any change of
 * those is refused at launch with WACOMM_B200_ERR_STATE (capture again). With the surrogate option
 * the per-cell layer 1, the tensor-core step, the displacement (or walk) kernel and the fallback
 * step of every interval are captured as well (the fallback step reads its list length on the
 * device); last_surrogate_stats then gives the counts of the last captured interval, without
 * kernel times. last_interval_stats after a launch reports the whole run (device ms,
 * particle-steps). No reference counterpart. */
int wacomm_b200_graph_capture(wacomm_b200_context *ctx, int first_time_index, int n_intervals);
int wacomm_b200_graph_launch(wacomm_b200_context *ctx);
int wacomm_b200_graph_release(wacomm_b200_context *ctx);

/* Times the interval at time_index once per launch configuration of the move kernel (FP32
 * arithmetic: launch_shape 0..3; reference arithmetic: block_size 64, 128, 192, 256), each from
 * the same resident records and concentration after a warm-up pass, keeps the fastest in the
 * options and restores records and concentration: only the options change. Writes the chosen
 * value and its device ms. With FP32 arithmetic it then times the interval with 1, 2 and 4
 * work items per thread at the chosen shape and keeps the fastest in
 * options.particles_per_thread. With the cell sort on and four intervals from time_index inside
 * the forcing window, it then times those four intervals from the same snapshot sorting every
 * 1, 2 or 4 of them and keeps the fastest cadence in options.sort_by_cell. No reference
 * counterpart. */
int wacomm_b200_autotune(wacomm_b200_context *ctx, int time_index, int *best, float *best_ms);

/* The same interval through host buffers: uploads n records from `particles` (pinned or
 * pageable host memory), moves them, and writes them back in place. Copies are pipelined
 * against the kernels in slabs; the resident set is replaced by these records. */
int wacomm_b200_move_interval_host(wacomm_b200_context *ctx, int time_index,
                                   wacomm_b200_particle *particles, size_t n);

/* Stable removal of records with health <= 0 (Wacomm.cpp:711-713). */
int wacomm_b200_remove_dead(wacomm_b200_context *ctx);

/* Emission of one interval on the device (Sources::emit, Sources.cpp:233-249): the release times
 * of every source in [interval_start, interval_end) seconds (sourceEmissionTimes,
 * SourceEmission.hpp:38-79, with source times start*86400 s, or julian_start*86400 s when start
 * < 0), merged across sources in time order with ties kept in source order, are appended to the
 * resident records in that order. Ids continue from the last resident record's id + 1 (0 when
 * none); positions take the seeded 0.25 N(0,1) index offsets when randomSources is set; type and
 * side follow the run parameters, the side drawn per id when leewayRandomSide is set
 * (Source.cpp:25-45). An invalid schedule (a non-finite or negative value, an empty interval, a
 * fractional count for the batch modes) returns WACOMM_B200_ERR_ARGUMENT and appends nothing.
 * *emitted (may be NULL) receives the number appended. Requires set_config. */
int wacomm_b200_emit(wacomm_b200_context *ctx, const wacomm_b200_source *sources, int n_sources,
                     double julian_start, double interval_start, double interval_end,
                     size_t *emitted);

/* The output grid of kji2deplatlon (OceanModelAdapter.hpp:20-34): lon and lat [eta][xi] (degrees
 * in the reference) and the s_w coordinate values (s_w entries, level 0 at the bottom), on the
 * grid of the last set_grid. */
int wacomm_b200_set_geo_grid(wacomm_b200_context *ctx, const double *lon, const double *lat,
                             const double *s_w_values);

/* Geographic position of every resident record (OceanModelAdapter::kji2deplatlon,
 * OceanModelAdapter.cpp:271-327) into host arrays of capacity n: depth in metres (negative
 * down) and lat/lon interpolated from the set_geo_grid arrays; 1e37 in all three for a record
 * outside the grid or its valid levels. Requires set_grid and set_geo_grid. */
int wacomm_b200_geo_positions(wacomm_b200_context *ctx, double *depth, double *lat, double *lon,
                              size_t n);

/* Wind (10 m) and Stokes drift fields on their own grids and times, regridded on the device to the
 * rho nodes of set_geo_grid and aligned to the set_times forcing times. Replaces the host
 * regridding the reference runs before its move loop (WacommPlusPlus.cpp:162-173, reaching
 * EnvironmentalRegridder::bilinearGeographic / bilinearCurvilinearGeographic,
 * EnvironmentalRegridder.cpp:239-334) and its same-grid, same-times requirement
 * (Wacomm.cpp:70-84).
 *   method GEOGRAPHIC: rectilinear source (lon depends on i only, lat on j only, 1e-10);
 *   method CURVILINEAR: any non-folded source grid, each target found by Newton inversion in the
 *   reference's cell index.
 * src_lon/src_lat [src_eta][src_xi] degrees; u, v [src_times][src_eta][src_xi]; times
 * [src_times] seconds, strictly increasing. A forcing time equal to a source time (1e-6 s) takes
 * that record; one between two source times blends the two regridded values linearly in time
 * (no reference counterpart: the reference requires equal times). Errors, as the reference
 * throws: a target outside the source grid or times (no extrapolation), a non-rectilinear
 * source for GEOGRAPHIC, a folded cell holding a target, non-finite values; also longitudes more
 * than 3600 degrees apart, where the reference's wrapping loop would not end. On error the field
 * is left unset. The regridded fields stay resident ([T][eta][xi] float per component) and feed
 * every interval whose records were uploaded without that field; an upload with the field takes
 * precedence for its record. Synchronous. */
#define WACOMM_B200_FIELD_WIND 0
#define WACOMM_B200_FIELD_STOKES 1
#define WACOMM_B200_REGRID_BILINEAR_GEOGRAPHIC 0
#define WACOMM_B200_REGRID_BILINEAR_CURVILINEAR_GEOGRAPHIC 1
int wacomm_b200_regrid_environment(wacomm_b200_context *ctx, int field, int method, int src_eta,
                                   int src_xi, const double *src_lon, const double *src_lat,
                                   int src_times, const double *times, const float *u,
                                   const float *v);

/* Drops a regridded field (wind or Stokes). */
int wacomm_b200_clear_environment(wacomm_b200_context *ctx, int field);

/* Copies forcing time t of a regridded field into host arrays of eta*xi values. */
int wacomm_b200_get_environment(wacomm_b200_context *ctx, int field, int t, float *u, float *v);

/* Concentration grid of n_conc_times records [n_conc_times][s_rho][eta][xi] as uint32 counts.
 * reset zeroes it; count adds the resident alive particles at conc_time_index
 * (Concentration.hpp:16-44); get copies it out (uint32) and get_float copies it as the reference
 * float grid, writing 1e37 into land cells (mask != 1) of every level when mask_land is set, in
 * the concentration times counted since the last reset (the solver masks each time it evaluates;
 * times never counted stay 0, Wacomm.cpp:174-196,722-739). */
int wacomm_b200_concentration_reset(wacomm_b200_context *ctx, int n_conc_times);
int wacomm_b200_concentration_count(wacomm_b200_context *ctx, int conc_time_index);
int wacomm_b200_concentration_get(wacomm_b200_context *ctx, uint32_t *out, size_t n);
int wacomm_b200_concentration_get_float(wacomm_b200_context *ctx, float *out, size_t n,
                                        int mask_land);

/* The device address of the context's uint32 concentration grid and its cell count, so that
 * particle shards held by several contexts (one per GPU) can sum their grids with a collective of
 * the caller's (the counts add modulo 2^32, so a signed 32-bit sum gives the same bits). The
 * memory stays owned by the context and valid until the next concentration_reset or destroy; the
 * context's stream (wacomm_b200_stream) orders the kernels that write it. */
int wacomm_b200_concentration_device(wacomm_b200_context *ctx, void **device_ptr, size_t *cells);

int wacomm_b200_synchronize(wacomm_b200_context *ctx);

/* Particle-steps of every interval (and captured run) since the context was created or the last
 * reset, counted by the kernels and summed on the device, so a caller can enqueue many intervals
 * without waiting between them and read the count once. Waits for the context's stream. */
int wacomm_b200_particle_steps_total(wacomm_b200_context *ctx, int reset, double *total);

/* Statistics of the last move_interval: device milliseconds of all its kernels (CUDA events on
 * the context stream around pack, sort and move), of the move kernel launches alone, how many
 * kernels it launched and how many particle-steps (substeps of active particles) it took. */
/* Device milliseconds of the dominant kernels of the eager intervals enqueued since the last call
 * (at most the last 256; captured runs are not included), oldest first, three values per
 * interval: plain step [move kernel, 0, 0]; surrogate [step kernel (tensor cores), post or walk
 * kernel, fallback step]. Events are recorded around the kernels of every interval, so intervals
 * enqueued back to back are timed without a host wait; this call waits for the stream. Writes at
 * most `capacity` intervals (3 * capacity floats), the newest ones, and their number to *count.
 * No reference counterpart. */
int wacomm_b200_kernel_times(wacomm_b200_context *ctx, float *ms, int capacity, int *count);

int wacomm_b200_last_interval_stats(const wacomm_b200_context *ctx, float *device_ms,
                                    float *move_ms, int *kernel_launches, double *particle_steps);

/* No counterpart in the reference: the learned one-interval advection surrogate. parameters holds
 * count = 231,939 FP32 values: w1 [256][388] (inputs: the 4x4x4 u, v, w stencil at both records,
 * then jF, iF, kF and the activation fraction), b1 [256], w2 [256][256], b2, w3 [256][256], b3,
 * w4 [3][256], b4 [3]. With the surrogate option on, move_interval moves each active particle of
 * a forward interval by one MLP evaluation (BF16 tensor-core GEMMs). Deterministic intervals
 * apply the displacement with the closures in closed form (paths near dry nodes use the FP32
 * step); with the random walk on, the displacement is spread evenly over the substeps and the
 * plain stochastic operator (Particle.cpp:518-533), the vertical cap and the closures run every
 * substep. Backward tracking, drifting objects, jibing, restart-clipped intervals and starts
 * outside the valid cells use the FP32 step. */
int wacomm_b200_set_surrogate(wacomm_b200_context *ctx, const float *parameters, size_t count);

/* No counterpart in the reference. A trust limit for the surrogate, in metres per interval: a
 * particle whose estimated one-interval error exceeds it goes to the FP32 step instead. The
 * estimate is the start-point method's error |grad u| |u| t^2 / 2 over the remaining time t, with
 * the velocity gradient taken from the RMS deviation of the particle's 4x4x4 stencil over 1.5
 * cells; a uniform stencil always stays with the surrogate (its start-point displacement is
 * exact there). metres > 0; INFINITY (the default) turns the limit off. */
int wacomm_b200_set_surrogate_error_limit(wacomm_b200_context *ctx, double metres);

/* Of the last move_interval with the surrogate on: particles it moved, particles handed to the
 * FP32 step, and device milliseconds of the per-cell layer-1 kernel and of the particle kernel. */
int wacomm_b200_last_surrogate_stats(const wacomm_b200_context *ctx, size_t *run, size_t *fallback,
                                     float *cell_ms, float *step_ms);

/* The CUDA stream (cudaStream_t) the context launches on, for callers that order their own work
 * or events against it. */
int wacomm_b200_stream(const wacomm_b200_context *ctx, void **out);

/* ------------------------------------------------------------------ device-pointer entry */

/* The reference GPU launcher (kernel.cu:370-382) behind a C name: every pointer is a device
 * pointer owned by the caller, particles (AoS particle_data) are updated in place,
 * the call is asynchronous on `stream` (a cudaStream_t, NULL = legacy default stream) and returns
 * the CUDA error code of the launch (0 = cudaSuccess). mask, num_thread and num_gpu are ignored
 * like the reference does; wind/stokes may be NULL. Device semantics, reference arithmetic.
 * The records are moved in horizontal-cell order (key, histogram, scan, scatter; the order
 * changes no result) with working memory taken from the device's memory pool on `stream`
 * (cudaMallocAsync, about 8 B per record + 8 B per cell, released with cudaFreeAsync); when the
 * pool has none, the records are moved in caller order. */
int wacomm_b200_cuda_move_particle(const wacomm_b200_config *config_device,
                                   wacomm_b200_particle *particles_device, int time_index,
                                   int ocean_time, int s_w, int s_rho, int eta, int xi,
                                   const double *times, const double *mask,
                                   const double *lon_rad, const double *lat_rad,
                                   const double *depth_intervals, const double *h,
                                   const float *zeta, const float *u, const float *v,
                                   const float *w, const float *akt, const float *wind_u10,
                                   const float *wind_v10, const float *stokes_u,
                                   const float *stokes_v, int particle_count, int num_thread,
                                   int num_gpu, void *stream);

/* No counterpart in the reference. The launcher above for callers that may not allocate device
 * memory: cudaFree synchronizes the whole device (and cudaMalloc may), stalling every other
 * stream a multi-stream or multi-GPU driver keeps in flight, and some host frameworks own all
 * device memory through their own pool. Same arguments, meaning and results as
 * wacomm_b200_cuda_move_particle, whose horizontal-cell ordering it shares, but its working
 * memory (keys, histogram, scan, order) is a fixed array of about 25 MB compiled into the library
 * and held on every GPU that loads it. Limits: particle_count <= 2,097,152 and eta*xi <=
 * 1,048,576 (eta*xi counts only on grids with at least two nodes along each axis; narrower grids
 * have no interpolation cell and their records are moved in caller order, as the launcher above
 * does); larger calls return -WACOMM_B200_ERR_CAPACITY and do nothing. Otherwise returns 0 or a
 * CUDA error code. Every call on a device shares the array: calls that overlap on the GPU race and
 * must not be issued; calls on one stream are ordered and safe. The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress, with that device current) and the SM
 * count; under lazy module loading (the CUDA default) it is also the call that loads the library's
 * kernels and makes the array resident on that device, which allocates and synchronizes once.
 * Make that first call during set-up, before the allocation-free phase and before any stream
 * capture begins. The address belongs to the device's context of that moment: a cudaDeviceReset
 * between calls is not supported. */
int wacomm_b200_cuda_move_particle_noalloc(const wacomm_b200_config *config_device,
                                           wacomm_b200_particle *particles_device, int time_index,
                                           int ocean_time, int s_w, int s_rho, int eta, int xi,
                                           const double *times, const double *mask,
                                           const double *lon_rad, const double *lat_rad,
                                           const double *depth_intervals, const double *h,
                                           const float *zeta, const float *u, const float *v,
                                           const float *w, const float *akt,
                                           const float *wind_u10, const float *wind_v10,
                                           const float *stokes_u, const float *stokes_v,
                                           int particle_count, int num_thread, int num_gpu,
                                           void *stream);

/* ------------------------------------------------------------------ surrogate training */

/* Scratch floats of wacomm_b200_mlp_train_step for a batch. */
size_t wacomm_b200_mlp_train_work_floats(int batch);

/* One training step of the surrogate MLP with the library's own kernels: forward pass
 * (388 -> 256 -> 256 -> 256 -> 3, GELU tanh form, outputs times the gate), mean-squared loss of
 * the gated outputs against the targets (over batch x 3), backward pass of all four layers into
 * grads, then, with update != 0, an Adam step (beta1 0.9, beta2 0.999, eps 1e-8, bias correction
 * at `step` >= 1) of params with moments m, v. The products of layers 1-3 and every weight
 * gradient run on the tcgen05 tensor cores with BF16 operands and FP32 accumulation; the weight
 * gradients reduce the batch in a fixed order, so a step is reproducible bit for bit. Device
 * pointers, asynchronous on `stream`: stencil [batch][384], particle [batch][4], gate [batch],
 * target [batch][3]; params, grads, m, v: the flat parameter layout of wacomm_b200_set_surrogate;
 * work: mlp_train_work_floats(batch) floats, whose first 32-bit word is set nonzero when a
 * tensor-core kernel gave up on a bounded wait (the step's results are then not valid); loss: one
 * float. Returns 0, WACOMM_B200_ERR_ARGUMENT or WACOMM_B200_ERR_CUDA. */
int wacomm_b200_mlp_train_step(const float *stencil, const float *particle, const float *gate,
                               const float *target, int batch, float *params, float *grads,
                               float *m, float *v, float *work, float *loss, int step, float lr,
                               int update, void *stream);

/* ------------------------------------------------------------------ history and restart files */

/* Text restart (Particles::saveAsTxt, Particles.cpp:28-55): a "\t<count>" line, then one line per
 * record: id i j k health age time object side, the reals with 17 significant digits (printf
 * "%.17g", what the reference's ostream with setprecision(max_digits10) prints), the drift object
 * and side as integers. Host records; formatted on all host threads. */
int wacomm_b200_text_write(const char *path, const wacomm_b200_particle *records, size_t n);

/* Reads a text restart (Particles::loadFromTxt, Particles.cpp:320-364): the first line is
 * skipped; a line of 5 fields is a Fortran record "i j k health age" (id = its line number,
 * time = -1); a line of 7 or more is "id i j k health age time [object side]"; any other line
 * is refused. Call with records = NULL to get the count in *n, then with capacity >= *n. */
int wacomm_b200_text_read(const char *path, wacomm_b200_particle *records, size_t capacity,
                          size_t *n);

/* Writes the resident records as a text restart: one device-to-host copy, then
 * wacomm_b200_text_write. */
int wacomm_b200_save_text(wacomm_b200_context *ctx, const char *path);

/* Provenance and run attributes of a NetCDF history (Provenance.hpp:20-27,
 * Particles.cpp:154-160); NULL strings are written empty, except proj_version, which is left out
 * when NULL (a build without PROJ). */
typedef struct wacomm_b200_history_meta {
    const char *git_revision, *compiler, *cmake_options;
    const char *configuration_file, *configuration;  /* the run's configuration path and JSON */
    const char *proj_version;
    const char *ocean_model;
    double checkpoint_time;  /* checkpoint_time attribute and the particle_time value */
} wacomm_b200_history_meta;

/* NetCDF history / restart of the resident records, schema version 3
 * (Particles::saveAsNetCDF, Particles.cpp:116-273): the records with j >= 0, i >= 0, k <= 0 and a
 * position on the grid, in order, as id, object_type, drift_side and lat, lon, depth, k, j, i,
 * health, age, time [particles][particle_time = 1], with the reference's attributes; tracking
 * direction and random seed from set_config, lat/lon/depth by kji2deplatlon from set_geo_grid.
 * Written as a CDF-5 (64-bit data) classic file, the classic variant that carries the schema's
 * uint64 and uint variables; the reference writes the same schema through NetCDF-4. The device
 * selects, locates and compacts the records and lays out every variable's big-endian payload;
 * the host writes the header and the payload. *written receives the number of records stored. */
int wacomm_b200_save_netcdf(wacomm_b200_context *ctx, const char *path,
                            const wacomm_b200_history_meta *meta, size_t *written);

/* What a NetCDF restart must match (Particles::loadFromNetCDF, Particles.cpp:380-430). */
typedef struct wacomm_b200_restart_expect {
    const char *ocean_model;  /* the configured ocean model */
    int backward;             /* the configured tracking direction: 0 forward, 1 backward */
    uint64_t random_seed;     /* the configured seed */
    int leeway;               /* drift.model = leeway: version 2 files lack the drift state */
} wacomm_b200_restart_expect;

/* Reads a NetCDF restart (CDF-1, CDF-2 or CDF-5 classic files): when it carries
 * wacomm_restart_version, the version must be 2 or 3 (2 refused under leeway), its tracking
 * direction must match, and random_seed, wacomm_random_key_scheme and ocean_model must match
 * when present. Records from id, i, j, k, health, age, time (first particle_time column) and,
 * when present, object_type and drift_side. *checkpoint_time and *has_checkpoint receive the
 * checkpoint_time attribute. Call with records = NULL for the count, then with capacity >= *n. */
int wacomm_b200_netcdf_read(const char *path, const wacomm_b200_restart_expect *expect,
                            wacomm_b200_particle *records, size_t capacity, size_t *n,
                            double *checkpoint_time, int *has_checkpoint);

/* The message of the last failed file call on this thread (text_write, text_read, netcdf_read). */
const char *wacomm_b200_file_error(void);

#ifdef __cplusplus
}
#endif

#endif /* WACOMM_B200_H */
