/*
 * CPU oracle of the WaComM++ particle-move path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithm, used by tests/, by
 * __graft_entry__.smoke() and by the cpu_baseline leg of bench.py as the checker. The
 * product library never links, loads or calls it. Each function cites the reference
 * file:line it restates. Parity is pinned two ways (tests/test_oracle_*.py): against the
 * reference's own known-answer tests (pinned RNG values, leeway catalogue, analytic
 * interval, integrator order ratios, concentration count preservation), and record-for-
 * record against the reference Particle::move compiled from its own sources
 * (oracle/_ref, built by oracle/Makefile when the reference tree is present). The regridders are
 * pinned the same two ways (EnvironmentalRegridderTest.cpp and EnvironmentalRegridder.cpp built
 * into oracle/_ref); the ROMS normalization only against the known answers of
 * ROMSAdapterTest.cpp, since the adapter reads NetCDF and is not built here.
 */
#ifndef WACOMM_ORACLE_H
#define WACOMM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same binary layout as the reference's particle_data (Particle.hpp:31-41), 64 bytes. */
typedef struct wo_particle {
    uint64_t id;
    double k, j, i;
    double health, age, time;
    uint16_t driftObjectType;
    int8_t driftSide;
} wo_particle;

typedef struct wo_region {
    double west, south, east, north;
    double windErrorStdDev, windErrorComponentCorrelation;
    double windErrorSpatialScale, windErrorTemporalScale;
} wo_region;

/* Same binary layout as the reference's config_data (Config.hpp:36-72), 1248 bytes. */
typedef struct wo_config {
    _Bool random;
    _Bool randomSources;
    double deltat, dti, survprob, tau0, sv, crid, sigma, shoreLimit;
    int upperClosure, lowerClosure, horizontalClosure;
    uint64_t randomSeed;
    int trackingDirection, backwardDiffusion, integrator;
    double restartCheckpoint;
    int driftModel;
    _Bool leewayCoefficientEnsemble;
    double leewayResidualCorrelation;
    _Bool leewayRandomSide;
    double leewayRightSideProbability, leewayJibeProbabilityHourly;
    double windErrorStdDev, windErrorComponentCorrelation;
    double windErrorSpatialScale, windErrorTemporalScale;
    uint32_t observationalCalibrationRegionCount;
    wo_region observationalCalibrationRegions[16];
    uint16_t driftObjectType;
    int8_t driftSide;
    _Bool hasWind;
    double windU10, windV10;
} wo_config;

/* A forcing window in the layout of the reference device contract (kernel.cu:63-69):
 * zeta/wind/stokes [T][eta][xi]; u,v [T][sRho][eta][xi]; w,akt [T][sW][eta][xi] with storage
 * level = logical k + levels - 1; depthIntervals[sW-1] indexed kI+sW-2; 2-D fields [eta][xi]. */
typedef struct wo_window {
    int T, sW, sRho, eta, xi;
    const double *times, *mask, *lonRad, *latRad, *depthIntervals, *h;
    const float *zeta, *u, *v, *w, *akt;
    const float *windU10, *windV10, *stokesU, *stokesV; /* may be NULL */
} wo_window;

enum { WO_SEMANTICS_HOST = 0, WO_SEMANTICS_DEVICE = 1 };
enum { WO_CLOSURE_CONSTRAINT = 1, WO_CLOSURE_KILL = 2, WO_CLOSURE_REFLECTION = 3 };
enum { WO_EULER = 1, WO_MIDPOINT = 2 };

/* NumericalHelpers.hpp:84-120 (scheme ordered-splitmix64-v2). */
uint64_t wo_mix(uint64_t value);
uint64_t wo_combine(uint64_t state, uint64_t coordinate);
double wo_uniform(uint64_t seed, uint64_t particle, int64_t interval, uint64_t substep,
                  uint64_t component);
double wo_normal(uint64_t seed, uint64_t particle, int64_t interval, uint64_t substep,
                 uint64_t component);
/* DriftModel.hpp:118-160, 176-219. */
double wo_forcing_error_normal(uint64_t seed, uint64_t particle, int64_t interval,
                               uint64_t substep, uint64_t component, double longitude,
                               double latitude, double physicalTime, double spatialScale,
                               double temporalScale);
double wo_correlated_normal(double first, double independent, double correlation);
double wo_jibe_step_probability(double hourly, double seconds);
int wo_drift_coefficients(int type, double out9[9]); /* returns 0 if type is in the catalogue */
void wo_compute_leeway(const double c9[9], double windU, double windV, int side,
                       double downwindNormal, double crosswindNormal, double outUV[2]);
int wo_calibration_region(const wo_region *regions, uint32_t count, double lonRad,
                          double latRad);
int wo_sample_drift_side(uint64_t seed, uint64_t particle, double rightProbability);
/* NumericalHelpers.hpp:45-74. */
double wo_restart_elapsed(double intervalStart, double intervalEnd, double checkpoint);
double wo_reflect_cell(double oldCoordinate, int oldCell, double candidate, int candidateCell);
double wo_reflect_domain(double coordinate, double maximum);

/* Moves n particles over the forcing interval starting at timeIndex.
 * semantics = WO_SEMANTICS_HOST restates Particle::move (Particle.cpp:71-824);
 * semantics = WO_SEMANTICS_DEVICE restates the reference kernel (kernel.cu:153-368).
 * Returns 0, or -1 when a particle names a drift object outside the catalogue in host
 * semantics (the reference throws there, DriftModel.cpp:51-54). threads<=0: all cores. */
int wo_move_batch(const wo_config *config, wo_particle *particles, long n,
                  const wo_window *window, int timeIndex, int semantics, int threads);

/* Concentration::evaluate (Concentration.hpp:16-44) into uint32 counts
 * conc[Tc][sRho][eta][xi] (accumulated, not cleared). */
void wo_concentration(const wo_particle *particles, long n, int concTimeIdx, int Tc, int sRho,
                      int eta, int xi, uint32_t *conc);

/* Land mask of the float concentration grid conc[][sRho][eta][xi] at one evaluated time
 * (Wacomm.cpp:188-196,724-737): 1e37 in every level of each cell whose mask is not 1. */
void wo_concentration_mask(float *conc, int concTimeIdx, int sRho, int eta, int xi,
                           const double *mask);

/* sourceEmissionTimes (SourceEmission.hpp:38-79): mode 0 uniform_rate, 1 forcing_interval_batch,
 * 2 single_pulse. Returns the count (writing at most cap values) or -1 on an invalid schedule. */
long wo_source_emission_times(int mode, double value, double sourceStart, double sourceEnd,
                              double intervalStart, double intervalEnd, double *out, long cap);
double wo_source_position_offset(uint64_t seed, uint64_t particle, uint64_t component);

/* A release point: the fields of Source (Source.hpp:19-60); start/end in days (< 0: run start /
 * no end), emission_mode as in wo_source_emission_times, and only mode 1 emits. */
typedef struct wo_source {
    double k, j, i;
    double start, end;
    double emission_value;
    int32_t emission_mode;
    int32_t mode;
} wo_source;

/* Sources::emit + Source::emissionTimes + Source::emit (Sources.cpp:233-249, Source.cpp:16-45):
 * appends the interval's releases of every source to out[0..) in stable time order, ids from
 * first_id on. Returns the count (writing at most cap records) or -1 on an invalid schedule. */
long wo_sources_emit(const wo_config *config, const wo_source *sources, int n_sources,
                     double julian_start, double interval_start, double interval_end,
                     uint64_t first_id, wo_particle *out, long cap);

/* kji2deplatlon / deplatlon2kji (OceanModelAdapter.cpp:271-442) on a grid with lon/lat in
 * degrees [eta][xi], h [eta][xi] and sW[sW] (indexed k+sW-1). kji2deplatlon returns -1 and
 * 1e37 outputs off the grid; deplatlon2kji returns -1 when the point is not on the grid. */
int wo_kji2deplatlon(int eta, int xi, int sW, const double *lon, const double *lat,
                     const double *h, const double *sWValues, double k, double j, double i,
                     double *dep, double *latOut, double *lonOut);
int wo_deplatlon2kji(int eta, int xi, int sW, const double *lon, const double *lat,
                     const double *h, const double *sWValues, double dep, double latIn,
                     double lonIn, double *k, double *j, double *i);

/* Environmental regridding to target nodes (EnvironmentalRegridder.cpp). Source coordinates
 * lon/lat [eta][xi] in degrees, source fields src[T][eta][xi], targets tLon/tLat[nTarget],
 * results out[T][nTarget]. Return 0, or a negative code where the reference throws:
 * WO_REGRID_GRID (source grid invalid: dimensions, not rectilinear, non-monotonic axis, span),
 * WO_REGRID_OUTSIDE (a target outside the source grid: extrapolation is prohibited),
 * WO_REGRID_FIELD (a non-finite source value), WO_REGRID_FOLDED (a folded or singular cell),
 * WO_REGRID_TARGET (a non-finite target coordinate). */
#define WO_REGRID_GRID (-1)
#define WO_REGRID_OUTSIDE (-2)
#define WO_REGRID_FIELD (-3)
#define WO_REGRID_FOLDED (-4)
#define WO_REGRID_TARGET (-5)
#define WO_REGRID_TIME (-6)
/* bilinearGeographic (EnvironmentalRegridder.cpp:239-275): rectilinear source axes. */
int wo_regrid_geographic(int eta, int xi, const double *lon, const double *lat, int T,
                         const float *src, long nTarget, const double *tLon, const double *tLat,
                         float *out);
/* bilinearCurvilinearGeographic (EnvironmentalRegridder.cpp:277-334) with the cell index of
 * CurvilinearCellIndex (:170-236): first cell in index order that holds the target. */
int wo_regrid_curvilinear(int eta, int xi, const double *lon, const double *lat, int T,
                          const float *src, long nTarget, const double *tLon, const double *tLat,
                          float *out);
/* Aligns records at srcTimes[nSrc] (strictly increasing) to dstTimes[nDst]: each destination
 * time between two source times (1e-6 s tolerance at the ends, the tolerance of the reference's
 * time check, Wacomm.cpp:70-84) takes (float)((1-a)*x0 + a*x1) with a = timeWeight
 * (NumericalHelpers.hpp:30-39); a destination time equal to a source time copies that record.
 * plane values per record; out[nDst][plane]. The reference requires equal times instead. */
int wo_align_times(int nSrc, const double *srcTimes, long plane, const float *src, int nDst,
                   const double *dstTimes, float *out);

/* The per-record normalization of ROMSAdapter::process (OceanModelAdapters/ROMSAdapter.cpp:
 * 228-306, uv2rho :309-368, wakt2wakt :431-462): zeta zeroed on land and at fill values (>= 1e36),
 * u/v averaged from the wet faces to the rho nodes, rotated by the grid angle to east/north
 * (angle NULL: already earth-relative), w/AKt zeroed on land. mask_rho [eta][xi], mask_u
 * [eta][xi-1], mask_v [eta-1][xi] (0 or 1); u [sRho][eta][xi-1], v [sRho][eta-1][xi], w/akt
 * [sRho+1][eta][xi], zeta [eta][xi]; outputs on the rho grid. Returns 0, WO_ROMS_MASK (a mask
 * value other than 0/1), WO_ROMS_ANGLE (a non-finite angle at a wet node), WO_ROMS_FACE (a
 * non-finite u/v at a wet face) or WO_ROMS_VELOCITY (a rotated velocity outside the float range). */
#define WO_ROMS_MASK (-1)
#define WO_ROMS_ANGLE (-2)
#define WO_ROMS_FACE (-3)
#define WO_ROMS_VELOCITY (-4)
int wo_roms_normalize(int eta, int xi, int sRho, const double *maskRho, const double *maskU,
                      const double *maskV, const double *angle, const float *zeta, const float *u,
                      const float *v, const float *w, const float *akt, float *zetaOut,
                      float *uOut, float *vOut, float *wOut, float *aktOut);

/* Particles::saveAsTxt (Particles.cpp:28-55): "\t<count>" then one line per record,
 * "id i j k health age time object side", the reals with printf "%.17g" (the reference's ostream
 * with setprecision(max_digits10) in the default float format), one record after the other on
 * one thread as the reference does. Returns 0, or -1 when the file cannot be written. */
int wo_text_restart(const char *path, const wo_particle *records, size_t n);

#ifdef __cplusplus
}
#endif

#endif
