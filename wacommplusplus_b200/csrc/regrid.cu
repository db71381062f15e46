// Wind and Stokes fields from their own grids and times to the ocean grid's rho nodes and the
// context's forcing times, on the device.
//
// Restates the two geographic bilinear regridders of EnvironmentalRegridder.cpp:
//   * bilinearGeographic (:239-275): rectilinear source axes, the longitude axis unwrapped and
//     each target put on its branch, then `bracket` (:14-28) on each axis -- the first interval
//     that holds the target within 1e-10 -- and the two-stage linear weights;
//   * bilinearCurvilinearGeographic (:277-334): the CurvilinearCellIndex bins (:170-236), then
//     for each target the candidates of its bin in index order, a 20-step Newton inversion of the
//     cell's bilinear map, and the first candidate that holds the target (parameters within 1e-9,
//     residual below 1e-8) is taken, a folded or singular accepted cell being an error.
// A target's cell and weights are found once (the plan); every record of the field is then read
// through the plan. The records are aligned to the forcing times in the same pass: a forcing time
// equal to a source time (1e-6 s) copies that record, one between two source times blends the two
// regridded values with the time weight of NumericalHelpers.hpp:30-39. The reference instead
// requires equal times and grids (Wacomm.cpp:70-84).
//
// The cell index is built by the host from the source coordinates (linear in the source cells,
// once per source grid); the per-target searches and the per-record interpolation run here.
// Compiled with -fmad=false: the weights, the Newton steps and the bilinear sums round exactly as
// the reference's unfused host arithmetic.
#include "engine.h"

namespace wb {

namespace {

constexpr int THREADS = 256;

__device__ __forceinline__ void raise(int *err, int code) { atomicOr(err, code); }

// nearLongitude (EnvironmentalRegridder.cpp:44-48); the caller bounds |value - reference|.
__device__ __forceinline__ double near_longitude(double value, double reference) {
    while (value - reference > 180) value -= 360;
    while (value - reference < -180) value += 360;
    return value;
}

// A longitude farther than this from the reference is refused instead of being stepped by 360
// for as long as it takes (the reference's loop never ends on a huge finite value).
constexpr double LONGITUDE_REACH = 3600.0;

__device__ __forceinline__ double bilinear(double f00, double f10, double f01, double f11,
                                           double x, double y) {
    return (1 - x) * (1 - y) * f00 + x * (1 - y) * f10 + (1 - x) * y * f01 + x * y * f11;
}

// bracket (EnvironmentalRegridder.cpp:14-28) by bisection: the first interval i whose far end
// holds value (a[i+1] + 1e-10 >= value on a rising axis, a[i+1] - 1e-10 <= value on a falling
// one). That predicate is monotone in i, and its first true index is the first interval of the
// linear scan, whose near-end test every earlier failure already implies.
__device__ __forceinline__ bool bracket(const double *axis, int n, bool increasing, double value,
                                        int &lower, double &weight) {
    double minimum = increasing ? axis[0] : axis[n - 1];
    double maximum = increasing ? axis[n - 1] : axis[0];
    if (value < minimum - 1.e-10 || value > maximum + 1.e-10) return false;
    int lo = 0, hi = n - 2;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        bool holds = increasing ? value <= axis[mid + 1] + 1.e-10 : value >= axis[mid + 1] - 1.e-10;
        if (holds) hi = mid;
        else lo = mid + 1;
    }
    lower = lo;
    weight = (value - axis[lo]) / (axis[lo + 1] - axis[lo]);
    return true;
}

__global__ void geographic_plan_kernel(RegridGeographic G, long long nTarget, const double *tLon,
                                       const double *tLat, RegridPlan *plan, int *err) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nTarget) return;
    double x = tLon[n], y = tLat[n];
    RegridPlan p{-1, 0.0, 0.0};
    if (!isfinite(x) || !isfinite(y)) {
        raise(err, REGRID_ERR_TARGET);
    } else if (!(fabs(x - G.center) <= LONGITUDE_REACH)) {
        raise(err, REGRID_ERR_TARGET);
    } else {
        int xl, yl;
        double wx, wy;
        if (bracket(G.axisX, G.xi, G.risingX, near_longitude(x, G.center), xl, wx) &&
            bracket(G.axisY, G.eta, G.risingY, y, yl, wy)) {
            p.node = yl * G.xi + xl;
            p.wx = wx;
            p.wy = wy;
        } else {
            raise(err, REGRID_ERR_OUTSIDE);
        }
    }
    plan[n] = p;
}

__device__ __forceinline__ int cell_bin(double v, double minimum, double maximum, int bins) {
    if (maximum == minimum) return 0;
    int b = (int)((v - minimum) / (maximum - minimum) * bins);
    return max(0, min(bins - 1, b));
}

__global__ void curvilinear_plan_kernel(RegridCurvilinear C, long long nTarget,
                                        const double *tLon, const double *tLat, RegridPlan *plan,
                                        int *err) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nTarget) return;
    double targetX = tLon[n], targetY = tLat[n];
    RegridPlan p{-1, 0.0, 0.0};
    plan[n] = p;
    if (!isfinite(targetX) || !isfinite(targetY) ||
        !(fabs(targetX - C.reference) <= LONGITUDE_REACH)) {
        raise(err, REGRID_ERR_TARGET);
        return;
    }
    // CurvilinearCellIndex::candidates moves the target to the branch of the index reference
    targetX = near_longitude(targetX, C.reference);
    int first = 0, last = 0;
    if (!(targetX < C.minX - 1.e-10 || targetX > C.maxX + 1.e-10 || targetY < C.minY - 1.e-10 ||
          targetY > C.maxY + 1.e-10)) {
        int bin = cell_bin(targetY, C.minY, C.maxY, C.binsY) * C.binsX +
                  cell_bin(targetX, C.minX, C.maxX, C.binsX);
        first = C.binStart[bin];
        last = C.binStart[bin + 1];
    }
    const int xi = C.xi;
    for (int c = first; c < last; c++) {
        const int cell = C.binCells[c];
        const int j = cell / (xi - 1), i = cell - j * (xi - 1);
        const double *L = C.lon + (size_t)j * xi + i, *A = C.lat + (size_t)j * xi + i;
        // the source longitudes are finite and within a revolution of each other (host checks)
        double x00 = near_longitude(L[0], targetX), x10 = near_longitude(L[1], targetX);
        double x01 = near_longitude(L[xi], targetX), x11 = near_longitude(L[xi + 1], targetX);
        double y00 = A[0], y10 = A[1], y01 = A[xi], y11 = A[xi + 1];
        const double4 box = C.box[cell];  // minimumX, maximumX, minimumY, maximumY
        if (targetX < box.x - 1.e-10 || targetX > box.y + 1.e-10 || targetY < box.z - 1.e-10 ||
            targetY > box.w + 1.e-10)
            continue;
        double x = .5, y = .5;
        for (int iteration = 0; iteration < 20; iteration++) {
            double mappedX = bilinear(x00, x10, x01, x11, x, y);
            double mappedY = bilinear(y00, y10, y01, y11, x, y);
            double dXdx = (1 - y) * (x10 - x00) + y * (x11 - x01);
            double dXdy = (1 - x) * (x01 - x00) + x * (x11 - x10);
            double dYdx = (1 - y) * (y10 - y00) + y * (y11 - y01);
            double dYdy = (1 - x) * (y01 - y00) + x * (y11 - y10);
            double determinant = dXdx * dYdy - dXdy * dYdx;
            if (fabs(determinant) < 1.e-14) break;
            double residualX = mappedX - targetX, residualY = mappedY - targetY;
            x -= (dYdy * residualX - dXdy * residualY) / determinant;
            y -= (-dYdx * residualX + dXdx * residualY) / determinant;
        }
        double residual = hypot(bilinear(x00, x10, x01, x11, x, y) - targetX,
                                bilinear(y00, y10, y01, y11, x, y) - targetY);
        if (x >= -1.e-9 && x <= 1 + 1.e-9 && y >= -1.e-9 && y <= 1 + 1.e-9 && residual < 1.e-8) {
            double d00 = (x10 - x00) * (y01 - y00) - (x01 - x00) * (y10 - y00);
            double d10 = (x10 - x00) * (y11 - y10) - (x11 - x10) * (y10 - y00);
            double d01 = (x11 - x01) * (y01 - y00) - (x01 - x00) * (y11 - y01);
            double d11 = (x11 - x01) * (y11 - y10) - (x11 - x10) * (y11 - y01);
            if (fabs(d00) < 1.e-14 || d00 * d10 <= 0 || d00 * d01 <= 0 || d00 * d11 <= 0) {
                raise(err, REGRID_ERR_FOLDED);
                return;
            }
            // std::max(0.0, std::min(1.0, v)), signed zeros included
            double mx = x < 1.0 ? x : 1.0, my = y < 1.0 ? y : 1.0;
            p.node = j * xi + i;
            p.wx = 0.0 < mx ? mx : 0.0;
            p.wy = 0.0 < my ? my : 0.0;
            plan[n] = p;
            return;
        }
    }
    raise(err, REGRID_ERR_OUTSIDE);
}

__global__ void finite_kernel(const float *values, long long count, int *err) {
    bool bad = false;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < count;
         n += (long long)gridDim.x * blockDim.x)
        bad |= !isfinite(values[n]);
    if (__syncthreads_or(bad) && threadIdx.x == 0) raise(err, REGRID_ERR_FIELD);
}

template <bool CURVILINEAR>
__device__ __forceinline__ float spatial(const float *s, int xi, const RegridPlan &p) {
    const float *q = s + p.node;
    if (CURVILINEAR) return (float)bilinear(q[0], q[1], q[xi], q[xi + 1], p.wx, p.wy);
    double lower = q[0] * (1 - p.wx) + q[1] * p.wx;
    double upper = q[xi] * (1 - p.wx) + q[xi + 1] * p.wx;
    return (float)(lower * (1 - p.wy) + upper * p.wy);
}

// One thread per (target, forcing time, component): the regridded value at the bracketing source
// record(s), blended in time, written into that forcing time's plane.
template <bool CURVILINEAR>
__global__ void apply_kernel(const RegridPlan *plan, long long nTarget, int srcXi,
                             long long srcPlane, const float *srcU, const float *srcV,
                             const RegridTime *times, float *outU, float *outV) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nTarget) return;
    const RegridTime T = times[blockIdx.y];
    const float *src = blockIdx.z ? srcV : srcU;
    float *out = (blockIdx.z ? outV : outU) + (size_t)blockIdx.y * nTarget;
    const RegridPlan p = plan[n];
    if (p.node < 0) return;
    float a = spatial<CURVILINEAR>(src + (size_t)T.k0 * srcPlane, srcXi, p);
    if (T.k1 == T.k0) {
        out[n] = a;
        return;
    }
    float b = spatial<CURVILINEAR>(src + (size_t)T.k1 * srcPlane, srcXi, p);
    out[n] = (float)((1.0 - T.alpha) * a + T.alpha * b);
}

unsigned grid_of(long long n) { return (unsigned)((n + THREADS - 1) / THREADS); }

}  // namespace

cudaError_t regrid_check_finite(const float *values, long long count, int *err,
                                cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    unsigned blocks = (unsigned)std::min<long long>(grid_of(count), 148 * 8);
    finite_kernel<<<blocks, THREADS, 0, stream>>>(values, count, err);
    return cudaGetLastError();
}

cudaError_t regrid_plan_geographic(const RegridGeographic &G, long long nTarget,
                                   const double *tLon, const double *tLat, RegridPlan *plan,
                                   int *err, cudaStream_t stream) {
    if (nTarget <= 0) return cudaSuccess;
    geographic_plan_kernel<<<grid_of(nTarget), THREADS, 0, stream>>>(G, nTarget, tLon, tLat, plan,
                                                                      err);
    return cudaGetLastError();
}

cudaError_t regrid_plan_curvilinear(const RegridCurvilinear &C, long long nTarget,
                                    const double *tLon, const double *tLat, RegridPlan *plan,
                                    int *err, cudaStream_t stream) {
    if (nTarget <= 0) return cudaSuccess;
    curvilinear_plan_kernel<<<grid_of(nTarget), THREADS, 0, stream>>>(C, nTarget, tLon, tLat,
                                                                       plan, err);
    return cudaGetLastError();
}

cudaError_t regrid_apply(bool curvilinear, const RegridPlan *plan, long long nTarget, int srcXi,
                         long long srcPlane, const float *srcU, const float *srcV,
                         const RegridTime *times, int nTimes, float *outU, float *outV,
                         cudaStream_t stream) {
    if (nTarget <= 0 || nTimes <= 0) return cudaSuccess;
    dim3 grid(grid_of(nTarget), (unsigned)nTimes, 2);
    if (curvilinear)
        apply_kernel<true><<<grid, THREADS, 0, stream>>>(plan, nTarget, srcXi, srcPlane, srcU,
                                                          srcV, times, outU, outV);
    else
        apply_kernel<false><<<grid, THREADS, 0, stream>>>(plan, nTarget, srcXi, srcPlane, srcU,
                                                           srcV, times, outU, outV);
    return cudaGetLastError();
}

}  // namespace wb
