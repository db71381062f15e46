// ROMS records normalized on the device into forcing records.
//
// Restates the per-record part of ROMSAdapter::process (OceanModelAdapters/ROMSAdapter.cpp):
//   * zeta zeroed on land and at fill values >= 1e36 (:254-265);
//   * uv2rho (:309-368): u and v averaged from the wet faces around each wet rho node (float sums
//     divided by the count of wet faces), 0 elsewhere;
//   * the rotation of grid-relative velocities to east/north by the grid angle (:273-302), in
//     double from the float averages, with a velocity outside the float range an error;
//   * wakt2wakt (:431-462): w and AKt zeroed on land;
// plus the adapter's check that u and v hold finite values on every wet face (:148-160). The grid
// part (masks as 0/1 bytes, the cosine and sine of the angle computed by the host's libm once per
// grid, exactly the values the reference computes) is set up once; each record is then one pass
// over its levels. Compiled with -fmad=false: the rotation's products and difference round as the
// reference's unfused host arithmetic.
#include <cfloat>

#include "engine.h"

namespace wb {

namespace {

__global__ void roms_record_kernel(RomsGrid G, RomsRecord R, int *err) {
    const int xi = G.xi, eta = G.eta, xiU = xi - 1, etaV = eta - 1;
    const size_t plane = (size_t)eta * xi;
    const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= plane) return;
    const int level = blockIdx.y;
    const int j = (int)(n / xi), i = (int)(n - (size_t)j * xi);
    const bool wet = G.maskRho[n] != 0;
    const size_t at = (size_t)level * plane + n;
    if (level == 0) {
        float z = R.zeta[n];
        R.zetaOut[n] = (!wet || z >= 1e+36f) ? 0.0f : z;
    }
    R.wOut[at] = wet ? R.w[at] : 0.0f;
    R.aktOut[at] = wet ? R.akt[at] : 0.0f;
    if (level >= G.sRho) return;
    const size_t planeU = (size_t)eta * xiU, planeV = (size_t)etaV * xi;
    const float *u = R.u + (size_t)level * planeU, *v = R.v + (size_t)level * planeV;
    // every wet face holds a value
    bool bad = (i < xiU && G.maskU[(size_t)j * xiU + i] && !isfinite(u[(size_t)j * xiU + i])) ||
               (j < etaV && G.maskV[(size_t)j * xi + i] && !isfinite(v[(size_t)j * xi + i]));
    if (bad) atomicOr(err, ROMS_ERR_FACE);
    float uo = 0.0f, vo = 0.0f;
    if (wet) {
        float usum = 0.0f, vsum = 0.0f;
        int ucount = 0, vcount = 0;
        if (i < xiU && G.maskU[(size_t)j * xiU + i]) {
            usum += u[(size_t)j * xiU + i];
            ucount++;
        }
        if (i > 0 && G.maskU[(size_t)j * xiU + i - 1]) {
            usum += u[(size_t)j * xiU + i - 1];
            ucount++;
        }
        if (j < etaV && G.maskV[(size_t)j * xi + i]) {
            vsum += v[(size_t)j * xi + i];
            vcount++;
        }
        if (j > 0 && G.maskV[(size_t)(j - 1) * xi + i]) {
            vsum += v[(size_t)(j - 1) * xi + i];
            vcount++;
        }
        uo = ucount > 0 ? usum / ucount : 0.0f;
        vo = vcount > 0 ? vsum / vcount : 0.0f;
        double gridU = uo, gridV = vo, east = gridU, north = gridV;
        if (G.rotation) {
            const double2 cs = G.rotation[n];
            east = gridU * cs.x - gridV * cs.y;
            north = gridU * cs.y + gridV * cs.x;
        }
        if (!isfinite(east) || !isfinite(north) || fabs(east) > FLT_MAX || fabs(north) > FLT_MAX) {
            atomicOr(err, ROMS_ERR_VELOCITY);
        } else {
            uo = (float)east;
            vo = (float)north;
        }
    }
    R.uOut[at] = uo;
    R.vOut[at] = vo;
}

}  // namespace

cudaError_t roms_record(const RomsGrid &G, const RomsRecord &R, int *err, cudaStream_t stream) {
    const size_t plane = (size_t)G.eta * G.xi;
    dim3 grid((unsigned)((plane + 255) / 256), (unsigned)(G.sRho + 1));
    roms_record_kernel<<<grid, 256, 0, stream>>>(G, R, err);
    return cudaGetLastError();
}

}  // namespace wb
