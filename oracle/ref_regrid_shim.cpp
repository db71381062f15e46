// Test-infrastructure shim around the reference's own environmental regridder.
//
// This file is ours; it is compiled together with the reference source EnvironmentalRegridder.cpp,
// taken in place from the reference tree by oracle/Makefile, into
// oracle/_ref/libwacomm_ref_regrid.so (built without PROJ, as the reference builds without
// WACOMM_USE_PROJ). It exposes EnvironmentalRegridder::bilinearGeographic and
// bilinearCurvilinearGeographic (EnvironmentalRegridder.cpp:239-334) on flat row-major buffers;
// a thrown std::runtime_error becomes return code -1. It is never linked into the product library.
#include "EnvironmentalRegridder.hpp"

#include <cstring>
#include <stdexcept>

namespace {

template <class F>
int regrid(F f, int eta, int xi, const double *lon, const double *lat, int T, const float *src,
           long n, const double *tLon, const double *tLat, float *out) {
    try {
        Array::Array2<double> sLon(eta, xi), sLat(eta, xi), gLon(1, n), gLat(1, n);
        Array::Array3<float> field(T, eta, xi);
        for (int j = 0; j < eta; j++)
            for (int i = 0; i < xi; i++) {
                sLon(j, i) = lon[(size_t)j * xi + i];
                sLat(j, i) = lat[(size_t)j * xi + i];
            }
        for (int t = 0; t < T; t++)
            for (int j = 0; j < eta; j++)
                for (int i = 0; i < xi; i++)
                    field(t, j, i) = src[((size_t)t * eta + j) * xi + i];
        for (long k = 0; k < n; k++) {
            gLon(0, k) = tLon[k];
            gLat(0, k) = tLat[k];
        }
        Array::Array3<float> result = f(sLon, sLat, field, gLon, gLat);
        for (int t = 0; t < T; t++)
            for (long k = 0; k < n; k++) out[(size_t)t * n + k] = result(t, 0, k);
        return 0;
    } catch (const std::runtime_error &) {
        return -1;
    }
}

}  // namespace

extern "C" {

int ref_regrid_geographic(int eta, int xi, const double *lon, const double *lat, int T,
                          const float *src, long n, const double *tLon, const double *tLat,
                          float *out) {
    return regrid(EnvironmentalRegridder::bilinearGeographic, eta, xi, lon, lat, T, src, n, tLon,
                  tLat, out);
}

int ref_regrid_curvilinear(int eta, int xi, const double *lon, const double *lat, int T,
                           const float *src, long n, const double *tLon, const double *tLat,
                           float *out) {
    return regrid(EnvironmentalRegridder::bilinearCurvilinearGeographic, eta, xi, lon, lat, T,
                  src, n, tLon, tLat, out);
}

}  // extern "C"
