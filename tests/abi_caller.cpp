// A C++ host program that drives the engine through the extern "C" ABI alone (include/wacomm_b200.h),
// the way a WaComM++ build would after replacing its per-interval staging (Wacomm.cpp:386-610):
// one context, a rectilinear grid, two forcing records of a uniform eastward current, particles
// in, one interval in reference arithmetic, particles out. Every particle must end where the
// uniform current puts it, i + u * 3600 / xdist(row) with xdist the haversine cell width
// (kernel.cu:145-149), within 1e-6 grid units (0.2 mm: the reference's per-cell metric and
// midpoint rescaling differ from this closed form in the ninth digit); j and k unchanged and
// the age one hour.
// Build: g++ -std=c++17 abi_caller.cpp -I include -L <lib dir> -lwacomm_b200. Exit 0: passed;
// 77: no CUDA device; 1: a call failed or a record is off.
#include <cmath>
#include <cstdio>
#include <vector>

#include "wacomm_b200.h"

namespace {

int check(int status, wacomm_b200_context *ctx, const char *what) {
    if (status != WACOMM_B200_OK)
        std::fprintf(stderr, "%s: status %d: %s\n", what, status, wacomm_b200_last_error(ctx));
    return status;
}

double haversine(double lat1, double lon1, double lat2, double lon2) {
    const double dLat = lat2 - lat1, dLon = lon2 - lon1;
    const double v = std::sin(.5 * dLat) * std::sin(.5 * dLat) +
                     std::sin(.5 * dLon) * std::sin(.5 * dLon) * std::cos(lat2) * std::cos(lat1);
    return 2.0 * std::atan2(std::sqrt(v), std::sqrt(1.0 - v)) * 6371000.0;
}

}  // namespace

int main() {
    if (wacomm_b200_device_count() == 0) return 77;
    const int eta = 48, xi = 64, sRho = 4, sW = sRho + 1, n = 2000;
    const double deg = 0.0174533, u0 = (double)0.2f;  // the current as the records hold it
    std::vector<double> lon(eta * xi), lat(eta * xi), h(eta * xi, 40.0), mask(eta * xi, 1.0);
    for (int j = 0; j < eta; j++)
        for (int i = 0; i < xi; i++) {
            lon[j * xi + i] = (14.0 + 0.002 * i) * deg;
            lat[j * xi + i] = (40.7 + 0.0015 * j) * deg;
        }
    std::vector<double> depth(sW - 1, 1.0 / sRho), times = {1.6759e9, 1.6759e9 + 3600.0};
    std::vector<float> zeta(eta * xi, 0.f), u(sRho * eta * xi, 0.2f), v(sRho * eta * xi, 0.f);
    std::vector<float> w(sW * eta * xi, 0.f), akt(sW * eta * xi, 1e-4f);

    wacomm_b200_context *ctx = nullptr;
    if (check(wacomm_b200_context_create(0, &ctx), ctx, "context_create")) return 1;
    wacomm_b200_options opt;
    wacomm_b200_default_options(&opt);
    opt.arithmetic = WACOMM_B200_ARITH_REFERENCE;
    wacomm_b200_config cfg = {};
    cfg.random = false;
    cfg.deltat = 3600;
    cfg.dti = 30;
    cfg.survprob = 1e-4;
    cfg.tau0 = 86400;
    cfg.crid = 1;
    cfg.sigma = 3.46;
    cfg.shoreLimit = 0.25;
    cfg.upperClosure = 1;
    cfg.lowerClosure = 2;
    cfg.horizontalClosure = 3;
    cfg.randomSeed = 5489;
    cfg.trackingDirection = 1;
    cfg.integrator = 2;
    cfg.restartCheckpoint = NAN;
    std::vector<wacomm_b200_particle> p(n), out(n);
    for (int q = 0; q < n; q++) {
        p[q] = wacomm_b200_particle{};
        p[q].id = 1000 + q;
        p[q].j = 5.0 + 37.0 * ((q * 7919) % n) / n;
        p[q].i = 4.0 + 30.0 * ((q * 104729) % n) / n;
        p[q].k = -0.1 - 0.8 * (q % 10) / 10.0;
        p[q].health = 1.0;
        p[q].time = times[0];
    }
    int rc = check(wacomm_b200_set_options(ctx, &opt), ctx, "set_options");
    if (!rc) rc = check(wacomm_b200_set_config(ctx, &cfg), ctx, "set_config");
    if (!rc)
        rc = check(wacomm_b200_set_grid(ctx, eta, xi, sRho, sW, mask.data(), lon.data(), lat.data(),
                                        h.data(), depth.data()),
                   ctx, "set_grid");
    if (!rc) rc = check(wacomm_b200_set_times(ctx, 2, times.data()), ctx, "set_times");
    for (int t = 0; t < 2 && !rc; t++)
        rc = check(wacomm_b200_upload_frame(ctx, t, zeta.data(), u.data(), v.data(), w.data(),
                                            akt.data(), nullptr, nullptr, nullptr, nullptr),
                   ctx, "upload_frame");
    if (!rc) rc = check(wacomm_b200_set_particles(ctx, p.data(), n), ctx, "set_particles");
    if (!rc) rc = check(wacomm_b200_move_interval(ctx, 0), ctx, "move_interval");
    if (!rc) rc = check(wacomm_b200_get_particles(ctx, out.data(), n), ctx, "get_particles");
    wacomm_b200_context_destroy(ctx);
    if (rc) return 1;
    int bad = 0;
    for (int q = 0; q < n; q++) {
        const int row = (int)std::floor(p[q].j);
        const double xdist = haversine(lat[row * xi], lon[row * xi], lat[row * xi + 1], lon[row * xi + 1]);
        const double want = p[q].i + u0 * 3600.0 / xdist;
        const bool ok = std::fabs(out[q].i - want) <= 1e-6 && out[q].j == p[q].j &&
                        out[q].k == p[q].k && out[q].age == 3600.0 && out[q].health > 0 &&
                        out[q].id == p[q].id;
        if (!ok && bad++ < 5)
            std::fprintf(stderr, "record %d: i %.17g (want %.17g) j %.17g k %.17g age %g\n", q,
                         out[q].i, want, out[q].j, out[q].k, out[q].age);
    }
    std::printf("%d records, %d off\n", n, bad);
    return bad ? 1 : 0;
}
