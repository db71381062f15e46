// Forcing views: how the step reads the bracketing forcing pair.
//
// PackedView is the engine layout. For each interval the two bracketing records are
// interleaved into one node record per (W level L, j, i):
//     {w(L), akt(L), u(L-1), v(L-1)} of record t0, then the same of record t1
// so that one particle's trilinear stencil (4 corners x 2 levels) is 8 records, each one
// 32-byte sector (16 bytes in half precision), instead of 48 scalar gathers from four fields
// and two frames. Surface data sit in a 16-byte {h, zeta(t0), zeta(t1)} record per node, the
// optional wind/Stokes pair in a 32-byte record, the cell metric in a per-cell table.
//
// RawView reads the reference device layout directly (kernel.cu:63-80): it serves the drop-in
// launcher, whose caller owns separate field arrays for the whole window.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"

namespace wb {

// Time pair of one node: upper record (u, v, w, akt) and lower record (w, akt).
struct NodeUp {
    float u0, u1, v0, v1, w0, w1, a0, a1;
};
struct NodeLo {
    float w0, w1, a0, a1;
};
struct SurfPair {
    double h;
    float z0, z1;
};
struct EnvPair {
    float wu0, wv0, su0, sv0, wu1, wv1, su1, sv1;
};

// Record of the packed pair in each storage precision.
template <int STORE>
struct NodeRecord;
template <>
struct NodeRecord<STORE_F32> {
    float4 t0, t1;  // (w, akt, u, v) of records t0 and t1
};
template <>
struct alignas(16) NodeRecord<STORE_F16> {
    __half2 wa0, uv0, wa1, uv1;
};
template <>
struct alignas(16) NodeRecord<STORE_BF16> {
    __nv_bfloat162 wa0, uv0, wa1, uv1;
};

template <int STORE>
__device__ __forceinline__ void load_node(const NodeRecord<STORE> *p, float &w0, float &a0,
                                          float &u0, float &v0, float &w1, float &a1, float &u1,
                                          float &v1);

template <>
__device__ __forceinline__ void load_node<STORE_F32>(const NodeRecord<STORE_F32> *p, float &w0,
                                                     float &a0, float &u0, float &v0, float &w1,
                                                     float &a1, float &u1, float &v1) {
    float4 x = __ldg(&p->t0), y = __ldg(&p->t1);
    w0 = x.x; a0 = x.y; u0 = x.z; v0 = x.w;
    w1 = y.x; a1 = y.y; u1 = y.z; v1 = y.w;
}

template <>
__device__ __forceinline__ void load_node<STORE_F16>(const NodeRecord<STORE_F16> *p, float &w0,
                                                     float &a0, float &u0, float &v0, float &w1,
                                                     float &a1, float &u1, float &v1) {
    uint4 raw = __ldg(reinterpret_cast<const uint4 *>(p));
    float2 wa0 = __half22float2(*reinterpret_cast<__half2 *>(&raw.x));
    float2 uv0 = __half22float2(*reinterpret_cast<__half2 *>(&raw.y));
    float2 wa1 = __half22float2(*reinterpret_cast<__half2 *>(&raw.z));
    float2 uv1 = __half22float2(*reinterpret_cast<__half2 *>(&raw.w));
    w0 = wa0.x; a0 = wa0.y; u0 = uv0.x; v0 = uv0.y;
    w1 = wa1.x; a1 = wa1.y; u1 = uv1.x; v1 = uv1.y;
}

template <>
__device__ __forceinline__ void load_node<STORE_BF16>(const NodeRecord<STORE_BF16> *p, float &w0,
                                                      float &a0, float &u0, float &v0, float &w1,
                                                      float &a1, float &u1, float &v1) {
    uint4 raw = __ldg(reinterpret_cast<const uint4 *>(p));
    float2 wa0 = __bfloat1622float2(*reinterpret_cast<__nv_bfloat162 *>(&raw.x));
    float2 uv0 = __bfloat1622float2(*reinterpret_cast<__nv_bfloat162 *>(&raw.y));
    float2 wa1 = __bfloat1622float2(*reinterpret_cast<__nv_bfloat162 *>(&raw.z));
    float2 uv1 = __bfloat1622float2(*reinterpret_cast<__nv_bfloat162 *>(&raw.w));
    w0 = wa0.x; a0 = wa0.y; u0 = uv0.x; v0 = uv0.y;
    w1 = wa1.x; a1 = wa1.y; u1 = uv1.x; v1 = uv1.y;
}

// Grid-level constants every view shares.
struct GridShape {
    int eta, xi, sW, sRho;
};

template <int STORE>
struct PackedView {
    GridShape g;
    const NodeRecord<STORE> *nodes;  // [sW][eta][xi]
    const SurfPair *surf;            // [eta][xi]
    const EnvPair *env;              // [eta][xi] or null
    bool hasWindU, hasWindV, hasStokes;
    const double *lonRad, *latRad;   // [eta][xi]
    const double *depthIntervals;    // [sW-1]
    const double2 *metric;           // [eta][xi] {xdist, ydist} of cell (j, i)

    __device__ __forceinline__ size_t node_index(int L, int j, int i) const {
        return ((size_t)L * (size_t)g.eta + (size_t)j) * (size_t)g.xi + (size_t)i;
    }
    // Upper node of logical level kI (W level kI with rho level kI), kI in [-sW+2, 0].
    __device__ __forceinline__ NodeUp up(int kI, int j, int i) const {
        NodeUp n;
        load_node<STORE>(nodes + node_index(kI + g.sW - 1, j, i), n.w0, n.a0, n.u0, n.v0, n.w1,
                         n.a1, n.u1, n.v1);
        return n;
    }
    // Lower node (W level kI-1).
    __device__ __forceinline__ NodeLo lo(int kI, int j, int i) const {
        float w0, a0, u0, v0, w1, a1, u1, v1;
        load_node<STORE>(nodes + node_index(kI + g.sW - 2, j, i), w0, a0, u0, v0, w1, a1, u1, v1);
        return NodeLo{w0, w1, a0, a1};
    }
    __device__ __forceinline__ SurfPair surface(int j, int i) const {
        double2 raw = __ldg(reinterpret_cast<const double2 *>(surf) + (size_t)j * g.xi + i);
        SurfPair s;
        s.h = raw.x;
        float2 z = *reinterpret_cast<float2 *>(&raw.y);
        s.z0 = z.x;
        s.z1 = z.y;
        return s;
    }
    __device__ __forceinline__ double h(int j, int i) const { return surface(j, i).h; }
    __device__ __forceinline__ EnvPair environment(int j, int i) const {
        const float4 *p = reinterpret_cast<const float4 *>(env + (size_t)j * g.xi + i);
        float4 a = __ldg(p), b = __ldg(p + 1);
        return EnvPair{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    }
    __device__ __forceinline__ double lon(int j, int i) const { return __ldg(lonRad + (size_t)j * g.xi + i); }
    __device__ __forceinline__ double lat(int j, int i) const { return __ldg(latRad + (size_t)j * g.xi + i); }
    __device__ __forceinline__ double depth_interval(int kI) const {
        return __ldg(depthIntervals + (kI + g.sW - 2));
    }
    __device__ __forceinline__ double2 cell_metric(int j, int i) const {
        return __ldg(metric + (size_t)j * g.xi + i);
    }
};

// ------------------------------------------------------------------ cell-column layout
// FP32 step layout. For every cell (j, i) and W level L the bracketing pair is stored at the
// four corners of the cell, corner order (j,i), (j+1,i), (j+1,i+1), (j,i+1):
//     A(L) = u, v of rho level L-1        B(L) = w, akt of W level L
// each as {field0 @ t0, field0 @ t1, field1 @ t0, field1 @ t1} x 4 corners, and the records of a
// cell are consecutive in L: ... A(L-1) B(L-1) A(L) B(L) ... so the stencil of a particle at
// level kI (L = kI + sW - 1) is the contiguous run B(L-1), A(L), B(L) read from one address.
// Surface per cell: h at the corners, zeta at t0 and t1 at the corners.

template <int STORE>
struct CellQuad;  // one field pair at 4 corners x 2 records
template <>
struct alignas(16) CellQuad<STORE_F32> {
    float4 a0, a1, b0, b1;  // field a @t0 corners, a @t1, field b @t0, b @t1
};
template <>
struct alignas(16) CellQuad<STORE_F16> {
    __half2 a0[2], a1[2], b0[2], b1[2];
};
template <>
struct alignas(16) CellQuad<STORE_BF16> {
    __nv_bfloat162 a0[2], a1[2], b0[2], b1[2];
};

struct Quad {
    float c1, c2, c3, c4;
};
struct QuadPair {  // a field at 4 corners for the two bracketing records
    Quad t0, t1;
};

__device__ __forceinline__ Quad quad_of(float4 v) { return Quad{v.x, v.y, v.z, v.w}; }

template <int STORE>
__device__ __forceinline__ void load_quad(const CellQuad<STORE> *p, QuadPair &a, QuadPair &b);

template <>
__device__ __forceinline__ void load_quad<STORE_F32>(const CellQuad<STORE_F32> *p, QuadPair &a,
                                                     QuadPair &b) {
    const float4 *q = reinterpret_cast<const float4 *>(p);
    a.t0 = quad_of(__ldg(q));
    a.t1 = quad_of(__ldg(q + 1));
    b.t0 = quad_of(__ldg(q + 2));
    b.t1 = quad_of(__ldg(q + 3));
}

__device__ __forceinline__ Quad quad_h(uint32_t x, uint32_t y) {
    float2 lo = __half22float2(*reinterpret_cast<__half2 *>(&x));
    float2 hi = __half22float2(*reinterpret_cast<__half2 *>(&y));
    return Quad{lo.x, lo.y, hi.x, hi.y};
}
__device__ __forceinline__ Quad quad_bf(uint32_t x, uint32_t y) {
    float2 lo = __bfloat1622float2(*reinterpret_cast<__nv_bfloat162 *>(&x));
    float2 hi = __bfloat1622float2(*reinterpret_cast<__nv_bfloat162 *>(&y));
    return Quad{lo.x, lo.y, hi.x, hi.y};
}

template <>
__device__ __forceinline__ void load_quad<STORE_F16>(const CellQuad<STORE_F16> *p, QuadPair &a,
                                                     QuadPair &b) {
    const uint4 *q = reinterpret_cast<const uint4 *>(p);
    uint4 x = __ldg(q), y = __ldg(q + 1);
    a.t0 = quad_h(x.x, x.y);
    a.t1 = quad_h(x.z, x.w);
    b.t0 = quad_h(y.x, y.y);
    b.t1 = quad_h(y.z, y.w);
}

template <>
__device__ __forceinline__ void load_quad<STORE_BF16>(const CellQuad<STORE_BF16> *p, QuadPair &a,
                                                      QuadPair &b) {
    const uint4 *q = reinterpret_cast<const uint4 *>(p);
    uint4 x = __ldg(q), y = __ldg(q + 1);
    a.t0 = quad_bf(x.x, x.y);
    a.t1 = quad_bf(x.z, x.w);
    b.t0 = quad_bf(y.x, y.y);
    b.t1 = quad_bf(y.z, y.w);
}

// The first field of a CellQuad only (w of a B record, without akt).
template <int STORE>
__device__ __forceinline__ void load_first(const CellQuad<STORE> *p, QuadPair &a);

template <>
__device__ __forceinline__ void load_first<STORE_F32>(const CellQuad<STORE_F32> *p, QuadPair &a) {
    const float4 *q = reinterpret_cast<const float4 *>(p);
    a.t0 = quad_of(__ldg(q));
    a.t1 = quad_of(__ldg(q + 1));
}

template <>
__device__ __forceinline__ void load_first<STORE_F16>(const CellQuad<STORE_F16> *p, QuadPair &a) {
    uint4 x = __ldg(reinterpret_cast<const uint4 *>(p));
    a.t0 = quad_h(x.x, x.y);
    a.t1 = quad_h(x.z, x.w);
}

template <>
__device__ __forceinline__ void load_first<STORE_BF16>(const CellQuad<STORE_BF16> *p, QuadPair &a) {
    uint4 x = __ldg(reinterpret_cast<const uint4 *>(p));
    a.t0 = quad_bf(x.x, x.y);
    a.t1 = quad_bf(x.z, x.w);
}

// The second field of a CellQuad only (akt of a B record, without w).
template <int STORE>
__device__ __forceinline__ void load_second(const CellQuad<STORE> *p, QuadPair &b);

template <>
__device__ __forceinline__ void load_second<STORE_F32>(const CellQuad<STORE_F32> *p, QuadPair &b) {
    const float4 *q = reinterpret_cast<const float4 *>(p);
    b.t0 = quad_of(__ldg(q + 2));
    b.t1 = quad_of(__ldg(q + 3));
}

template <>
__device__ __forceinline__ void load_second<STORE_F16>(const CellQuad<STORE_F16> *p, QuadPair &b) {
    uint4 y = __ldg(reinterpret_cast<const uint4 *>(p) + 1);
    b.t0 = quad_h(y.x, y.y);
    b.t1 = quad_h(y.z, y.w);
}

template <>
__device__ __forceinline__ void load_second<STORE_BF16>(const CellQuad<STORE_BF16> *p, QuadPair &b) {
    uint4 y = __ldg(reinterpret_cast<const uint4 *>(p) + 1);
    b.t0 = quad_bf(y.x, y.y);
    b.t1 = quad_bf(y.z, y.w);
}

struct CellSurface {  // FP32 at the 4 corners: h + zeta@t0, and zeta@t1 - zeta@t0
    float4 s0, dz;
};

template <int STORE>
struct CellView {
    int eta, xi, sW;
    const CellQuad<STORE> *columns;   // [cell][sW][2] (A, B)
    const CellSurface *surface;       // [cell]

    // Velocity stencil of level kI (valid memory level) in cell (j, i): u, v at rho level kI;
    // w, akt at W levels kI (up) and kI-1 (lo).
    __device__ __forceinline__ void stencil(int kI, int j, int i, QuadPair &u, QuadPair &v,
                                            QuadPair &wUp, QuadPair &aUp, QuadPair &wLo,
                                            QuadPair &aLo) const {
        size_t L = (size_t)(kI + sW - 1);
        const CellQuad<STORE> *col = columns + (((size_t)j * xi + i) * sW + L) * 2;
        load_quad<STORE>(col - 1, wLo, aLo);  // B(L-1)
        load_quad<STORE>(col, u, v);          // A(L)
        load_quad<STORE>(col + 1, wUp, aUp);  // B(L)
    }
    // The same without the diffusivity (deterministic steps).
    __device__ __forceinline__ void stencil_w(int kI, int j, int i, QuadPair &u, QuadPair &v,
                                              QuadPair &wUp, QuadPair &wLo) const {
        size_t L = (size_t)(kI + sW - 1);
        const CellQuad<STORE> *col = columns + (((size_t)j * xi + i) * sW + L) * 2;
        load_first<STORE>(col - 1, wLo);  // B(L-1)
        load_quad<STORE>(col, u, v);      // A(L)
        load_first<STORE>(col + 1, wUp);  // B(L)
    }
    __device__ __forceinline__ CellSurface surf(int j, int i) const {
        const float4 *q = reinterpret_cast<const float4 *>(surface + ((size_t)j * xi + i));
        return CellSurface{__ldg(q), __ldg(q + 1)};
    }
};

// Reference device layout (kernel.cu:63-69), whole window, records t0/t1 given per interval.
struct RawView {
    GridShape g;
    int t0, t1;
    const float *zeta, *u, *v, *w, *akt;
    const float *windU, *windV, *stokesU, *stokesV;
    const double *hField, *lonRad, *latRad, *depthIntervals;
    bool hasWindU, hasWindV, hasStokes;

    __device__ __forceinline__ size_t plane() const { return (size_t)g.eta * (size_t)g.xi; }
    __device__ __forceinline__ size_t i3(int t, int j, int i) const {
        return ((size_t)t * g.eta + j) * g.xi + i;
    }
    __device__ __forceinline__ size_t i4(int t, int storageLevel, int levels, int j, int i) const {
        return (((size_t)t * levels + storageLevel) * g.eta + j) * g.xi + i;
    }
    __device__ __forceinline__ NodeUp up(int kI, int j, int i) const {
        int Lw = kI + g.sW - 1, Lr = kI + g.sRho - 1;
        NodeUp n;
        n.u0 = __ldg(u + i4(t0, Lr, g.sRho, j, i));
        n.u1 = __ldg(u + i4(t1, Lr, g.sRho, j, i));
        n.v0 = __ldg(v + i4(t0, Lr, g.sRho, j, i));
        n.v1 = __ldg(v + i4(t1, Lr, g.sRho, j, i));
        n.w0 = __ldg(w + i4(t0, Lw, g.sW, j, i));
        n.w1 = __ldg(w + i4(t1, Lw, g.sW, j, i));
        n.a0 = __ldg(akt + i4(t0, Lw, g.sW, j, i));
        n.a1 = __ldg(akt + i4(t1, Lw, g.sW, j, i));
        return n;
    }
    __device__ __forceinline__ NodeLo lo(int kI, int j, int i) const {
        int Lw = kI + g.sW - 2;
        return NodeLo{__ldg(w + i4(t0, Lw, g.sW, j, i)), __ldg(w + i4(t1, Lw, g.sW, j, i)),
                      __ldg(akt + i4(t0, Lw, g.sW, j, i)), __ldg(akt + i4(t1, Lw, g.sW, j, i))};
    }
    __device__ __forceinline__ SurfPair surface(int j, int i) const {
        return SurfPair{__ldg(hField + (size_t)j * g.xi + i), __ldg(zeta + i3(t0, j, i)),
                        __ldg(zeta + i3(t1, j, i))};
    }
    __device__ __forceinline__ double h(int j, int i) const { return __ldg(hField + (size_t)j * g.xi + i); }
    __device__ __forceinline__ EnvPair environment(int j, int i) const {
        EnvPair e{0, 0, 0, 0, 0, 0, 0, 0};
        if (hasWindU) { e.wu0 = __ldg(windU + i3(t0, j, i)); e.wu1 = __ldg(windU + i3(t1, j, i)); }
        if (hasWindV) { e.wv0 = __ldg(windV + i3(t0, j, i)); e.wv1 = __ldg(windV + i3(t1, j, i)); }
        if (hasStokes) {
            e.su0 = __ldg(stokesU + i3(t0, j, i)); e.su1 = __ldg(stokesU + i3(t1, j, i));
            e.sv0 = __ldg(stokesV + i3(t0, j, i)); e.sv1 = __ldg(stokesV + i3(t1, j, i));
        }
        return e;
    }
    __device__ __forceinline__ double lon(int j, int i) const { return __ldg(lonRad + (size_t)j * g.xi + i); }
    __device__ __forceinline__ double lat(int j, int i) const { return __ldg(latRad + (size_t)j * g.xi + i); }
    __device__ __forceinline__ double depth_interval(int kI) const {
        return __ldg(depthIntervals + (kI + g.sW - 2));
    }
    // Full haversine between the nodes of the cell's edges (kernel.cu:145-149,278-279).
    __device__ __forceinline__ double2 cell_metric(int j, int i) const {
        double lat0 = lat(j, i), lon0 = lon(j, i);
        double latN = lat(j + 1, i), lonN = lon(j + 1, i);
        double latE = lat(j, i + 1), lonE = lon(j, i + 1);
        double dLat = latN - lat0, dLon = lonN - lon0;
        double value = sin(.5 * dLat) * sin(.5 * dLat) + sin(.5 * dLon) * sin(.5 * dLon) * cos(latN) * cos(lat0);
        double ydist = 2.0 * atan2(sqrt(value), sqrt(1.0 - value)) * 6371000.0;
        dLat = latE - lat0;
        dLon = lonE - lon0;
        value = sin(.5 * dLat) * sin(.5 * dLat) + sin(.5 * dLon) * sin(.5 * dLon) * cos(latE) * cos(lat0);
        double xdist = 2.0 * atan2(sqrt(value), sqrt(1.0 - value)) * 6371000.0;
        return make_double2(xdist, ydist);
    }
};

}  // namespace wb
