// A drop-in move that never allocates device memory.
//
// Who needs it: host programs that may not call cudaMalloc/cudaFree while they drive the
// particle step. cudaFree synchronizes the whole device and cudaMalloc may too, which stalls
// every other stream a multi-GPU or multi-stream driver keeps in flight (the reference runs one
// stream per GPU section, Wacomm.cpp:529-609); and some host frameworks own all device memory
// through their own pool and forbid the CUDA allocator outright. Such callers pass their inputs and
// outputs; the only working memory this entry point touches is a fixed array compiled into the
// library.
//
// What it does: the same update as wacomm_b200_cuda_move_particle (device rules, reference
// arithmetic, the caller's particle_data records updated in place), but it first orders the work
// by horizontal cell -- key per record, histogram, exclusive scan, scatter -- so that the
// threads of a warp gather the same forcing cells. Keys, histogram, offsets, scan partials and
// the work order live in `noalloc_scratch` below.
//
// Limits: at most NOALLOC_MAX_PARTICLES records and NOALLOC_MAX_CELLS horizontal cells (eta*xi)
// per call; larger calls are refused with -WACOMM_B200_ERR_CAPACITY before any work. The array
// (about 25 MB) is held on every GPU that loads the library until the process exits. A grid with
// fewer than two nodes along an axis has no interpolation cell: its records are moved in caller
// order without the sort (every one of them leaves the grid), as the drop-in launcher does.
//
// Sharing: every call on a device uses the same array and leaves its contents behind; the
// histogram is cleared at the start of each call. Two calls whose work overlaps on the GPU (on
// different streams, or from different host threads without ordering) race on the array and
// must not be issued; calls on one stream are ordered and safe.
//
// Set-up: the first call made on a device, with that device current, looks up the array's
// device address with cudaGetSymbolAddress and the device's SM count, once; later calls reuse
// them. Under lazy module loading (the CUDA default) that first call is also the one that loads
// the library's kernels on the device and makes the array resident there, which allocates device
// memory and synchronizes once: make it during the caller's own set-up, before its
// allocation-free phase and before any stream capture begins on the device. The looked-up address
// belongs to the device's context of that moment; a cudaDeviceReset between calls is not
// supported.
//
// Compiled with -fmad=false like dropin.cu, so the moved records are the same as that entry
// point's, bit for bit.
#include <mutex>

#include "engine.h"
#include "move_kernels.cuh"

namespace wb {
namespace {

constexpr int NOALLOC_MAX_PARTICLES = 1 << 21;  // 2,097,152 records per call
constexpr int NOALLOC_MAX_CELLS = 1 << 20;      // 1,048,576 horizontal cells per call
constexpr size_t NOALLOC_SCAN_WORDS = 4096;     // scan partials for up to NOALLOC_MAX_CELLS + 1 bins
constexpr size_t NOALLOC_BINS = (size_t)NOALLOC_MAX_CELLS + 2;
constexpr size_t NOALLOC_WORDS =
    2 * (size_t)NOALLOC_MAX_PARTICLES + 2 * NOALLOC_BINS + NOALLOC_SCAN_WORDS;
constexpr int NOALLOC_MAX_DEVICES = 64;

// keys[MAXP] | order[MAXP] | histogram[BINS] | offsets[BINS] | scan partials
static __device__ __align__(256) uint32_t noalloc_scratch[NOALLOC_WORDS];

// What the first call on a device looks up: the array's device address and the SM count that
// sizes the grid-stride launches.
struct DeviceSetup {
    uint32_t *scratch = nullptr;
    int smCount = 0;
};

std::mutex setup_mutex;
DeviceSetup device_setup[NOALLOC_MAX_DEVICES];

// Set-up of the current device (done once per device, on its first call).
cudaError_t setup_for_current_device(DeviceSetup *out) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(setup_mutex);
    DeviceSetup &d = device_setup[device];
    if (!d.scratch) {
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess) return e;
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, noalloc_scratch);
        if (e != cudaSuccess) return e;
        d.smCount = sms > 0 ? sms : 1;
        d.scratch = static_cast<uint32_t *>(ptr);
    }
    *out = d;
    return cudaSuccess;
}

__global__ void noalloc_clear_kernel(uint32_t *hist, size_t bins) {
    for (size_t b = blockIdx.x * (size_t)blockDim.x + threadIdx.x; b < bins;
         b += (size_t)gridDim.x * blockDim.x)
        hist[b] = 0;
}

// Cell key of each record (last bin for records outside the interpolation cells) and the
// warp-aggregated histogram of the keys.
__global__ void noalloc_key_kernel(const wacomm_b200_particle *particles, int n, int eta, int xi,
                                   uint32_t *keys, uint32_t *hist) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        double fj = floor(particles[p].j), fi = floor(particles[p].i);
        uint32_t key = (fj >= 0.0 && fi >= 0.0 && fj < (double)(eta - 1) && fi < (double)(xi - 1))
                           ? (uint32_t)((int)fj * xi + (int)fi)
                           : (uint32_t)((size_t)eta * xi);
        keys[p] = key;
        unsigned peers = __match_any_sync(__activemask(), key);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(hist + key, (uint32_t)__popc(peers));
    }
}

__global__ void noalloc_scatter_kernel(const uint32_t *keys, int n, uint32_t *cursor,
                                       uint32_t *order) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        uint32_t key = keys[p];
        unsigned peers = __match_any_sync(__activemask(), key);
        int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(cursor + key, (uint32_t)__popc(peers));
        base = __shfl_sync(peers, base, leader);
        order[base + __popc(peers & ((1u << lane) - 1u))] = (uint32_t)p;
    }
}

// The drop-in step over the records in cell order (order null: caller order).
__global__ void __launch_bounds__(256) noalloc_move_kernel(
    const wacomm_b200_config *__restrict__ config, wacomm_b200_particle *particles,
    const uint32_t *__restrict__ order, int timeIndex, int oceanTime,
    const double *__restrict__ times, RawView V, int count) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const wacomm_b200_config &cfg = *config;
    IntervalParams P;
    make_interval(cfg, times, oceanTime, timeIndex, V.g.sW, SEM_DEVICE, P);
    if (P.skip) return;
    RawView view = V;
    view.t0 = P.t0;
    view.t1 = P.t1;
    uint32_t idx = order ? order[t] : (uint32_t)t;
    wacomm_b200_particle rec = particles[idx];
    ParticleState p;
    p.id = rec.id;
    p.k = rec.k;
    p.j = rec.j;
    p.i = rec.i;
    p.health = rec.health;
    p.age = rec.age;
    p.time = rec.time;
    p.type = rec.driftObjectType;
    p.side = rec.driftSide;
    double elapsed = P.elapsed0;
    move_particle<SEM_DEVICE, ARITH_REF>(cfg, P, view, p, elapsed, nullptr);
    rec.k = p.k;
    rec.j = p.j;
    rec.i = p.i;
    rec.health = p.health;
    rec.age = p.age;
    rec.driftSide = (int8_t)p.side;
    particles[idx] = rec;
}

}  // namespace
}  // namespace wb

// See the file comment. Same arguments and meaning as wacomm_b200_cuda_move_particle; returns 0,
// a CUDA error code, or -WACOMM_B200_ERR_CAPACITY (nothing done) when particle_count exceeds
// 2,097,152 or eta*xi exceeds 1,048,576 (on a grid with at least two nodes along each axis).
extern "C" int wacomm_b200_cuda_move_particle_noalloc(
    const wacomm_b200_config *config_device, wacomm_b200_particle *particles_device,
    int time_index, int ocean_time, int s_w, int s_rho, int eta, int xi, const double *times,
    const double *mask, const double *lon_rad, const double *lat_rad,
    const double *depth_intervals, const double *h, const float *zeta, const float *u,
    const float *v, const float *w, const float *akt, const float *wind_u10,
    const float *wind_v10, const float *stokes_u, const float *stokes_v, int particle_count,
    int num_thread, int num_gpu, void *stream_handle) {
    using namespace wb;
    (void)mask;
    (void)num_thread;
    (void)num_gpu;
    if (particle_count <= 0) return (int)cudaGetLastError();
    const bool sorted = eta >= 2 && xi >= 2;  // else no interpolation cell: caller order
    if (particle_count > NOALLOC_MAX_PARTICLES ||
        (sorted && (size_t)eta * (size_t)xi > (size_t)NOALLOC_MAX_CELLS))
        return -WACOMM_B200_ERR_CAPACITY;
    size_t bins = sorted ? (size_t)eta * xi + 1 : 0;
    if (sorted && scan_temp_words(bins) > NOALLOC_SCAN_WORDS) return -WACOMM_B200_ERR_CAPACITY;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
    DeviceSetup setup;
    cudaError_t e = setup_for_current_device(&setup);
    if (e != cudaSuccess) return (int)e;
    uint32_t *order = nullptr;
    if (sorted) {
        uint32_t *keys = setup.scratch;
        uint32_t *hist = keys + 2 * (size_t)NOALLOC_MAX_PARTICLES;
        uint32_t *offsets = hist + NOALLOC_BINS;
        uint32_t *partials = offsets + NOALLOC_BINS;
        order = keys + NOALLOC_MAX_PARTICLES;
        // grid-stride kernels: at most 16 blocks of 256 threads per SM
        const int cap = setup.smCount * 16;
        int blocks = (particle_count + 255) / 256;
        if (blocks > cap) blocks = cap;
        int clearBlocks = (int)((bins + 255) / 256);
        if (clearBlocks > cap) clearBlocks = cap;
        noalloc_clear_kernel<<<clearBlocks, 256, 0, stream>>>(hist, bins);
        noalloc_key_kernel<<<blocks, 256, 0, stream>>>(particles_device, particle_count, eta, xi,
                                                       keys, hist);
        e = exclusive_scan(hist, offsets, bins, offsets + bins, partials, stream);
        if (e != cudaSuccess) return (int)e;
        noalloc_scatter_kernel<<<blocks, 256, 0, stream>>>(keys, particle_count, offsets, order);
    }

    RawView V;
    V.g = GridShape{eta, xi, s_w, s_rho};
    V.t0 = V.t1 = 0;
    V.zeta = zeta;
    V.u = u;
    V.v = v;
    V.w = w;
    V.akt = akt;
    V.windU = wind_u10;
    V.windV = wind_v10;
    V.stokesU = stokes_u;
    V.stokesV = stokes_v;
    V.hField = h;
    V.lonRad = lon_rad;
    V.latRad = lat_rad;
    V.depthIntervals = depth_intervals;
    V.hasWindU = wind_u10 != nullptr;
    V.hasWindV = wind_v10 != nullptr;
    V.hasStokes = stokes_u != nullptr && stokes_v != nullptr;
    noalloc_move_kernel<<<(particle_count + 127) / 128, 128, 0, stream>>>(
        config_device, particles_device, order, time_index, ocean_time, times, V, particle_count);
    return (int)cudaGetLastError();
}
