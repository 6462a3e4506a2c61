// les_noalloc.cu -- lesgpu_monitor_noalloc: the monitor reductions of write_monitor_log
// (total mass, T/G range, minimum fuel fraction) for callers that cannot allocate device
// memory.
//
// Who needs it: a host that has handed every byte of HBM to fixed-size request slots (a
// serving loop admitting solves against a memory budget), or a caller on a latency-bound
// path where cudaMalloc's implicit device-wide synchronisation is not acceptable.  Such a
// caller owns the field arrays and a 6-double output buffer on the device and must not see
// the library allocate anything behind its back.
//
// Scratch lives in one file-scope __device__ array of kScratchDoubles doubles (3 MiB, for
// LESGPU_NOALLOC_MAX_CELLS cells), so every GPU that loads the library holds it until the
// process exits.  The array is shared by
// all calls on a device and keeps the previous call's contents; the completion counter at
// its start is cleared on every call, and the per-block partials are rewritten before they
// are read.  Calls whose work overlaps on the GPU (different streams, or different threads
// on one device) race on the array and must be serialised by the caller.  The scratch address
// is the current device's, so the stream and the buffers must belong to the current device;
// a mismatch is refused (LESGPU_EINVAL) rather than launched on another device's memory.
//
// Reductions: the minima and maxima start from the monitor's own +-1e9 sentinels (as
// write_monitor_log does, les_combustion_solver.c:3880-3897), so a field entirely beyond
// them reports the sentinel; fmin/fmax skip NaN operands, where the reference's comparisons
// would keep the first value -- the reference's NaN guard is check_for_nan, not the monitor.
#include <cuda_runtime.h>

#include <mutex>

#include "les_common.cuh"
#include "les_gpu.h"

namespace {

constexpr int kThreads = 256;
// At most 65536 blocks of 256 cells: grids of up to 16,777,216 cells.
constexpr size_t kMaxBlocks = LESGPU_NOALLOC_MAX_CELLS / kThreads;
// 256 bytes for the completion counter, then 6 partials per block.
constexpr size_t kScratchDoubles = 32 + 6 * kMaxBlocks;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device.  The array's name in host
// code is only a host-side stand-in, so the address is looked up once per device with
// cudaGetSymbolAddress (with that device current) and cached.
int scratch_for_current_device(double** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return LESGPU_ECUDA;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return LESGPU_ECUDA;
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return LESGPU_OK;
}

__global__ void __launch_bounds__(kThreads) k_monitor_noalloc(const double* __restrict__ rho, const double* __restrict__ T,
                                                              const double* __restrict__ G, const double* __restrict__ Y0,
                                                              size_t n, double dx, double dy, double dz,
                                                              double* __restrict__ scratch, double* __restrict__ out) {
    __shared__ double sh[kThreads / 32];
    __shared__ bool last;
    const int tid = threadIdx.x;
    const unsigned nb = gridDim.x;
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch);
    double* part = scratch + 32;
    const size_t id = (size_t)blockIdx.x * kThreads + tid;
    double mass = 0.0, tmin = 1.0e9, tmax = -1.0e9, gmin = 1.0e9, gmax = -1.0e9, ymin = 1.0e9;
    if (id < n) {
        mass = ((rho[id] * dx) * dy) * dz;
        tmin = tmax = T[id];
        gmin = gmax = G[id];
        ymin = Y0[id];
    }
    double v[6];
    v[0] = les::block_sum<kThreads>(mass, sh, tid);
    v[1] = les::block_min<kThreads>(tmin, sh, tid);
    v[2] = les::block_max<kThreads>(tmax, sh, tid);
    v[3] = les::block_min<kThreads>(gmin, sh, tid);
    v[4] = les::block_max<kThreads>(gmax, sh, tid);
    v[5] = les::block_min<kThreads>(ymin, sh, tid);
    if (tid == 0) {
        for (int q = 0; q < 6; q++) part[q * (size_t)nb + blockIdx.x] = v[q];
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        last = (t == nb - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc[6] = {0.0, 1.0e9, -1.0e9, 1.0e9, -1.0e9, 1.0e9};
    for (unsigned q = tid; q < nb; q += kThreads) {
        acc[0] += __ldcg(&part[q]);
        acc[1] = fmin(acc[1], __ldcg(&part[nb + q]));
        acc[2] = fmax(acc[2], __ldcg(&part[2 * (size_t)nb + q]));
        acc[3] = fmin(acc[3], __ldcg(&part[3 * (size_t)nb + q]));
        acc[4] = fmax(acc[4], __ldcg(&part[4 * (size_t)nb + q]));
        acc[5] = fmin(acc[5], __ldcg(&part[5 * (size_t)nb + q]));
    }
    acc[0] = les::block_sum<kThreads>(acc[0], sh, tid);
    acc[1] = les::block_min<kThreads>(acc[1], sh, tid);
    acc[2] = les::block_max<kThreads>(acc[2], sh, tid);
    acc[3] = les::block_min<kThreads>(acc[3], sh, tid);
    acc[4] = les::block_max<kThreads>(acc[4], sh, tid);
    acc[5] = les::block_min<kThreads>(acc[5], sh, tid);
    if (tid == 0) {
        for (int q = 0; q < 6; q++) out[q] = acc[q];
        *counter = 0u;
    }
}

}  // namespace

extern "C" int lesgpu_monitor_noalloc(const double* rho, const double* T, const double* G, const double* Y0, size_t n,
                                      double dx, double dy, double dz, double* out, void* stream) {
    if (!rho || !T || !G || !Y0 || !out || n == 0) return LESGPU_EINVAL;
    if (n > (size_t)LESGPU_NOALLOC_MAX_CELLS) return LESGPU_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return LESGPU_ECUDA;
    // the output must be device memory of the current device, and so must the stream's device
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, out) != cudaSuccess) {
        cudaGetLastError();
        return LESGPU_EINVAL;
    }
    if ((pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged) || pa.device != dev) return LESGPU_EINVAL;
    if (st) {
        int sdev = -1;
        if (cudaStreamGetDevice(st, &sdev) != cudaSuccess) {
            cudaGetLastError();
            return LESGPU_EINVAL;
        }
        if (sdev != dev) return LESGPU_EINVAL;
    }
    double* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc != LESGPU_OK) return rc;
    // the completion counter must start at zero on every call
    if (cudaMemsetAsync(scratch, 0, 256, st) != cudaSuccess) return LESGPU_ECUDA;
    const unsigned nb = (unsigned)((n + kThreads - 1) / kThreads);
    k_monitor_noalloc<<<nb, kThreads, 0, st>>>(rho, T, G, Y0, n, dx, dy, dz, scratch, out);
    if (cudaGetLastError() != cudaSuccess) return LESGPU_ECUDA;
    return LESGPU_OK;
}
