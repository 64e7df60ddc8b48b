// CFL time step for callers that cannot allocate device memory.
//
// Some callers of this library must not call cudaMalloc: a host code that owns
// every device allocation through its own pool or arena (and forbids others
// from allocating behind its back), code running where an allocation could
// stall or fail at a bad moment (inside a time-critical loop, under a memory
// budget already spent on the grid), or a caller that only holds a device
// pointer to a state it does not own.  cfs_compute_dt needs a context, and a
// context allocates.  cfs_compute_dt_static computes the same time step from a
// caller-owned device state and allocates nothing: its scratch is the
// file-scope array below, which every GPU that loads this library holds until
// the process exits.
//
// Built with -fmad=false, like the context's reduction, so the per-cell wave
// speed sum and hence dt are the same bits as cfs_compute_dt's for a state
// held by an FP64 or FP64_EXACT context (an FP32-mixed context reduces its
// FP32-rounded, offset storage instead).  Every call copies dt to pageable
// host memory and waits for the stream, so no call may be made on a stream
// that is being captured into a CUDA graph.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "cfs.h"

namespace cfs {
void record_global_error(int code, const std::string& msg);  // cfs_api.cpp
}

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 2048;
constexpr int kCellsPerThread = 32;
constexpr long long kMaxCells = static_cast<long long>(kMaxBlocks) * kThreads * kCellsPerThread;  // 4096 x 4096

// One partial maximum per block (FP64 bit patterns; the sums are non-negative,
// so their bit patterns order like the values), plus the final maximum.
// Every launch writes every slot it later reads, so nothing has to start at zero.
static __device__ __align__(256) unsigned long long g_cfl_scratch[kMaxBlocks + 1];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned long long* g_scratch_addr[kMaxDevices] = {};

__device__ __forceinline__ double wave_sum_static(double rho, double mx, double my, double E, double g, double dx,
                                                  double dy) {
    const double p = (g - 1) * (E - 0.5 * (mx * mx + my * my) / rho);
    const double a = sqrt(g * p / rho);
    const double u = mx / rho, v = my / rho;
    return (fabs(u) + a) / dx + (fabs(v) + a) / dy;
}

__device__ __forceinline__ double block_max_static(double m, double* red) {
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = m;
    __syncthreads();
    if (w == 0) {
        m = (l < kThreads / 32) ? red[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    return m;
}

// Block b reduces cells [b*kThreads*kCellsPerThread, (b+1)*kThreads*kCellsPerThread)
// of U[4][n] (n = nx*ny cells, reference order) into scratch[b].
__global__ void __launch_bounds__(kThreads) cfl_partial_kernel(const double* U, const uint8_t* types, long long n,
                                                               double g, double dx, double dy,
                                                               unsigned long long* scratch) {
    __shared__ double red[kThreads / 32];
    double m = 0.0;
    const long long base = static_cast<long long>(blockIdx.x) * kThreads * kCellsPerThread + threadIdx.x;
    for (int c = 0; c < kCellsPerThread; ++c) {
        const long long k = base + static_cast<long long>(c) * kThreads;
        if (k >= n) break;
        if (types && types[k] != 0) continue;
        // a non-finite sum (a blown-up cell) counts as +infinity: dt becomes 0
        // and the call reports CFS_ERR_NUMERIC, as cfs_compute_dt does
        double w = wave_sum_static(U[k], U[n + k], U[2 * n + k], U[3 * n + k], g, dx, dy);
        if (!(w == w)) w = __longlong_as_double(0x7ff0000000000000LL);
        if (w > m) m = w;
    }
    m = block_max_static(m, red);
    if (threadIdx.x == 0) scratch[blockIdx.x] = static_cast<unsigned long long>(__double_as_longlong(m));
}

// One block: maximum of scratch[0 .. nb) into scratch[kMaxBlocks].
__global__ void __launch_bounds__(kThreads) cfl_final_kernel(int nb, unsigned long long* scratch) {
    __shared__ double red[kThreads / 32];
    double m = 0.0;
    for (int b = threadIdx.x; b < nb; b += kThreads) {
        const double v = __longlong_as_double(static_cast<long long>(scratch[b]));
        if (v > m) m = v;
    }
    m = block_max_static(m, red);
    if (threadIdx.x == 0) scratch[kMaxBlocks] = static_cast<unsigned long long>(__double_as_longlong(m));
}

// Device address of g_cfl_scratch on the current device.  The array's name in
// host code is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, taken once per device with that device current.
cudaError_t scratch_on_current_device(unsigned long long** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_cfl_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = static_cast<unsigned long long*>(p);
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

int fail_static(int code, const std::string& msg) {
    cfs::record_global_error(code, msg);
    return code;
}

}  // namespace

extern "C" int cfs_compute_dt_static(const double* U, const uint8_t* types, int nx, int ny, double lx, double ly,
                                     double gamma, double cfl, void* stream, double* dt) {
    if (!U || !dt) return fail_static(CFS_ERR_INVALID, "cfs_compute_dt_static: null state or output pointer");
    if (nx < 1 || ny < 1 || !(lx > 0) || !(ly > 0) || !(gamma > 1.0) || !(cfl > 0))
        return fail_static(CFS_ERR_INVALID, "cfs_compute_dt_static: bad grid, gamma or cfl");
    const long long n = static_cast<long long>(nx) * ny;
    if (n > kMaxCells)
        return fail_static(CFS_ERR_INVALID, "cfs_compute_dt_static: " + std::to_string(n) +
                                                " cells exceed the static scratch limit of " +
                                                std::to_string(kMaxCells) + " cells (4096 x 4096)");
    unsigned long long* scratch = nullptr;
    cudaError_t e = scratch_on_current_device(&scratch);
    if (e != cudaSuccess) return fail_static(CFS_ERR_CUDA, std::string("cfs_compute_dt_static: ") + cudaGetErrorString(e));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long per_block = static_cast<long long>(kThreads) * kCellsPerThread;
    const int nb = static_cast<int>((n + per_block - 1) / per_block);
    cfl_partial_kernel<<<nb, kThreads, 0, s>>>(U, types, n, gamma, lx / nx, ly / ny, scratch);
    cfl_final_kernel<<<1, kThreads, 0, s>>>(nb, scratch);
    unsigned long long bits = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, scratch + kMaxBlocks, sizeof(bits), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail_static(CFS_ERR_CUDA, std::string("cfs_compute_dt_static: ") + cudaGetErrorString(e));
    double m;
    std::memcpy(&m, &bits, sizeof(m));
    if (!(m > 0) || !std::isfinite(m))
        return fail_static(CFS_ERR_NUMERIC, "cfs_compute_dt_static: a fluid cell is non-finite or every wave speed is 0");
    *dt = cfl / m;
    return CFS_OK;
}
