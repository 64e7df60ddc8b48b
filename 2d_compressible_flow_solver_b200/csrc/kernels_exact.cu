// Kernels whose FP64 rounding must follow the reference's operation order:
// built with -fmad=false so no multiply-add is contracted, IEEE division and
// square root (nvcc defaults).  Holds the CFS_FP64_EXACT stage, the immersed-
// ghost fill, the CFL reduction and the layout helpers for both storage types.
#include "cfs_kernels.cuh"
#include "cfs_launch.h"

namespace cfs {

namespace {
inline dim3 stage_grid(const Layout& L) {
    return dim3((L.ny + kTileJ - 1) / kTileJ, (L.nx + kTileI - 1) / kTileI);
}
inline int flat_blocks(long long work, int nt) {
    long long b = (work + nt - 1) / nt;
    if (b < 1) b = 1;
    if (b > 148 * 16) b = 148 * 16;
    return static_cast<int>(b);
}
}  // namespace

cudaError_t launch_stage_exact(const StageArgs& a, cudaStream_t s) {
    stage_kernel<PolExact, kTileI, kTileJ><<<stage_grid(a.L), kTileI * kTileJ, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_ib_fill(int elem_bytes, const IbArgs& a, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    const int nt = 128, nb = (a.n + nt - 1) / nt;
    if (elem_bytes == 8) ib_fill_kernel<double><<<nb, nt, 0, s>>>(a);
    else ib_fill_kernel<float><<<nb, nt, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_batch_ib_fill(int elem_bytes, const IbArgs* args, const int* cases, const int* local, int total,
                                 cudaStream_t s) {
    if (total <= 0) return cudaSuccess;
    const int nt = 128, nb = (total + nt - 1) / nt;
    if (elem_bytes == 8) batch_ib_fill_kernel<double><<<nb, nt, 0, s>>>(args, cases, local, total);
    else batch_ib_fill_kernel<float><<<nb, nt, 0, s>>>(args, cases, local, total);
    return cudaGetLastError();
}

cudaError_t launch_wmax(int elem_bytes, const void* U, const Layout& L, const uint8_t* types, double g, double dx,
                        double dy, unsigned long long* out, cudaStream_t s) {
    constexpr int nt = 256;
    const int nb = flat_blocks(static_cast<long long>(L.nx) * L.ny, nt);
    if (elem_bytes == 8) wmax_kernel<double, nt><<<nb, nt, 0, s>>>(static_cast<const double*>(U), L, types, g, dx, dy, out);
    else wmax_kernel<float, nt><<<nb, nt, 0, s>>>(static_cast<const float*>(U), L, types, g, dx, dy, out);
    return cudaGetLastError();
}

cudaError_t launch_batch_wmax(int elem_bytes, const StageArgs* args, int ncases, cudaStream_t s) {
    constexpr int nt = 256, per_case = 64;
    for (int c0 = 0; c0 < ncases; c0 += 65535) {  // gridDim.y limit
        const int nc = ncases - c0 < 65535 ? ncases - c0 : 65535;
        if (elem_bytes == 8) batch_wmax_kernel<double, nt><<<dim3(per_case, nc), nt, 0, s>>>(args + c0);
        else batch_wmax_kernel<float, nt><<<dim3(per_case, nc), nt, 0, s>>>(args + c0);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Sums of the four planes of a host-order FP64 state [4][n], in a fixed order
// (the same bits on every run): kSumBlocks strided partial sums per plane,
// each reduced as a tree in its block, then the partials added in index order.
constexpr int kSumBlocks = 256, kSumThreads = 256;

__global__ void __launch_bounds__(kSumThreads) plane_partial_sums_kernel(const double* U, long long n, double* partial) {
    __shared__ double red[kSumThreads];
    const int v = blockIdx.y;
    double s = 0.0;
    for (long long k = static_cast<long long>(blockIdx.x) * kSumThreads + threadIdx.x; k < n;
         k += static_cast<long long>(kSumBlocks) * kSumThreads)
        s += U[v * n + k];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = kSumThreads / 2; w > 0; w >>= 1) {
        if (static_cast<int>(threadIdx.x) < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[v * kSumBlocks + blockIdx.x] = red[0];
}

__global__ void plane_final_sums_kernel(const double* partial, double* out4) {
    const int v = threadIdx.x;
    if (v >= kVars) return;
    double s = 0.0;
    for (int b = 0; b < kSumBlocks; ++b) s += partial[v * kSumBlocks + b];
    out4[v] = s;
}

int plane_sums_scratch_doubles() { return kVars * kSumBlocks + kVars; }

cudaError_t launch_plane_sums(const double* U, long long n, double* scratch, cudaStream_t s) {
    plane_partial_sums_kernel<<<dim3(kSumBlocks, kVars), kSumThreads, 0, s>>>(U, n, scratch);
    plane_final_sums_kernel<<<1, 32, 0, s>>>(scratch, scratch + kVars * kSumBlocks);
    return cudaGetLastError();
}

cudaError_t launch_totals(int elem_bytes, const void* U, const Layout& L, const uint8_t* types, double* scratch,
                          double* out, cudaStream_t s) {
    const dim3 grid(kSumBlocks, kVars);
    if (elem_bytes == 8)
        totals_partial_kernel<double, kSumThreads, kSumBlocks><<<grid, kSumThreads, 0, s>>>(static_cast<const double*>(U), L, types, scratch);
    else
        totals_partial_kernel<float, kSumThreads, kSumBlocks><<<grid, kSumThreads, 0, s>>>(static_cast<const float*>(U), L, types, scratch);
    plane_final_sums_kernel<<<1, 32, 0, s>>>(scratch, out);
    return cudaGetLastError();
}

cudaError_t launch_pack(int elem_bytes, const double* src, void* dst, const Layout& L, cudaStream_t s) {
    const int nt = 256, nb = flat_blocks(4LL * L.nx * L.ny, nt);
    if (elem_bytes == 8) pack_kernel<double><<<nb, nt, 0, s>>>(src, static_cast<double*>(dst), L);
    else pack_kernel<float><<<nb, nt, 0, s>>>(src, static_cast<float*>(dst), L);
    return cudaGetLastError();
}

cudaError_t launch_unpack(int elem_bytes, const void* src, double* dst, const Layout& L, cudaStream_t s) {
    const int nt = 256, nb = flat_blocks(4LL * L.nx * L.ny, nt);
    if (elem_bytes == 8) unpack_kernel<double><<<nb, nt, 0, s>>>(static_cast<const double*>(src), dst, L);
    else unpack_kernel<float><<<nb, nt, 0, s>>>(static_cast<const float*>(src), dst, L);
    return cudaGetLastError();
}

cudaError_t launch_ghost_fill(int elem_bytes, void* U, const Layout& L, const BcSides& sides, cudaStream_t s) {
    const int per = L.nx > L.ny ? L.nx : L.ny;
    const int nt = 256, nb = flat_blocks(4LL * kGhost * per * kVars + 4LL * kGhost * kGhost * kVars, nt);
    if (elem_bytes == 8) ghost_fill_kernel<double><<<nb, nt, 0, s>>>(static_cast<double*>(U), L, sides);
    else ghost_fill_kernel<float><<<nb, nt, 0, s>>>(static_cast<float*>(U), L, sides);
    return cudaGetLastError();
}

cudaError_t launch_weno_faces_exact(int n, const double* st, double* l, double* r, double g, double eps, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    weno_faces_kernel<PolExact><<<(n + 127) / 128, 128, 0, s>>>(n, st, l, r, g, eps);
    return cudaGetLastError();
}

cudaError_t launch_hll_faces_exact(int n, int dir, const double* L, const double* R, double* F, double g, int v,
                                   cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    hll_faces_kernel<PolExact><<<(n + 127) / 128, 128, 0, s>>>(n, dir, L, R, F, g, v);
    return cudaGetLastError();
}

}  // namespace cfs
