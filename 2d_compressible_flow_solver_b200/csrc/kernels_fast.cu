// Kernels of the throughput forms: FP64 with FMA contraction and the
// FP32-mixed form.  Built with FMA contraction on (nvcc default).
#include "cfs_kernels.cuh"
#include "cfs_launch.h"

namespace cfs {

namespace {
inline dim3 stage_grid(const Layout& L) {
    return dim3((L.ny + kTileJ - 1) / kTileJ, (L.nx + kTileI - 1) / kTileI);
}
}  // namespace

cudaError_t launch_stage_f64(const StageArgs& a, cudaStream_t s) {
    stage_kernel<PolF64, kTileI, kTileJ><<<stage_grid(a.L), kTileI * kTileJ, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_stage_f32(const StageArgs& a, cudaStream_t s) {
    stage_kernel<PolF32, kTileI, kTileJ><<<stage_grid(a.L), kTileI * kTileJ, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_weno_faces_f64(int n, const double* st, double* l, double* r, double g, double eps, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    weno_faces_kernel<PolF64><<<(n + 127) / 128, 128, 0, s>>>(n, st, l, r, g, eps);
    return cudaGetLastError();
}

cudaError_t launch_weno_faces_f32(int n, const double* st, double* l, double* r, double g, double eps, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    weno_faces_kernel<PolF32><<<(n + 127) / 128, 128, 0, s>>>(n, st, l, r, g, eps);
    return cudaGetLastError();
}

cudaError_t launch_hll_faces_f64(int n, int dir, const double* L, const double* R, double* F, double g, int v,
                                 cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    hll_faces_kernel<PolF64><<<(n + 127) / 128, 128, 0, s>>>(n, dir, L, R, F, g, v);
    return cudaGetLastError();
}

cudaError_t launch_hll_faces_f32(int n, int dir, const double* L, const double* R, double* F, double g, int v,
                                 cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    hll_faces_kernel<PolF32><<<(n + 127) / 128, 128, 0, s>>>(n, dir, L, R, F, g, v);
    return cudaGetLastError();
}

}  // namespace cfs
