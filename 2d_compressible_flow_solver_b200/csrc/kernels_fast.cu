// Kernels of the throughput forms: FP64 with FMA contraction and the
// FP32-mixed form.  Built with FMA contraction on (nvcc default).
#include "cfs_kernels.cuh"
#include "cfs_launch.h"
#include "cfs_march.cuh"

namespace cfs {

template <class Pol, int R, int W, int B, int Ld>
cudaError_t launch_march(const StageArgs& a, cudaStream_t s) {
    const int nseg = (a.L.ny + kSeg - 1) / kSeg;
    const dim3 grid((nseg + W - 1) / W, (a.L.nx + R - 1) / R);
    march_kernel<Pol, R, W, B, Ld><<<grid, 32 * W, 0, s>>>(a);
    return cudaGetLastError();
}

template <class Pol, int K>
cudaError_t launch_march_k(const StageArgs& a, cudaStream_t s) {
    constexpr MarchVariant v = kVariants[K];
    return launch_march<Pol, v.rows, v.warps, v.min_blocks, v.load>(a, s);
}

template <class Pol>
cudaError_t launch_march_variant(const StageArgs& a, int v, cudaStream_t s) {
    static_assert(kNumVariants == 20, "variant table and dispatch disagree");
    switch (v) {
        case 1: return launch_march_k<Pol, 0>(a, s);
        case 2: return launch_march_k<Pol, 1>(a, s);
        case 3: return launch_march_k<Pol, 2>(a, s);
        case 4: return launch_march_k<Pol, 3>(a, s);
        case 5: return launch_march_k<Pol, 4>(a, s);
        case 6: return launch_march_k<Pol, 5>(a, s);
        case 7: return launch_march_k<Pol, 6>(a, s);
        case 8: return launch_march_k<Pol, 7>(a, s);
        case 9: return launch_march_k<Pol, 8>(a, s);
        case 10: return launch_march_k<Pol, 9>(a, s);
        case 11: return launch_march_k<Pol, 10>(a, s);
        case 12: return launch_march_k<Pol, 11>(a, s);
        case 13: return launch_march_k<Pol, 12>(a, s);
        case 14: return launch_march_k<Pol, 13>(a, s);
        case 15: return launch_march_k<Pol, 14>(a, s);
        case 16: return launch_march_k<Pol, 15>(a, s);
        case 17: return launch_march_k<Pol, 16>(a, s);
        case 18: return launch_march_k<Pol, 17>(a, s);
        case 19: return launch_march_k<Pol, 18>(a, s);
        case 20: return launch_march_k<Pol, 19>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_stage_f64(const StageArgs& a, cudaStream_t s) {
    return launch_march_variant<PolF64>(a, a.variant > 0 ? a.variant : kDefaultVariantF64, s);
}

cudaError_t launch_stage_f32(const StageArgs& a, cudaStream_t s) {
    return launch_march_variant<PolF32>(a, a.variant > 0 ? a.variant : kDefaultVariantF32, s);
}

cudaError_t launch_batch_stage(Prec p, const StageArgs* args, const int* item_case, const int* item_local,
                               const int* case_rows, const int* case_items_x, int total, unsigned int* counter,
                               int grid, cudaStream_t s) {
    if (total <= 0) return cudaSuccess;
    if (p == kF32Mixed)
        batch_march_kernel<PolF32, kBatchWarps, kBatchMinBlocksF32, kBatchLoadF32><<<grid, 32 * kBatchWarps, 0, s>>>(
            args, item_case, item_local, case_rows, case_items_x, total, counter);
    else
        batch_march_kernel<PolF64, kBatchWarps, kBatchMinBlocksF64><<<grid, 32 * kBatchWarps, 0, s>>>(
            args, item_case, item_local, case_rows, case_items_x, total, counter);
    return cudaGetLastError();
}

int batch_blocks_per_sm(Prec p) {
    int n = 0;
    if (p == kF32Mixed)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_march_kernel<PolF32, kBatchWarps, kBatchMinBlocksF32, kBatchLoadF32>,
                                                      32 * kBatchWarps, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_march_kernel<PolF64, kBatchWarps, kBatchMinBlocksF64>,
                                                      32 * kBatchWarps, 0);
    return n > 0 ? n : 1;
}

constexpr int kViscTI = 8;
constexpr int kViscTJ = 32;

inline dim3 visc_grid(const Layout& L) {
    return dim3((L.ny + kViscTJ - 1) / kViscTJ, (L.nx + kViscTI - 1) / kViscTI);
}

cudaError_t launch_viscous_f64(const ViscArgs& a, cudaStream_t s) {
    viscous_kernel<PolF64, kViscTI, kViscTJ><<<visc_grid(a.L), kViscTI * kViscTJ, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_viscous_f32(const ViscArgs& a, cudaStream_t s) {
    viscous_kernel<PolF32, kViscTI, kViscTJ><<<visc_grid(a.L), kViscTI * kViscTJ, 0, s>>>(a);
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
