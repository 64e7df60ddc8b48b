// Kernels of the throughput forms: FP64 with FMA contraction and the
// FP32-mixed form.  Built with FMA contraction on (nvcc default).
#include <atomic>

#include "cfs_kernels.cuh"
#include "cfs_launch.h"
#include "cfs_march.cuh"

namespace cfs {

// Boundary-face fluxes of the stage (physical sides only), then the row march
// of the stage's feature set.
template <class Pol>
cudaError_t launch_boundary_flux(const StageArgs& a, cudaStream_t s) {
    if (!(physical_side(a, 0) || physical_side(a, 1) || physical_side(a, 2) || physical_side(a, 3)))
        return cudaSuccess;
    if (!a.bflux) return cudaErrorInvalidValue;
    const int n = a.L.nx > a.L.ny ? a.L.nx : a.L.ny;
    boundary_flux_kernel<Pol><<<dim3((n + 127) / 128, 4), 128, 0, s>>>(a);
    return cudaGetLastError();
}

// SM count of the current device (cached per device).
int sm_count() {
    constexpr int kMaxDev = 64;
    static std::atomic<int> count[kMaxDev] = {};  // every writer stores the same value
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return 148;
    int c = count[dev].load(std::memory_order_relaxed);
    if (c == 0) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        c = n > 0 ? n : 148;
        count[dev].store(c, std::memory_order_relaxed);
    }
    return c;
}

// The FP64 default variant stages rows in a shared ring, kRingBlocksPerSmF64
// blocks per SM.  When its grid fills more than one but fewer than three such
// waves and the last one is under half full, the register-window variant
// finishes first (measured with the earlier 3-block ring on the Mach-3
// cylinder, 2048 x 1024: 2,105 against 1,832 Mcell-steps/s; the 4-block ring
// now fills that grid in one wave and runs it at 2,376).
int default_variant_f64(const Layout& L, int rows) {
    const MarchVariant& d = kVariants[kDefaultVariantF64 - 1];
    const long long nseg = (L.ny + kSeg - 1) / kSeg;
    const long long blocks = (nseg * ((L.nx + rows - 1) / rows) + d.warps - 1) / d.warps;
    const double waves = static_cast<double>(blocks) / (static_cast<double>(sm_count()) * kRingBlocksPerSmF64);
    if (waves > 1.0 && waves < 3.0 && waves - static_cast<double>(static_cast<long long>(waves)) < 0.5)
        return kWindowVariantF64;
    return kDefaultVariantF64;
}

cudaError_t launch_stage_f64(const StageArgs& a, cudaStream_t s) {
    const cudaError_t e = launch_boundary_flux<PolF64>(a, s);
    if (e != cudaSuccess) return e;
    // (with the row chunk chosen per launch to fill whole waves, the ring
    // variant stays; the fallback serves fixed chunks)
    const int v = a.variant > 0 ? a.variant : a.rows > 0 ? default_variant_f64(a.L, a.rows) : kDefaultVariantF64;
    switch (march_features(a)) {
        case 0: return launch_march_f64_0(a, v, s);
        case 1: return launch_march_f64_1(a, v, s);
        case 2: return launch_march_f64_2(a, v, s);
        case 3: return launch_march_f64_3(a, v, s);
        case 4: return launch_march_f64_4(a, v, s);
        case 5: return launch_march_f64_5(a, v, s);
        case 6: return launch_march_f64_6(a, v, s);
        default: return launch_march_f64_7(a, v, s);
    }
}

cudaError_t launch_stage_f32(const StageArgs& a, cudaStream_t s) {
    const cudaError_t e = launch_boundary_flux<PolF32>(a, s);
    if (e != cudaSuccess) return e;
    const int v = a.variant > 0 ? a.variant : (march_features(a) & kFeatEdge) ? kEdgeVariantF32 : kDefaultVariantF32;
    switch (march_features(a)) {
        case 0: return launch_march_f32_0(a, v, s);
        case 1: return launch_march_f32_1(a, v, s);
        case 2: return launch_march_f32_2(a, v, s);
        case 3: return launch_march_f32_3(a, v, s);
        case 4: return launch_march_f32_4(a, v, s);
        case 5: return launch_march_f32_5(a, v, s);
        case 6: return launch_march_f32_6(a, v, s);
        default: return launch_march_f32_7(a, v, s);
    }
}

// The batch's feature set is common to its cases: positivity, and the edge
// code when some case has a physical side or cell types (batches keep no RHS
// and have no viscous terms).
// Dynamic shared memory of a batched march (the FP64 ring), 0 for the others.
template <class Pol, int kLoad>
constexpr size_t batch_dyn_bytes() {
    return (kLoad == 3 && sizeof(typename Pol::T) == 8) ? static_cast<size_t>(kBatchWarps) * ring_words<double>() * 8 : 0;
}

template <class Kernel>
cudaError_t allow_dyn(Kernel k, size_t bytes) {
    if (bytes == 0) return cudaSuccess;
    return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}

template <class Pol, int kMinBlocks, int kLoad>
cudaError_t launch_batch_march(const StageArgs* args, const int* item_case, const int* item_local,
                               const int* case_rows, const int* case_nseg, int total, unsigned int* counter,
                               int grid, int feat, cudaStream_t s) {
    constexpr size_t dyn = batch_dyn_bytes<Pol, kLoad>();
    cudaError_t e = cudaSuccess;
    switch (feat) {
        case 0: e = allow_dyn(batch_march_kernel<Pol, kBatchWarps, kMinBlocks, kLoad, 0>, dyn); break;
        case kFeatPos: e = allow_dyn(batch_march_kernel<Pol, kBatchWarps, kMinBlocks, kLoad, kFeatPos>, dyn); break;
        case kFeatEdge: e = allow_dyn(batch_march_kernel<Pol, kBatchWarps, kMinBlocks, kLoad, kFeatEdge>, dyn); break;
        case kFeatEdge | kFeatPos:
            e = allow_dyn(batch_march_kernel<Pol, kBatchWarps, kMinBlocks, kLoad, kFeatEdge | kFeatPos>, dyn);
            break;
        default: return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    switch (feat) {
        case 0:
            batch_march_kernel<Pol, kBatchWarps, kMinBlocks, kLoad, 0><<<grid, 32 * kBatchWarps, dyn, s>>>(
                args, item_case, item_local, case_rows, case_nseg, total, counter);
            break;
        case kFeatPos:
            batch_march_kernel<Pol, kBatchWarps, kMinBlocks, kLoad, kFeatPos><<<grid, 32 * kBatchWarps, dyn, s>>>(
                args, item_case, item_local, case_rows, case_nseg, total, counter);
            break;
        case kFeatEdge:
            batch_march_kernel<Pol, kBatchWarps, kMinBlocks, kLoad, kFeatEdge><<<grid, 32 * kBatchWarps, dyn, s>>>(
                args, item_case, item_local, case_rows, case_nseg, total, counter);
            break;
        case kFeatEdge | kFeatPos:
            batch_march_kernel<Pol, kBatchWarps, kMinBlocks, kLoad, kFeatEdge | kFeatPos><<<grid, 32 * kBatchWarps, dyn, s>>>(
                args, item_case, item_local, case_rows, case_nseg, total, counter);
            break;
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_batch_stage(Prec p, const StageArgs* args, const int* item_case, const int* item_local,
                               const int* case_rows, const int* case_nseg, int total, unsigned int* counter,
                               int grid, int feat, cudaStream_t s) {
    if (total <= 0) return cudaSuccess;
    if (p == kF32Mixed)
        return launch_batch_march<PolF32, kBatchMinBlocksF32, kBatchLoadF32>(args, item_case, item_local, case_rows,
                                                                             case_nseg, total, counter, grid, feat, s);
    return launch_batch_march<PolF64, kBatchMinBlocksF64, kBatchLoadF64>(args, item_case, item_local, case_rows,
                                                                         case_nseg, total, counter, grid, feat, s);
}

// Boundary-face fluxes of every case of a batch (cases without physical sides
// carry no bflux and return at once).
cudaError_t launch_batch_boundary_flux(Prec p, const StageArgs* args, int ncases, int max_edge, cudaStream_t s) {
    for (int c0 = 0; c0 < ncases; c0 += 65535) {  // gridDim.z limit
        const int nc = ncases - c0 < 65535 ? ncases - c0 : 65535;
        const dim3 grid((max_edge + 127) / 128, 4, nc);
        if (p == kF32Mixed) batch_boundary_flux_kernel<PolF32><<<grid, 128, 0, s>>>(args + c0);
        else batch_boundary_flux_kernel<PolF64><<<grid, 128, 0, s>>>(args + c0);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int batch_blocks_per_sm(Prec p) {
    int n = 0;
    if (p == kF32Mixed)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, batch_march_kernel<PolF32, kBatchWarps, kBatchMinBlocksF32, kBatchLoadF32, kFeatEdge | kFeatPos>,
            32 * kBatchWarps, 0);
    else
    {
        constexpr size_t dyn = batch_dyn_bytes<PolF64, kBatchLoadF64>();
        auto k = batch_march_kernel<PolF64, kBatchWarps, kBatchMinBlocksF64, kBatchLoadF64, kFeatEdge | kFeatPos>;
        if (allow_dyn(k, dyn) == cudaSuccess) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, 32 * kBatchWarps, dyn);
    }
    return n > 0 ? n : 1;
}

constexpr int kViscTI = 8;
constexpr int kViscTJ = 32;
// FP32 tiles twice as tall: the 3-cell halo of the primitive, gradient and
// face phases is recomputed on fewer cells (37.5 KB of static shared memory;
// the FP64 tile would not fit in 48 KB)
constexpr int kViscTI32 = 16;

inline dim3 visc_grid(const Layout& L, int ti) {
    return dim3((L.ny + kViscTJ - 1) / kViscTJ, (L.nx + ti - 1) / ti);
}

cudaError_t launch_viscous_f64(const ViscArgs& a, cudaStream_t s) {
    viscous_kernel<PolF64, kViscTI, kViscTJ><<<visc_grid(a.L, kViscTI), kViscTI * kViscTJ, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_viscous_f32(const ViscArgs& a, cudaStream_t s) {
    viscous_kernel<PolF32, kViscTI32, kViscTJ><<<visc_grid(a.L, kViscTI32), kViscTI32 * kViscTJ, 0, s>>>(a);
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
