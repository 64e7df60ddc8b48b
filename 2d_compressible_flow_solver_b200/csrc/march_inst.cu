// Row-march launchers of one (form, feature set): compiled once per pair, with
//   -DCFS_MARCH_POL=PolF32|PolF64  -DCFS_MARCH_FEAT=0..7  -DCFS_MARCH_FN=<launcher name>
// (the build gives each pair its own object, so the 160 kernels compile in
// parallel).  The launcher runs the variant `v` of kVariants (1-based).
#include <mutex>

#include "cfs_kernels.cuh"
#include "cfs_launch.h"
#include "cfs_march.cuh"

#if !defined(CFS_MARCH_POL) || !defined(CFS_MARCH_FEAT) || !defined(CFS_MARCH_FN)
#error "march_inst.cu needs CFS_MARCH_POL, CFS_MARCH_FEAT and CFS_MARCH_FN"
#endif

namespace cfs {
namespace {

template <class Pol, int R, int W, int B, int Ld, int F>
cudaError_t launch_march(const StageArgs& a, cudaStream_t s) {
    const int nseg = (a.L.ny + kSeg - 1) / kSeg;
    const int nrows = stage_row_hi(a) - stage_row_lo(a);
    if (nrows <= 0) return cudaSuccess;
    const dim3 grid((nseg + W - 1) / W, (nrows + R - 1) / R);
    size_t dyn = 0;
    if constexpr (Ld == 4) {
        if (!a.has_tmaps || !a.err) return cudaErrorInvalidValue;
    }
    if constexpr (Ld >= 3 && sizeof(typename Pol::T) == 8) {
        // the FP64 ring lives in dynamic shared memory; allow it once per
        // device (std::call_once: host threads may make their first launches
        // on one device at the same time)
        constexpr int kMaxDev = 64;
        static std::once_flag once[kMaxDev];
        static cudaError_t allow_err[kMaxDev];
        dyn = static_cast<size_t>(W) * ring_words<double>() * sizeof(double);
        auto allow = [dyn] {
            return cudaFuncSetAttribute(march_kernel<Pol, R, W, B, Ld, F>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(dyn));
        };
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= kMaxDev) {
            e = allow();
        } else {
            std::call_once(once[dev], [&] { allow_err[dev] = allow(); });
            e = allow_err[dev];
        }
        if (e != cudaSuccess) return e;
    }
    march_kernel<Pol, R, W, B, Ld, F><<<grid, 32 * W, dyn, s>>>(a);
    return cudaGetLastError();
}

template <class Pol, int K, int F>
cudaError_t launch_march_k(const StageArgs& a, cudaStream_t s) {
    constexpr MarchVariant v = kVariants[K];
    return launch_march<Pol, v.rows, v.warps, v.min_blocks, v.load, F>(a, s);
}

}  // namespace

cudaError_t CFS_MARCH_FN(const StageArgs& a, int v, cudaStream_t s) {
    using P = CFS_MARCH_POL;
    constexpr int F = CFS_MARCH_FEAT;
    static_assert(kNumVariants == 13, "variant table and dispatch disagree");
    switch (v) {
        case 1: return launch_march_k<P, 0, F>(a, s);
        case 2: return launch_march_k<P, 1, F>(a, s);
        case 3: return launch_march_k<P, 2, F>(a, s);
        case 4: return launch_march_k<P, 3, F>(a, s);
        case 5: return launch_march_k<P, 4, F>(a, s);
        case 6: return launch_march_k<P, 5, F>(a, s);
        case 7: return launch_march_k<P, 6, F>(a, s);
        case 8: return launch_march_k<P, 7, F>(a, s);
        case 9: return launch_march_k<P, 8, F>(a, s);
        case 10: return launch_march_k<P, 9, F>(a, s);
        case 11: return launch_march_k<P, 10, F>(a, s);
        case 12: return launch_march_k<P, 11, F>(a, s);
        case 13: return launch_march_k<P, 12, F>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace cfs
