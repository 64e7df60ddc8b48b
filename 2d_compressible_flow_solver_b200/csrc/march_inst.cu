// Row-march launchers of one (form, feature set): compiled once per pair, with
//   -DCFS_MARCH_POL=PolF32|PolF64  -DCFS_MARCH_FEAT=0..7  -DCFS_MARCH_FN=<launcher name>
// (the build gives each pair its own object, so the 160 kernels compile in
// parallel).  The launcher runs the variant `v` of kVariants (1-based).
#include <climits>
#include <mutex>

#include "cfs_kernels.cuh"
#include "cfs_launch.h"
#include "cfs_march.cuh"

#if !defined(CFS_MARCH_POL) || !defined(CFS_MARCH_FEAT) || !defined(CFS_MARCH_FN)
#error "march_inst.cu needs CFS_MARCH_POL, CFS_MARCH_FEAT and CFS_MARCH_FN"
#endif

namespace cfs {
namespace {

constexpr int kMaxDev = 64;

// Row chunk of a launch whose warps (nseg per chunk of rows, w per block) run
// on `slots` resident blocks.  An item costs its R rows plus about 2 more (the x-work of
// the row above and below the chunk), and the launch ends with a partly
// filled stretch of about half an item, so the launch lasts about
// (R + 2) (blocks / slots + 1/2): short chunks pay the per-item rows, long
// ones the tail.  The minimum lies near R = 2 sqrt(nseg nrows / (w slots)): 28 rows
// at 4096^2, 14 at 2048^2, 7 at 1024^2 (FP32, 740 slots).  Fitted to a sweep of
// fixed chunks of 8 .. 196 rows at 512^2 .. 4096^2, FP32 and FP64; a
// whole-wave model that ignored the tail picked 196 rows at 4096^2 and lost
// 12 % against 32.  Searched over 6 .. 128 rows (the whole range when it is
// shorter), ties to the longer chunk.
int choose_rows(int nseg, int w, int nrows, long long slots) {
    if (nrows <= 6 || slots <= 0) return nrows <= 6 ? nrows : 32;
    int best_r = 32;
    long long best_cost = LLONG_MAX;
    const int r_max = nrows < 128 ? nrows : 128;
    for (int r = 6; r <= r_max; ++r) {
        const long long blocks = (static_cast<long long>(nseg) * ((nrows + r - 1) / r) + w - 1) / w;
        const long long cost = static_cast<long long>(r + 2) * (2 * blocks + slots);
        if (cost <= best_cost) {
            best_cost = cost;
            best_r = r;
        }
    }
    return best_r;
}

template <class Pol, int R, int W, int B, int Ld, int F>
cudaError_t launch_march(const StageArgs& a_in, cudaStream_t s) {
    const int nseg = (a_in.L.ny + kSeg - 1) / kSeg;
    const int nrows = stage_row_hi(a_in) - stage_row_lo(a_in);
    if (nrows <= 0) return cudaSuccess;
    size_t dyn = 0;
    const StageArgs& a = a_in;
    if constexpr (Ld == 4) {
        if (!a.has_tmaps || !a.err) return cudaErrorInvalidValue;
    }
    if constexpr (Ld >= 3 && sizeof(typename Pol::T) == 8) {
        // the FP64 ring lives in dynamic shared memory; allow it once per
        // device (std::call_once: host threads may make their first launches
        // on one device at the same time)
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
    int rows = a.rows;
    if (rows <= 0) {
        // resident blocks of this kernel (SMs x blocks per SM), once per device
        static std::once_flag once_slots[kMaxDev];
        static long long slots_of[kMaxDev];
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        auto query = [dyn]() -> long long {
            int per_sm = 0, sms = 0, d = 0;
            if (cudaGetDevice(&d) != cudaSuccess ||
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d) != cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, march_kernel<Pol, R, W, B, Ld, F>, 32 * W,
                                                              dyn) != cudaSuccess)
                return 0;
            return static_cast<long long>(per_sm) * sms;
        };
        long long slots = 0;
        if (dev < 0 || dev >= kMaxDev) {
            slots = query();
        } else {
            std::call_once(once_slots[dev], [&] { slots_of[dev] = query(); });
            slots = slots_of[dev];
        }
        if (slots <= 0) (void)cudaGetLastError();  // a failed query leaves no error behind; fixed rows then
        rows = slots > 0 ? choose_rows(nseg, W, nrows, slots) : R;
    }
    // one warp per (segment, row chunk), segments fastest
    const long long items = static_cast<long long>(nseg) * ((nrows + rows - 1) / rows);
    const dim3 grid(static_cast<unsigned>((items + W - 1) / W));
    if (rows == a.rows) {
        march_kernel<Pol, R, W, B, Ld, F><<<grid, 32 * W, dyn, s>>>(a);
    } else {
        StageArgs b = a;
        b.rows = rows;
        march_kernel<Pol, R, W, B, Ld, F><<<grid, 32 * W, dyn, s>>>(b);
    }
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
