// Host-callable launchers of the kernels in cfs_kernels.cuh and cfs_march.cuh.
// Each policy's kernels live in the translation unit whose compile flags they
// need: kernels_exact.cu (-fmad=false), kernels_fast.cu and march_inst.cu (FMA
// on; the latter once per form and feature set).
#pragma once
#include <cuda_runtime.h>

#include "cfs_layout.h"

namespace cfs {

enum Prec : int { kF64 = 0, kF32Mixed = 1, kF64Exact = 2 };

// Tile of the stage kernel: TI rows (x) by TJ columns (y, contiguous).
constexpr int kTileI = 8;
constexpr int kTileJ = 32;

cudaError_t launch_stage(Prec p, const StageArgs& a, cudaStream_t s);
cudaError_t launch_ib_fill(int elem_bytes, const IbArgs& a, cudaStream_t s);
cudaError_t launch_wmax(int elem_bytes, const void* U, const Layout& L, const uint8_t* types, double g, double dx,
                        double dy, unsigned long long* out, cudaStream_t s);
// CFL maxima of every case of a batch: args[c].in into args[c].P->wmax[0].
cudaError_t launch_batch_wmax(int elem_bytes, const StageArgs* args, int ncases, cudaStream_t s);
// Sums of the four planes of a device FP64 state [4][n], deterministic; the 4
// sums land at scratch[plane_sums_scratch_doubles() - 4 ..].
int plane_sums_scratch_doubles();
cudaError_t launch_plane_sums(const double* U, long long n, double* scratch, cudaStream_t s);
// Sums of the four planes over fluid cells, deterministic (fixed order);
// scratch holds plane_sums_scratch_doubles() doubles, the 4 sums go to out.
cudaError_t launch_totals(int elem_bytes, const void* U, const Layout& L, const uint8_t* types, double* scratch,
                          double* out, cudaStream_t s);
cudaError_t launch_pack(int elem_bytes, const double* src, void* dst, const Layout& L, cudaStream_t s);
cudaError_t launch_unpack(int elem_bytes, const void* src, double* dst, const Layout& L, cudaStream_t s);
cudaError_t launch_ghost_fill(int elem_bytes, void* U, const Layout& L, const BcSides& sides, cudaStream_t s);
cudaError_t launch_viscous(Prec p, const ViscArgs& a, cudaStream_t s);
cudaError_t launch_weno_faces(Prec p, int n, const double* st, double* left, double* right, double g, double eps,
                              cudaStream_t s);
cudaError_t launch_hll_faces(Prec p, int n, int dir, const double* L, const double* R, double* F, double g,
                             int variant, cudaStream_t s);

// TMA load schedule: one tensor map (CUtensorMap, 128 bytes, 64-byte
// aligned) per state buffer, box of 4 variables x kTmaBoxCells cells x 1 row
// (tma_maps.cpp; the row march's ring rows are that wide).
constexpr int kTmaBoxCells = 36;
constexpr int kTensorMapBytes = 128;
cudaError_t encode_state_map(const void* base, const Layout& L, void* map);

// Stage-kernel variants of the throughput forms (march_kernel template shapes).
struct MarchVariant {
    int rows, warps, min_blocks;
    int load;  // load schedule of the row march: 0 at use, 1 early in the iteration, 2 rows ahead,
               // 3 rows staged in shared memory by cp.async, 4 rows staged by TMA
};
constexpr int kNumVariants = 13;
constexpr MarchVariant kVariants[kNumVariants] = {
    {64, 4, 1, 0}, {32, 4, 5, 0}, {64, 8, 2, 0}, {32, 4, 4, 1}, {64, 8, 2, 1},
    {32, 4, 5, 2}, {32, 4, 5, 3}, {32, 4, 4, 3}, {64, 4, 4, 3}, {32, 4, 6, 3},
    {32, 4, 5, 4}, {32, 4, 4, 4}, {64, 4, 4, 4},
};
// 1-based defaults, from the committed tuning table
// (2d_compressible_flow_solver_b200/tuning.json): FP32 stages its ring rows by
// per-lane 16-byte cp.async (variant 7: 10,937 Mcell-steps/s at 4096^2 against
// 10,552 for the same shape staged by TMA, whose lane-0 issue and mbarrier
// waits cost more instructions than the copies they replace once cells are
// interleaved); FP64 by cp.async too (variant 8): with the row chunk chosen per
// launch it matches the TMA ring on periodic grids (4096^2: 5,986 against
// 5,999; 2048^2: 5,527 against 5,523) and wins with edge code (2048^2
// transmissive 5,186 against 5,120, with floors and a cylinder 4,734 against
// 4,448).
constexpr int kDefaultVariantF32 = 7;
constexpr int kDefaultVariantF64 = 8;
// FP32 grids with edge code (physical sides, cell types) run the same ring
// march with 128 registers and 4 blocks per SM: 2048^2 transmissive with floors
// and a cylinder 5,672 against 5,476 Mcell-steps/s, the 2048 x 1024 Mach-3
// cylinder 5,237 against 5,039.
constexpr int kEdgeVariantF32 = 8;
// FP64 ring blocks per SM (4 warps at 128 registers; 37 KB dynamic + 4.6 KB
// static shared memory), and the register-window variant the FP64 default
// falls back to when the ring's last wave would run nearly empty
// (launch_stage_f64).
constexpr int kRingBlocksPerSmF64 = 4;
constexpr int kWindowVariantF64 = 4;

// Batched forms (cfs_batch_*): one launch covers every case of a batch.
constexpr int kBatchWarps = 4;
// 4 blocks of 4 warps per SM (128 registers): the uneven 512-case batch ran
// 6,074 / 7,241 / 6,629 Mcell-steps/s at 5 / 4 / 3 blocks per SM.
constexpr int kBatchMinBlocksF32 = 4;
constexpr int kBatchLoadF32 = 3;  // FP32 batches stage rows in the shared ring
constexpr int kBatchMinBlocksF64 = 4;
// FP64 batches stage rows in the ring too (dynamic shared memory, 4 blocks per
// SM): the uneven 512-case batch 3,230 against 2,938 Mcell-steps/s without it
// (the earlier ring that also held U^0 rows allowed 3 blocks and lost, 2,775).
constexpr int kBatchLoadF64 = 3;
// Rows of a batch work unit (cfs_case.rows = 0): the persistent warps pull
// units until none are left, so the launch's tail is one unit per warp and
// longer units cost less per row (the uneven 512-case batch: FP32 8,408 /
// 8,651 / 8,763 / 8,838 / 8,854 and FP64 5,019 / 5,217 / 5,294 / 5,340 / 5,341
// Mcell-steps/s at 16 / 24 / 32 / 48 / 64 rows).
constexpr int kBatchRows = 64;
cudaError_t launch_batch_stage(Prec p, const StageArgs* args, const int* item_case, const int* item_local,
                               const int* case_rows, const int* case_nseg, int total, unsigned int* counter,
                               int grid, int feat, cudaStream_t s);  // feat: kFeatPos | kFeatEdge bits
// Boundary-face fluxes of every case (grid: max_edge = the largest nx or ny).
cudaError_t launch_batch_boundary_flux(Prec p, const StageArgs* args, int ncases, int max_edge, cudaStream_t s);
cudaError_t launch_batch_ib_fill(int elem_bytes, const IbArgs* args, const int* cases, const int* local, int total,
                                 cudaStream_t s);
int batch_blocks_per_sm(Prec p);

// Per-policy entry points behind the dispatchers above.
cudaError_t launch_stage_exact(const StageArgs& a, cudaStream_t s);
cudaError_t launch_stage_f64(const StageArgs& a, cudaStream_t s);
cudaError_t launch_stage_f32(const StageArgs& a, cudaStream_t s);
// Row march of one form and feature set (march_inst.cu, kFeat* bits), variant v (1-based).
cudaError_t launch_march_f64_0(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f64_1(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f64_2(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f64_3(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f64_4(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f64_5(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f64_6(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f64_7(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f32_0(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f32_1(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f32_2(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f32_3(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f32_4(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f32_5(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f32_6(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_march_f32_7(const StageArgs& a, int v, cudaStream_t s);
cudaError_t launch_viscous_f64(const ViscArgs& a, cudaStream_t s);
cudaError_t launch_viscous_f32(const ViscArgs& a, cudaStream_t s);
cudaError_t launch_weno_faces_exact(int n, const double* st, double* l, double* r, double g, double eps, cudaStream_t s);
cudaError_t launch_weno_faces_f64(int n, const double* st, double* l, double* r, double g, double eps, cudaStream_t s);
cudaError_t launch_weno_faces_f32(int n, const double* st, double* l, double* r, double g, double eps, cudaStream_t s);
cudaError_t launch_hll_faces_exact(int n, int dir, const double* L, const double* R, double* F, double g, int v, cudaStream_t s);
cudaError_t launch_hll_faces_f64(int n, int dir, const double* L, const double* R, double* F, double g, int v, cudaStream_t s);
cudaError_t launch_hll_faces_f32(int n, int dir, const double* L, const double* R, double* F, double g, int v, cudaStream_t s);

}  // namespace cfs
