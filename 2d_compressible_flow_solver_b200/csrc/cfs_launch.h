// Host-callable launchers of the kernels in cfs_kernels.cuh.  Each policy's
// kernels live in the translation unit whose compile flags they need:
// kernels_exact.cu (-fmad=false) and kernels_fast.cu (FMA on).
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
cudaError_t launch_totals(int elem_bytes, const void* U, const Layout& L, const uint8_t* types, double* out,
                          cudaStream_t s);
cudaError_t launch_pack(int elem_bytes, const double* src, void* dst, const Layout& L, cudaStream_t s);
cudaError_t launch_unpack(int elem_bytes, const void* src, double* dst, const Layout& L, cudaStream_t s);
cudaError_t launch_ghost_fill(int elem_bytes, void* U, const Layout& L, const BcSides& sides, cudaStream_t s);
cudaError_t launch_weno_faces(Prec p, int n, const double* st, double* left, double* right, double g, double eps,
                              cudaStream_t s);
cudaError_t launch_hll_faces(Prec p, int n, int dir, const double* L, const double* R, double* F, double g,
                             int variant, cudaStream_t s);

// Per-policy entry points behind the dispatchers above.
cudaError_t launch_stage_exact(const StageArgs& a, cudaStream_t s);
cudaError_t launch_stage_f64(const StageArgs& a, cudaStream_t s);
cudaError_t launch_stage_f32(const StageArgs& a, cudaStream_t s);
cudaError_t launch_weno_faces_exact(int n, const double* st, double* l, double* r, double g, double eps, cudaStream_t s);
cudaError_t launch_weno_faces_f64(int n, const double* st, double* l, double* r, double g, double eps, cudaStream_t s);
cudaError_t launch_weno_faces_f32(int n, const double* st, double* l, double* r, double g, double eps, cudaStream_t s);
cudaError_t launch_hll_faces_exact(int n, int dir, const double* L, const double* R, double* F, double g, int v, cudaStream_t s);
cudaError_t launch_hll_faces_f64(int n, int dir, const double* L, const double* R, double* F, double g, int v, cudaStream_t s);
cudaError_t launch_hll_faces_f32(int n, int dir, const double* L, const double* R, double* F, double g, int v, cudaStream_t s);

}  // namespace cfs
