// Tensor maps of the state buffers for the row march's TMA load schedule.
//
// One map per state buffer: a 3-D view (variable, column, row) of the
// interleaved layout -- dimension 0 the 4 variables of a cell (contiguous),
// dimension 1 the pitch cells of a row, dimension 2 the nx + 6 rows -- with a
// box of 4 variables x 36 cells x 1 row: one ring row of a warp's 30-column
// segment and its 3-cell halo per copy.  Columns past the row's end read as
// zeros (those cells are never used).  The encoder is the driver's
// cuTensorMapEncodeTiled, reached through the runtime's driver entry-point
// query so that the library needs no link to libcuda.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <mutex>

#include "cfs_launch.h"
#include "cfs_layout.h"

namespace cfs {
namespace {

std::once_flag g_once;
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
cudaError_t g_lookup = cudaSuccess;

void lookup_encoder() {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    g_lookup = cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q);
    if (g_lookup == cudaSuccess && (q != cudaDriverEntryPointSuccess || !fn)) g_lookup = cudaErrorNotSupported;
    if (g_lookup == cudaSuccess) g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
}

}  // namespace

cudaError_t encode_state_map(const void* base, const Layout& L, void* map) {
    std::call_once(g_once, lookup_encoder);
    if (g_lookup != cudaSuccess) return g_lookup;
    const CUtensorMapDataType type = L.elem_bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const cuuint64_t dims[3] = {static_cast<cuuint64_t>(kVars), static_cast<cuuint64_t>(L.pitch),
                                static_cast<cuuint64_t>(L.nx + 2 * kGhost)};
    const cuuint64_t strides[2] = {static_cast<cuuint64_t>(kVars) * L.elem_bytes, static_cast<cuuint64_t>(L.row_bytes())};
    const cuuint32_t box[3] = {static_cast<cuuint32_t>(kVars), static_cast<cuuint32_t>(kTmaBoxCells), 1u};
    const cuuint32_t elem_strides[3] = {1u, 1u, 1u};
    const CUresult r = g_encode(static_cast<CUtensorMap*>(map), type, 3, const_cast<void*>(base), dims, strides, box,
                                elem_strides, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace cfs
