// Batched cases (cfs_batch_*): many independent grids of uneven size in one
// device arena, every stage of every case in one persistent launch, per-case
// CFL dt on the device, whole steps replayed from a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "cfs.h"
#include "cfs_launch.h"
#include "cfs_layout.h"
#include "ib_setup.h"

using cfs::kVars;

namespace {

struct BatchCase {
    cfs_case desc{};
    cfs::Layout L{};
    cfs::BcSides sides{};
    double dx = 0, dy = 0;
    size_t state_off = 0;   // bytes from the arena start to S0 (S1, S2 follow)
    long long types_off = -1;
    int rows = 32, nseg = 0, items_y = 0;  // row chunk, 30-column segments, row chunks
    std::vector<uint8_t> types;
    std::vector<uint8_t> lowo;   // CFS_POSITIVITY_BODY face flags, [nx+1][ny+1]
    long long lowo_off = -1;
    std::vector<uint8_t> cflags;  // row-march cell flags, [nx+2][ny+2] (cases with cell types)
    long long cflags_off = -1;
    long long bflux_off = -1;     // bytes from the arena start to the boundary-face fluxes
    int ib_n = 0, ib_mode = 0;
    int ib_first = 0;       // first immersed-ghost index in the flattened lists
    int feat = 0;           // row-march features this case needs (kFeatPos, kFeatEdge)
};

// Work items of one feature set: one persistent launch per stage runs them
// with the row march compiled for exactly those features, so a case with
// neither physical sides nor a body runs no edge code.
struct FeatureGroup {
    int feat = 0;
    int first = 0, count = 0;  // range of the group's items in item_case / item_local
};
constexpr int kMaxGroups = 4;  // the feature sets a batch launches: 0, Pos, Edge, Edge | Pos

}  // namespace

struct cfs_batch {
    cfs_config common{};
    cfs::Prec prec = cfs::kF32Mixed;
    int elem = 4;
    int n = 0;
    std::vector<BatchCase> cases;
    cudaStream_t stream = nullptr;
    char* arena = nullptr;
    uint8_t* types_d = nullptr;
    uint8_t* lowo_d = nullptr;
    uint8_t* cflags_d = nullptr;
    bool any_bflux = false;  // some case has a physical side
    std::vector<FeatureGroup> groups;  // work items by feature set, largest cases first in each
    int max_edge = 0;        // largest nx or ny of the cases
    int total_ig = 0;
    int* ib_cell = nullptr;
    int* ib_donor = nullptr;
    int* ib_perm = nullptr;
    double* ib_img = nullptr;
    double* ib_fac = nullptr;
    int* ig_case = nullptr;
    int* ig_local = nullptr;
    cfs::DevParams* P = nullptr;
    cfs::StageArgs* dargs = nullptr;  // [parity][stage][case]
    cfs::IbArgs* dib = nullptr;       // [input buffer][case]
    int total_items = 0;
    int* item_case = nullptr;
    int* item_local = nullptr;
    int* case_rows = nullptr;
    int* case_nseg = nullptr;
    unsigned int* counters = nullptr;  // [parity][stage][group]
    double* staging = nullptr;
    double* sums = nullptr;  // plane sums of an uploaded case state (FP32 storage offsets)
    int grid = 0;
    long long total_cells = 0;
    bool args_dirty = true;
    unsigned int steps_done = 0;  // completed RK steps: the stochastic-rounding step counter
    std::vector<double> dt_last;  // per case: dt of the last step taken (0 before any)
    cudaGraphExec_t graph2 = nullptr;
    std::string err;
};

namespace {

int bfail(cfs_batch* b, int code, const std::string& m);

#define CFSB_CUDA(b, call)                                                                                   \
    do {                                                                                                     \
        cudaError_t e_ = (call);                                                                             \
        if (e_ != cudaSuccess) return bfail((b), CFS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

thread_local std::string g_batch_create_error;

// As fail() of the single-grid API: consumes the thread's last CUDA error on
// CUDA and allocation failures (argument errors leave it alone).
int bfail(cfs_batch* b, int code, const std::string& m) {
    if (b) b->err = m;
    else g_batch_create_error = m;
    if (code == CFS_ERR_CUDA || code == CFS_ERR_NOMEM) (void)cudaGetLastError();
    return code;
}

int stages_of(int rk) { return rk == CFS_RK_TVD2 ? 2 : 3; }

// FP64 bit pattern of +infinity: the CFL maximum of a state with a non-finite fluid cell
constexpr unsigned long long kInfBits = 0x7ff0000000000000ull;

void* state_buf(const cfs_batch* b, const BatchCase& c, int k) {
    return b->arena + c.state_off + static_cast<size_t>(k) * static_cast<size_t>(c.L.bytes());
}

// Host images of the per-case stage and fill arguments (device copies in
// dargs / dib); rebuilt when storage offsets change.
int upload_args(cfs_batch* b) {
    const int S = stages_of(b->common.rk);
    std::vector<cfs::StageArgs> args(static_cast<size_t>(2) * 3 * b->n);
    std::vector<cfs::IbArgs> ibs(static_cast<size_t>(3) * b->n);
    for (int ci = 0; ci < b->n; ++ci) {
        const BatchCase& c = b->cases[ci];
        for (int p = 0; p < 2; ++p)
            for (int s = 0; s < S; ++s) {
                cfs::StageArgs a{};
                a.L = c.L;
                for (int q = 0; q < 4; ++q) a.bc[q] = c.sides.bc[q];
                a.gamma = b->common.gamma;
                a.eps = b->common.weno_eps;
                a.dx = c.dx;
                a.dy = c.dy;
                a.rk = b->common.rk;
                a.hll = b->common.hll;
                a.types = c.types_off >= 0 ? b->types_d + c.types_off : nullptr;
                a.positivity = b->common.positivity;
                a.rounding = b->common.rounding;
                a.lowo = c.lowo_off >= 0 ? b->lowo_d + c.lowo_off : nullptr;
                a.cflags = c.cflags_off >= 0 ? b->cflags_d + c.cflags_off : nullptr;
                a.bflux = c.bflux_off >= 0 ? b->arena + c.bflux_off : nullptr;
                a.stage = s;
                // buffer roles of a step that starts in S0 (as cfs_advance)
                int in = 0, out = 1, u0 = 0, u1 = -1;
                if (s == 1) {
                    in = 1;
                    u1 = 1;
                    out = b->common.rk == CFS_RK_TVD2 ? 0 : 2;
                } else if (s == 2) {
                    in = 2;
                    u1 = 1;
                    out = 0;
                }
                a.in = state_buf(b, c, in);
                a.out = state_buf(b, c, out);
                a.u0 = state_buf(b, c, u0);
                a.u1 = u1 >= 0 ? state_buf(b, c, u1) : nullptr;
                a.P = b->P + ci;
                a.parity = p;
                a.first_stage = s == 0 ? 1 : 0;
                a.last_stage = s == S - 1 ? 1 : 0;
                args[(static_cast<size_t>(p) * 3 + s) * b->n + ci] = a;
            }
        for (int k = 0; k < 3; ++k) {
            cfs::IbArgs ia{};
            ia.U = state_buf(b, c, k);
            ia.L = c.L;
            ia.n = c.ib_n;
            ia.mode = c.ib_mode;
            ia.cell = b->ib_cell ? b->ib_cell + c.ib_first : nullptr;
            ia.donor = b->ib_donor ? b->ib_donor + 4 * static_cast<size_t>(c.ib_first) : nullptr;
            ia.perm = b->ib_perm ? b->ib_perm + 4 * static_cast<size_t>(c.ib_first) : nullptr;
            ia.image = b->ib_img ? b->ib_img + 2 * static_cast<size_t>(c.ib_first) : nullptr;
            ia.fac = b->ib_fac ? b->ib_fac + 16 * static_cast<size_t>(c.ib_first) : nullptr;
            ibs[static_cast<size_t>(k) * b->n + ci] = ia;
        }
    }
    CFSB_CUDA(b, cudaMemcpy(b->dargs, args.data(), sizeof(cfs::StageArgs) * args.size(), cudaMemcpyHostToDevice));
    CFSB_CUDA(b, cudaMemcpy(b->dib, ibs.data(), sizeof(cfs::IbArgs) * ibs.size(), cudaMemcpyHostToDevice));
    if (b->graph2) {
        cudaGraphExecDestroy(b->graph2);
        b->graph2 = nullptr;
    }
    b->args_dirty = false;
    return CFS_OK;
}

int enqueue_batch_step(cfs_batch* b, int parity) {
    const int S = stages_of(b->common.rk);
    for (int s = 0; s < S; ++s) {
        const int slot = parity * 3 + s;
        const int in = s;  // stage s reads S_s (S0, S1, S2)
        CFSB_CUDA(b, cudaMemsetAsync(b->counters + slot * kMaxGroups, 0, sizeof(unsigned int) * kMaxGroups, b->stream));
        if (b->total_ig > 0)
            CFSB_CUDA(b, cfs::launch_batch_ib_fill(b->elem, b->dib + static_cast<size_t>(in) * b->n, b->ig_case,
                                                   b->ig_local, b->total_ig, b->stream));
        if (b->any_bflux)
            CFSB_CUDA(b, cfs::launch_batch_boundary_flux(b->prec, b->dargs + static_cast<size_t>(slot) * b->n, b->n,
                                                         b->max_edge, b->stream));
        for (size_t g = 0; g < b->groups.size(); ++g) {
            const FeatureGroup& fg = b->groups[g];
            CFSB_CUDA(b, cfs::launch_batch_stage(b->prec, b->dargs + static_cast<size_t>(slot) * b->n,
                                                 b->item_case + fg.first, b->item_local + fg.first, b->case_rows,
                                                 b->case_nseg, fg.count, b->counters + slot * kMaxGroups + g, b->grid,
                                                 fg.feat, b->stream));
        }
    }
    return CFS_OK;
}

}  // namespace

extern "C" {

const char* cfs_batch_last_error(const cfs_batch* b) { return b ? b->err.c_str() : g_batch_create_error.c_str(); }

int cfs_batch_destroy(cfs_batch* b) {
    if (!b) return CFS_OK;
    cudaSetDevice(b->common.device);  // best effort: the frees below belong to that device
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph2) cudaGraphExecDestroy(b->graph2);
    cudaFree(b->arena);
    cudaFree(b->types_d);
    cudaFree(b->lowo_d);
    cudaFree(b->cflags_d);
    cudaFree(b->ib_cell);
    cudaFree(b->ib_donor);
    cudaFree(b->ib_perm);
    cudaFree(b->ib_img);
    cudaFree(b->ib_fac);
    cudaFree(b->ig_case);
    cudaFree(b->ig_local);
    cudaFree(b->P);
    cudaFree(b->dargs);
    cudaFree(b->dib);
    cudaFree(b->item_case);
    cudaFree(b->item_local);
    cudaFree(b->case_rows);
    cudaFree(b->case_nseg);
    cudaFree(b->counters);
    cudaFree(b->staging);
    cudaFree(b->sums);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return CFS_OK;
}

int cfs_batch_create(const cfs_config* common, int ncases, const cfs_case* cases, cfs_batch** out) {
    if (!out || !common || ncases <= 0 || !cases) return bfail(nullptr, CFS_ERR_INVALID, "bad batch arguments");
    *out = nullptr;
    if (common->precision != CFS_FP32_MIXED && common->precision != CFS_FP64)
        return bfail(nullptr, CFS_ERR_INVALID, "batches run the throughput forms (CFS_FP32_MIXED or CFS_FP64)");
    if (common->rk < 0 || common->rk > 2 || common->hll < 0 || common->hll > 1 || !(common->gamma > 1) ||
        !(common->weno_eps > 0))
        return bfail(nullptr, CFS_ERR_INVALID, "bad common configuration");
    if (common->viscous != CFS_VISCOUS_OFF) return bfail(nullptr, CFS_ERR_INVALID, "batches are inviscid");
    if (common->positivity < CFS_POSITIVITY_OFF || common->positivity > CFS_POSITIVITY_FLOOR)
        return bfail(nullptr, CFS_ERR_INVALID, "unknown positivity mode");
    if (common->rounding != CFS_ROUND_STOCHASTIC && common->rounding != CFS_ROUND_NEAREST &&
        common->rounding != CFS_ROUND_STOCHASTIC_ALL)
        return bfail(nullptr, CFS_ERR_INVALID, "unknown rounding mode");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return bfail(nullptr, CFS_ERR_CUDA, "no CUDA device available (the engine has no CPU path)");
    cfs_batch* b = new (std::nothrow) cfs_batch();
    if (!b) return bfail(nullptr, CFS_ERR_NOMEM, "host allocation failed");
    auto bail = [&](int code, const std::string& m) {
        cfs_batch_destroy(b);
        return bfail(nullptr, code, m);
    };
    b->common = *common;
    b->prec = common->precision == CFS_FP32_MIXED ? cfs::kF32Mixed : cfs::kF64;
    b->elem = b->prec == cfs::kF32Mixed ? 4 : 8;
    b->n = ncases;
    b->cases.resize(ncases);
    b->dt_last.assign(ncases, 0.0);
    if (cudaSetDevice(common->device) != cudaSuccess) return bail(CFS_ERR_CUDA, "cudaSetDevice failed");
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(CFS_ERR_CUDA, "stream creation failed");

    // --- per-case layout, boundaries, immersed boundary (host)
    size_t arena = 0, types_bytes = 0, lowo_bytes = 0, cflags_bytes = 0, max_cells = 0;
    std::vector<int32_t> h_cell, h_donor, h_perm, h_igc, h_igl;
    std::vector<double> h_img, h_fac;
    for (int ci = 0; ci < ncases; ++ci) {
        BatchCase& c = b->cases[ci];
        c.desc = cases[ci];
        const cfs_case& d = c.desc;
        if (d.nx < 3 || d.ny < 3 || !(d.lx > 0) || !(d.ly > 0))
            return bail(CFS_ERR_INVALID, "case " + std::to_string(ci) + ": bad grid");
        for (int s = 0; s < 4; ++s) {
            if (d.bc[s] < 0 || d.bc[s] > 2) return bail(CFS_ERR_INVALID, "case " + std::to_string(ci) + ": bad side");
            c.sides.bc[s] = d.bc[s];
            const double rho = d.bc_prim[s][0], u = d.bc_prim[s][1], v = d.bc_prim[s][2], p = d.bc_prim[s][3];
            if (d.bc[s] == CFS_BC_DIRICHLET && !(rho > 0))
                return bail(CFS_ERR_INVALID, "case " + std::to_string(ci) + ": Dirichlet density must be positive");
            const double mx = rho * u, my = rho * v;
            c.sides.U[s][0] = rho;
            c.sides.U[s][1] = mx;
            c.sides.U[s][2] = my;
            c.sides.U[s][3] = d.bc[s] == CFS_BC_DIRICHLET ? p / (common->gamma - 1) + 0.5 * (mx * mx + my * my) / rho : 0.0;
        }
        if ((d.bc[0] == CFS_BC_PERIODIC) != (d.bc[1] == CFS_BC_PERIODIC) ||
            (d.bc[2] == CFS_BC_PERIODIC) != (d.bc[3] == CFS_BC_PERIODIC))
            return bail(CFS_ERR_INVALID, "case " + std::to_string(ci) + ": periodic sides come in pairs");
        c.L = cfs::Layout::make(d.nx, d.ny, b->elem);
        c.dx = d.lx / d.nx;
        c.dy = d.ly / d.ny;
        c.rows = d.rows > 0 ? d.rows : cfs::kBatchRows;
        c.nseg = (d.ny + 29) / 30;
        c.items_y = (d.nx + c.rows - 1) / c.rows;
        c.state_off = arena;
        arena += static_cast<size_t>(3) * static_cast<size_t>(c.L.bytes());
        arena = (arena + 255) & ~static_cast<size_t>(255);
        bool physical = false;
        for (int s = 0; s < 4; ++s) physical = physical || d.bc[s] == CFS_BC_NEUMANN || d.bc[s] == CFS_BC_DIRICHLET;
        if (physical) {
            c.bflux_off = static_cast<long long>(arena);
            arena += static_cast<size_t>(cfs::bflux_count(c.L)) * b->elem;
            arena = (arena + 255) & ~static_cast<size_t>(255);
            b->any_bflux = true;
        }
        b->max_edge = std::max(b->max_edge, std::max(d.nx, d.ny));
        max_cells = std::max(max_cells, static_cast<size_t>(d.nx) * d.ny);
        b->total_cells += static_cast<long long>(d.nx) * d.ny;
        if (d.circle) {
            cfs::IbList ib;
            std::string e;
            // per-cell set-up on the device (bit for bit the host set-up's result)
            if (!cfs::build_circle_device(d.nx, d.ny, d.lx, d.ly, d.radius, d.cx, d.cy, d.npoints > 0 ? d.npoints : 400,
                                          b->stream, ib, e))
                return bail(e.rfind("device circle set-up", 0) == 0 ? CFS_ERR_CUDA : CFS_ERR_INVALID,
                            "case " + std::to_string(ci) + ": " + e);
            c.types = ib.types;
            c.types_off = static_cast<long long>(types_bytes);
            types_bytes += c.types.size();
            if (common->positivity >= CFS_POSITIVITY_BODY) {
                c.lowo = cfs::low_order_faces(c.types.data(), d.nx, d.ny, d.bc);
                c.lowo_off = static_cast<long long>(lowo_bytes);
                lowo_bytes += c.lowo.size();
            }
            c.cflags = cfs::cell_flags(c.types.data(), c.lowo.empty() ? nullptr : c.lowo.data(), d.nx, d.ny);
            c.cflags_off = static_cast<long long>(cflags_bytes);
            cflags_bytes += c.cflags.size();
            c.ib_n = static_cast<int>(ib.cell.size());
            c.ib_mode = d.ib_mode;
            c.ib_first = static_cast<int>(h_cell.size());
            std::vector<int32_t> dd;
            std::vector<double> fac;
            std::vector<int> perm;
            cfs::ib_factors(d.ib_mode, c.types.data(), d.nx, d.ny, c.dx, c.dy, c.ib_n, ib.donor.data(), ib.image.data(),
                            ib.normal.data(), dd, fac, perm);
            h_cell.insert(h_cell.end(), ib.cell.begin(), ib.cell.end());
            h_donor.insert(h_donor.end(), dd.begin(), dd.end());
            h_perm.insert(h_perm.end(), perm.begin(), perm.end());
            h_img.insert(h_img.end(), ib.image.begin(), ib.image.end());
            h_fac.insert(h_fac.end(), fac.begin(), fac.end());
            for (int g = 0; g < c.ib_n; ++g) {
                h_igc.push_back(ci);
                h_igl.push_back(g);
            }
        }
    }
    b->total_ig = static_cast<int>(h_cell.size());

    // --- features per case: edge code where a case has a physical side or
    // a body, positivity code as the batch's mode asks
    for (BatchCase& c : b->cases) {
        bool physical = false;
        for (int s = 0; s < 4; ++s)
            physical = physical || c.desc.bc[s] == CFS_BC_NEUMANN || c.desc.bc[s] == CFS_BC_DIRICHLET;
        c.feat = (common->positivity ? cfs::kFeatPos : 0) |
                 (physical || c.cflags_off >= 0 || c.desc.edge_code ? cfs::kFeatEdge : 0);
    }
    // --- work items grouped by feature set, largest cases first in each group
    std::vector<int> order(ncases);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        if (b->cases[x].feat != b->cases[y].feat) return b->cases[x].feat < b->cases[y].feat;
        return static_cast<long long>(b->cases[x].desc.nx) * b->cases[x].desc.ny >
               static_cast<long long>(b->cases[y].desc.nx) * b->cases[y].desc.ny;
    });
    // one work unit per (segment, row chunk): a warp's share of a stage
    std::vector<int> it_case, it_local, c_rows(ncases), c_ix(ncases);
    for (int ci : order) {
        const BatchCase& c = b->cases[ci];
        if (b->groups.empty() || b->groups.back().feat != c.feat) {
            FeatureGroup g;
            g.feat = c.feat;
            g.first = static_cast<int>(it_case.size());
            b->groups.push_back(g);
        }
        for (int li = 0; li < c.nseg * c.items_y; ++li) {
            it_case.push_back(ci);
            it_local.push_back(li);
        }
        b->groups.back().count = static_cast<int>(it_case.size()) - b->groups.back().first;
    }
    for (int ci = 0; ci < ncases; ++ci) {
        c_rows[ci] = b->cases[ci].rows;
        c_ix[ci] = b->cases[ci].nseg;
    }
    b->total_items = static_cast<int>(it_case.size());

    // --- device allocations
    auto dalloc = [&](void** p, size_t bytes) { return bytes == 0 || cudaMalloc(p, bytes) == cudaSuccess; };
    if (!dalloc(reinterpret_cast<void**>(&b->arena), arena)) return bail(CFS_ERR_NOMEM, "state arena allocation failed");
    if (!dalloc(reinterpret_cast<void**>(&b->types_d), types_bytes) ||
        !dalloc(reinterpret_cast<void**>(&b->lowo_d), lowo_bytes) ||
        !dalloc(reinterpret_cast<void**>(&b->cflags_d), cflags_bytes) ||
        !dalloc(reinterpret_cast<void**>(&b->ib_cell), sizeof(int) * h_cell.size()) ||
        !dalloc(reinterpret_cast<void**>(&b->ib_donor), sizeof(int) * h_donor.size()) ||
        !dalloc(reinterpret_cast<void**>(&b->ib_perm), sizeof(int) * h_perm.size()) ||
        !dalloc(reinterpret_cast<void**>(&b->ib_img), sizeof(double) * h_img.size()) ||
        !dalloc(reinterpret_cast<void**>(&b->ib_fac), sizeof(double) * h_fac.size()) ||
        !dalloc(reinterpret_cast<void**>(&b->ig_case), sizeof(int) * h_igc.size()) ||
        !dalloc(reinterpret_cast<void**>(&b->ig_local), sizeof(int) * h_igl.size()) ||
        !dalloc(reinterpret_cast<void**>(&b->P), sizeof(cfs::DevParams) * ncases) ||
        !dalloc(reinterpret_cast<void**>(&b->dargs), sizeof(cfs::StageArgs) * 6 * ncases) ||
        !dalloc(reinterpret_cast<void**>(&b->dib), sizeof(cfs::IbArgs) * 3 * ncases) ||
        !dalloc(reinterpret_cast<void**>(&b->item_case), sizeof(int) * it_case.size()) ||
        !dalloc(reinterpret_cast<void**>(&b->item_local), sizeof(int) * it_local.size()) ||
        !dalloc(reinterpret_cast<void**>(&b->case_rows), sizeof(int) * ncases) ||
        !dalloc(reinterpret_cast<void**>(&b->case_nseg), sizeof(int) * ncases) ||
        !dalloc(reinterpret_cast<void**>(&b->counters), sizeof(unsigned int) * 6 * kMaxGroups) ||
        !dalloc(reinterpret_cast<void**>(&b->staging), sizeof(double) * kVars * max_cells) ||
        !dalloc(reinterpret_cast<void**>(&b->sums), sizeof(double) * cfs::plane_sums_scratch_doubles()))
        return bail(CFS_ERR_NOMEM, "batch device allocation failed");
    auto h2d = [&](void* dst, const void* src, size_t bytes) {
        return bytes == 0 || cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
    };
    bool ok = cudaMemset(b->arena, 0, arena) == cudaSuccess;
    for (const BatchCase& c : b->cases)
        if (c.types_off >= 0) ok = ok && h2d(b->types_d + c.types_off, c.types.data(), c.types.size());
    for (const BatchCase& c : b->cases)
        if (c.lowo_off >= 0) ok = ok && h2d(b->lowo_d + c.lowo_off, c.lowo.data(), c.lowo.size());
    for (const BatchCase& c : b->cases)
        if (c.cflags_off >= 0) ok = ok && h2d(b->cflags_d + c.cflags_off, c.cflags.data(), c.cflags.size());
    ok = ok && h2d(b->ib_cell, h_cell.data(), sizeof(int) * h_cell.size()) &&
         h2d(b->ib_donor, h_donor.data(), sizeof(int) * h_donor.size()) &&
         h2d(b->ib_perm, h_perm.data(), sizeof(int) * h_perm.size()) &&
         h2d(b->ib_img, h_img.data(), sizeof(double) * h_img.size()) &&
         h2d(b->ib_fac, h_fac.data(), sizeof(double) * h_fac.size()) &&
         h2d(b->ig_case, h_igc.data(), sizeof(int) * h_igc.size()) &&
         h2d(b->ig_local, h_igl.data(), sizeof(int) * h_igl.size()) &&
         h2d(b->item_case, it_case.data(), sizeof(int) * it_case.size()) &&
         h2d(b->item_local, it_local.data(), sizeof(int) * it_local.size()) &&
         h2d(b->case_rows, c_rows.data(), sizeof(int) * ncases) && h2d(b->case_nseg, c_ix.data(), sizeof(int) * ncases) &&
         cudaMemset(b->P, 0, sizeof(cfs::DevParams) * ncases) == cudaSuccess;
    if (!ok) return bail(CFS_ERR_CUDA, "batch upload failed");
    for (int ci = 0; ci < ncases; ++ci)
        for (int k = 0; k < 3; ++k)
            if (cfs::launch_ghost_fill(b->elem, state_buf(b, b->cases[ci], k), b->cases[ci].L, b->cases[ci].sides,
                                       b->stream) != cudaSuccess)
                return bail(CFS_ERR_CUDA, "ghost fill failed");
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, common->device) != cudaSuccess || sms <= 0)
        return bail(CFS_ERR_CUDA, "SM count query failed");
    b->grid = sms * cfs::batch_blocks_per_sm(b->prec);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
        return bail(CFS_ERR_CUDA, "batch initialisation failed");
    *out = b;
    return CFS_OK;
}

void* cfs_batch_get_stream(cfs_batch* b) { return b ? static_cast<void*>(b->stream) : nullptr; }

int cfs_batch_info(const cfs_batch* b, long long* cells, int* items) {
    if (!b) return bfail(nullptr, CFS_ERR_INVALID, "null batch");
    if (cells) *cells = b->total_cells;
    if (items) *items = b->total_items;
    return CFS_OK;
}

int cfs_batch_set_state(cfs_batch* b, int ci, const double* U) {
    if (!b || !U || ci < 0 || ci >= b->n) return bfail(b, CFS_ERR_INVALID, "bad case or state");
    CFSB_CUDA(b, cudaSetDevice(b->common.device));
    BatchCase& c = b->cases[ci];
    const size_t n = static_cast<size_t>(c.desc.nx) * c.desc.ny;
    CFSB_CUDA(b, cudaMemcpyAsync(b->staging, U, sizeof(double) * kVars * n, cudaMemcpyHostToDevice, b->stream));
    if (b->elem == 4) {
        // FP32 storage offsets: the FP32-rounded means, summed on the device as
        // a single grid's (cfs_set_state) are
        double sums[kVars];
        CFSB_CUDA(b, cfs::launch_plane_sums(b->staging, static_cast<long long>(n), b->sums, b->stream));
        CFSB_CUDA(b, cudaMemcpyAsync(sums, b->sums + cfs::plane_sums_scratch_doubles() - kVars, sizeof(sums),
                                     cudaMemcpyDeviceToHost, b->stream));
        CFSB_CUDA(b, cudaStreamSynchronize(b->stream));
        for (int v = 0; v < kVars; ++v) {
            float off = static_cast<float>(sums[v] / static_cast<double>(n));
            if (!std::isfinite(off)) off = 0.0f;
            if (off != c.L.off[v]) b->args_dirty = true;
            c.L.off[v] = off;
        }
    }
    CFSB_CUDA(b, cfs::launch_pack(b->elem, b->staging, state_buf(b, c, 0), c.L, b->stream));
    for (int k = 0; k < 3; ++k) CFSB_CUDA(b, cfs::launch_ghost_fill(b->elem, state_buf(b, c, k), c.L, c.sides, b->stream));
    CFSB_CUDA(b, cudaStreamSynchronize(b->stream));
    return CFS_OK;
}

int cfs_batch_get_state(cfs_batch* b, int ci, double* U) {
    if (!b || !U || ci < 0 || ci >= b->n) return bfail(b, CFS_ERR_INVALID, "bad case or state");
    CFSB_CUDA(b, cudaSetDevice(b->common.device));
    const BatchCase& c = b->cases[ci];
    const size_t n = static_cast<size_t>(c.desc.nx) * c.desc.ny;
    CFSB_CUDA(b, cfs::launch_unpack(b->elem, state_buf(b, c, 0), b->staging, c.L, b->stream));
    CFSB_CUDA(b, cudaMemcpyAsync(U, b->staging, sizeof(double) * kVars * n, cudaMemcpyDeviceToHost, b->stream));
    CFSB_CUDA(b, cudaStreamSynchronize(b->stream));
    return CFS_OK;
}

namespace {

// nsteps steps of every case: per-case CFL dt (cfl > 0), else a fixed dt per
// case (dt_case[c], or the common dt when dt_case is null).
int batch_advance(cfs_batch* b, int nsteps, double cfl, double dt, const double* dt_case, double* t) {
    CFSB_CUDA(b, cudaSetDevice(b->common.device));
    if (b->args_dirty) {
        const int rc = upload_args(b);
        if (rc != CFS_OK) return rc;
    }
    std::vector<cfs::DevParams> hp(b->n);
    for (int ci = 0; ci < b->n; ++ci) {
        cfs::DevParams& p = hp[ci];
        p = cfs::DevParams{};
        p.use_cfl = cfl > 0 ? 1 : 0;
        p.seed[0] = p.seed[1] = b->steps_done;
        p.cfl = cfl;
        p.dt_fixed = dt_case ? dt_case[ci] : dt;
    }
    CFSB_CUDA(b, cudaMemcpyAsync(b->P, hp.data(), sizeof(cfs::DevParams) * b->n, cudaMemcpyHostToDevice, b->stream));
    // first step's CFL maxima: the stage-0 arguments of parity 0 read S0 and
    // point at each case's parameters
    if (cfl > 0) CFSB_CUDA(b, cfs::launch_batch_wmax(b->elem, b->dargs, b->n, b->stream));
    if (nsteps >= 2 && !b->graph2) {
        cudaGraph_t g = nullptr;
        CFSB_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_batch_step(b, 0);
        if (rc == CFS_OK) rc = enqueue_batch_step(b, 1);
        const cudaError_t ec = cudaStreamEndCapture(b->stream, &g);
        if (rc != CFS_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ec != cudaSuccess) return bfail(b, CFS_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(ec));
        const cudaError_t ei = cudaGraphInstantiate(&b->graph2, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            b->graph2 = nullptr;
            return bfail(b, CFS_ERR_CUDA, std::string("graph instantiation failed: ") + cudaGetErrorString(ei));
        }
    }
    for (int k = 0; k + 1 < nsteps; k += 2) CFSB_CUDA(b, cudaGraphLaunch(b->graph2, b->stream));
    if (nsteps % 2 == 1) {
        const int rc = enqueue_batch_step(b, 0);
        if (rc != CFS_OK) return rc;
    }
    CFSB_CUDA(b, cudaMemcpyAsync(hp.data(), b->P, sizeof(cfs::DevParams) * b->n, cudaMemcpyDeviceToHost, b->stream));
    CFSB_CUDA(b, cudaStreamSynchronize(b->stream));
    b->steps_done += static_cast<unsigned int>(nsteps);
    for (int ci = 0; ci < b->n; ++ci) {
        if (t) t[ci] = hp[ci].t;
        if (nsteps > 0) b->dt_last[ci] = hp[ci].dt_last;
        if (nsteps > 0 && (!(hp[ci].dt_last > 0) || !std::isfinite(hp[ci].dt_last)))
            return bfail(b, CFS_ERR_NUMERIC, "case " + std::to_string(ci) + ": time step became non-finite or non-positive");
        // the final state's CFL maximum (left by the last stage) is +infinity
        // when a fluid cell of it is non-finite
        if (nsteps > 0 && cfl > 0 && hp[ci].wmax[nsteps % 2 == 1 ? 1 : 0] == kInfBits)
            return bfail(b, CFS_ERR_NUMERIC, "case " + std::to_string(ci) + ": a fluid cell became non-finite");
    }
    return CFS_OK;
}

}  // namespace

int cfs_batch_advance(cfs_batch* b, int nsteps, double cfl, double dt, double* t) {
    if (!b) return bfail(nullptr, CFS_ERR_INVALID, "null batch");
    if (nsteps < 0 || (!(cfl > 0) && !(dt > 0))) return bfail(b, CFS_ERR_INVALID, "give nsteps >= 0 and cfl > 0 or dt > 0");
    return batch_advance(b, nsteps, cfl, dt, nullptr, t);
}

int cfs_batch_advance_dt(cfs_batch* b, int nsteps, const double* dt_case, double* t) {
    if (!b) return bfail(nullptr, CFS_ERR_INVALID, "null batch");
    if (nsteps < 0 || !dt_case) return bfail(b, CFS_ERR_INVALID, "give nsteps >= 0 and a dt per case");
    for (int ci = 0; ci < b->n; ++ci)
        if (!(dt_case[ci] > 0) || !std::isfinite(dt_case[ci]))
            return bfail(b, CFS_ERR_INVALID, "case " + std::to_string(ci) + ": dt must be finite and positive");
    return batch_advance(b, nsteps, 0.0, 0.0, dt_case, t);
}

int cfs_batch_dt_last(const cfs_batch* b, double* dt) {
    if (!b || !dt) return bfail(nullptr, CFS_ERR_INVALID, "null argument");
    for (int ci = 0; ci < b->n; ++ci) dt[ci] = b->dt_last[ci];
    return CFS_OK;
}

}  // extern "C"
