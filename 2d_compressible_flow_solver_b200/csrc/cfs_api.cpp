// C ABI of the stage engine (include/cfs.h): context, device memory, stage
// sequencing, CUDA-graph replay of whole steps, immersed-boundary upload.
#include "cfs.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "cfs_launch.h"
#include "cfs_layout.h"
#include "host_stage.h"
#include "ib_setup.h"

using cfs::kGhost;
using cfs::kVars;

struct cfs_ctx {
    cfs_config cfg{};
    cfs::Prec prec = cfs::kF64;
    cfs::Layout L{};
    cfs::BcSides sides{};
    double dx = 0, dy = 0;
    cudaStream_t stream = nullptr;
    void* S[3] = {nullptr, nullptr, nullptr};
    int cur = 0;          // buffer holding the current state
    int u0_idx = -1;      // buffer holding the stage-0 input of the running step
    int u1_idx = -1;      // buffer holding the stage-1 input (TVD3)
    int next_stage = 0;   // stage the RK sequence expects next
    double* rhs = nullptr;
    double* staging = nullptr;
    double* sums = nullptr;  // plane sums of an uploaded state (FP32 storage offsets)
    void* host_stage = nullptr;   // pinned host buffer of the staged copies of large pageable arrays
    size_t host_stage_bytes = 0;
    void* rv = nullptr;   // viscous RHS [3][nx][ny] (Navier-Stokes form only)
    uint8_t* types_d = nullptr;
    uint8_t* lowo_d = nullptr;  // [nx+1][ny+1] face flags of CFS_POSITIVITY_BODY
    uint8_t* cflags_d = nullptr;  // [nx+2][ny+2] per-cell flags of the row march (with cell types)
    void* bflux = nullptr;        // boundary-face fluxes of the row march (physical sides)
    bool has_tmaps = false;       // throughput forms: TMA tensor maps of S0, S1, S2 encoded
    alignas(64) unsigned char tmaps[3][cfs::kTensorMapBytes] = {};
    unsigned int* err_d = nullptr;   // device error flags (cfs::kErr* bits)
    unsigned int steps_done = 0;  // completed RK steps: the stochastic-rounding step counter
    // CFL maximum of the current state from the last stage of the last advance
    // (FP64 bits), reused by the next advance while nothing changed the state
    bool wmax_carry = false;
    unsigned long long wmax_bits = 0;
    bool fixed_offsets = false;   // FP32 storage offsets set by cfs_set_storage_offsets
    float fixed_off[4] = {0, 0, 0, 0};
    bool has_types = false;
    std::vector<uint8_t> types_h;
    // immersed ghosts
    int ib_n = 0, ib_mode = 0;
    int* ib_cell = nullptr;
    int* ib_donor = nullptr;
    int* ib_perm = nullptr;
    double* ib_img = nullptr;
    double* ib_fac = nullptr;
    std::vector<int32_t> ib_cell_h, ib_donor_h;
    std::vector<double> ib_img_h;
    // reductions / graph-mode parameters
    cfs::DevParams* P = nullptr;
    unsigned long long* wmax = nullptr;
    double* totals = nullptr;
    cudaGraphExec_t graph2 = nullptr;  // two full steps (parity 0 then 1)
    cudaGraphExec_t graph1 = nullptr;  // one full step (parity 0): an odd step count's last step
    cfs::DevParams* hp_pin = nullptr;  // pinned host copies of cfs_advance's parameters in [0] and results in [1]
    // device-ordered stepping (cfs_steps_*): between begin and end
    bool in_steps = false;
    bool steps_cfl = false;
    int steps_parity = 0;         // DevParams slot parity of the running step
    int steps_part = 0;           // part of the current stage already enqueued (CFS_PART_*)
    std::string err;
};

namespace {

thread_local std::string g_create_error;

// Device buffer of one call, freed on every return path (cudaFree waits for
// the device, so a copy still queued on an error path ends first).
struct DeviceScratch {
    void* p = nullptr;
    DeviceScratch() = default;
    DeviceScratch(const DeviceScratch&) = delete;
    DeviceScratch& operator=(const DeviceScratch&) = delete;
    ~DeviceScratch() { cudaFree(p); }
    cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes); }
    template <class T>
    T* get() const { return static_cast<T*>(p); }
};

// Every error reaches the caller through here.  A failed runtime call (an
// allocation, a launch) also leaves its error as this thread's last CUDA
// error; on those paths (CFS_ERR_CUDA, CFS_ERR_NOMEM) it is consumed here, so
// that the launch checks of later calls do not report it again as their own.
// Argument and state errors made no CUDA call and leave any error pending
// from other code on the thread untouched.
int fail(cfs_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    else g_create_error = msg;
    if (code == CFS_ERR_CUDA || code == CFS_ERR_NOMEM) (void)cudaGetLastError();
    return code;
}

#define CFS_CUDA(ctx, call)                                                                          \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) return fail((ctx), CFS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int stages_per_step(int rk) { return rk == CFS_RK_TVD2 ? 2 : 3; }

// Stage index from the loop counter: TVD2rdRK.cpp:11, TVD3rdRK.cpp:15.
int stage_of_counter(int rk, int counter) {
    if (rk == CFS_RK_TVD2) return (counter % 2 == 0) ? 1 : 0;
    return (counter % 3 == 0) ? 2 : (counter % 3 == 1) ? 0 : 1;
}

void release_graph(cfs_ctx* c) {
    if (c->graph2) {
        cudaGraphExecDestroy(c->graph2);
        c->graph2 = nullptr;
    }
    if (c->graph1) {
        cudaGraphExecDestroy(c->graph1);
        c->graph1 = nullptr;
    }
}

int validate(const cfs_config* g, std::string& msg) {
    if (!g) { msg = "null config"; return CFS_ERR_INVALID; }
    if (g->nx < 3 || g->ny < 3) { msg = "nx and ny must be at least 3"; return CFS_ERR_INVALID; }
    if (static_cast<long long>(g->nx) * g->ny > (1LL << 31) - 1) { msg = "nx*ny must fit in 31 bits"; return CFS_ERR_INVALID; }
    if (!(g->lx > 0) || !(g->ly > 0)) { msg = "lx and ly must be positive"; return CFS_ERR_INVALID; }
    if (!(g->gamma > 1.0)) { msg = "gamma must exceed 1"; return CFS_ERR_INVALID; }
    if (!(g->weno_eps > 0)) { msg = "weno_eps must be positive"; return CFS_ERR_INVALID; }
    if (g->precision < 0 || g->precision > 2) { msg = "unknown precision"; return CFS_ERR_INVALID; }
    if (g->rk < 0 || g->rk > 2) { msg = "unknown rk variant"; return CFS_ERR_INVALID; }
    if (g->hll < 0 || g->hll > 1) { msg = "unknown hll variant"; return CFS_ERR_INVALID; }
    for (int s = 0; s < 4; ++s)
        if (g->bc[s] < 0 || g->bc[s] > 3) { msg = "unknown boundary kind on side " + std::to_string(s); return CFS_ERR_INVALID; }
    if (g->bc[2] == CFS_BC_HALO || g->bc[3] == CFS_BC_HALO) { msg = "halo sides are left/right only"; return CFS_ERR_INVALID; }
    if ((g->bc[0] == CFS_BC_PERIODIC) != (g->bc[1] == CFS_BC_PERIODIC) ||
        (g->bc[2] == CFS_BC_PERIODIC) != (g->bc[3] == CFS_BC_PERIODIC)) {
        msg = "periodic sides come in pairs (left/right, bottom/top)";
        return CFS_ERR_INVALID;
    }
    for (int s = 0; s < 4; ++s)
        if (g->bc[s] == CFS_BC_DIRICHLET && !(g->bc_prim[s][0] > 0)) {
            msg = "Dirichlet density must be positive on side " + std::to_string(s);
            return CFS_ERR_INVALID;
        }
    if (g->viscous != CFS_VISCOUS_OFF && g->viscous != CFS_VISCOUS_NS) { msg = "unknown viscous mode"; return CFS_ERR_INVALID; }
    if (g->variant < 0 || g->variant > cfs::kNumVariants) { msg = "unknown kernel variant"; return CFS_ERR_INVALID; }
    if (g->march_rows < 0 || g->march_rows > 4096) { msg = "march_rows out of range 0..4096"; return CFS_ERR_INVALID; }
    if (g->positivity < CFS_POSITIVITY_OFF || g->positivity > CFS_POSITIVITY_FLOOR) {
        msg = "unknown positivity mode";
        return CFS_ERR_INVALID;
    }
    if (g->rounding != CFS_ROUND_STOCHASTIC && g->rounding != CFS_ROUND_NEAREST &&
        g->rounding != CFS_ROUND_STOCHASTIC_ALL) {
        msg = "unknown rounding mode";
        return CFS_ERR_INVALID;
    }
    if (g->precision == CFS_FP64_EXACT && g->positivity != CFS_POSITIVITY_OFF) {
        msg = "FP64_EXACT runs the reference's scheme: positivity fallbacks need FP64 or FP32_MIXED";
        return CFS_ERR_INVALID;
    }
    if (g->viscous == CFS_VISCOUS_NS && (!(g->mu >= 0) || !(g->prandtl > 0) || !(g->mach > 0))) {
        msg = "viscous terms need mu >= 0, prandtl > 0 and mach > 0";
        return CFS_ERR_INVALID;
    }
    return CFS_OK;
}

cfs::StageArgs base_args(const cfs_ctx* c) {
    cfs::StageArgs a{};
    a.L = c->L;
    for (int s = 0; s < 4; ++s) a.bc[s] = c->sides.bc[s];
    a.gamma = c->cfg.gamma;
    a.eps = c->cfg.weno_eps;
    a.dx = c->dx;
    a.dy = c->dy;
    a.rk = c->cfg.rk;
    a.hll = c->cfg.hll;
    a.viscous = c->cfg.viscous;
    a.mu = c->cfg.mu;
    a.prandtl = c->cfg.prandtl;
    a.mach = c->cfg.mach;
    a.types = c->has_types ? c->types_d : nullptr;
    a.variant = c->cfg.variant;
    a.rows = c->cfg.march_rows;
    a.positivity = c->cfg.positivity;
    a.rounding = c->cfg.rounding;
    a.seed = c->steps_done;
    a.lowo = c->cfg.positivity >= CFS_POSITIVITY_BODY && c->has_types ? c->lowo_d : nullptr;
    a.cflags = c->has_types ? c->cflags_d : nullptr;
    a.bflux = c->bflux;
    a.err = c->err_d;
    return a;
}

// Device error flags set by bounded waits in the kernels; read (and cleared)
// at the calls that wait for the stream.
int check_device_errors(cfs_ctx* c) {
    unsigned int e = 0;
    CFS_CUDA(c, cudaMemcpyAsync(&e, c->err_d, sizeof(e), cudaMemcpyDeviceToHost, c->stream));
    CFS_CUDA(c, cudaStreamSynchronize(c->stream));
    if (e != 0) {
        CFS_CUDA(c, cudaMemsetAsync(c->err_d, 0, sizeof(unsigned int), c->stream));
        return fail(c, CFS_ERR_CUDA, "a TMA row copy did not complete within its bounded wait (device flag " +
                                         std::to_string(e) + ")");
    }
    return CFS_OK;
}

cfs::IbArgs ib_args(const cfs_ctx* c, void* U) {
    cfs::IbArgs a{};
    a.U = U;
    a.L = c->L;
    a.n = c->ib_n;
    a.mode = c->ib_mode;
    a.cell = c->ib_cell;
    a.donor = c->ib_donor;
    a.image = c->ib_img;
    a.fac = c->ib_fac;
    a.perm = c->ib_perm;
    return a;
}

// Buffer roles of one stage: reads `in` (+ u0, u1 pointwise), writes `out`.
struct Roles {
    int in, out, u0, u1;
};

Roles roles_for(const cfs_ctx* c, int stage, int cur, int u0_idx, int u1_idx) {
    Roles r{cur, -1, u0_idx, u1_idx};
    if (stage == 0) {
        r.u0 = cur;
        r.out = (cur + 1) % 3;
    } else if (stage == 1) {
        r.u1 = cur;
        if (c->cfg.rk == CFS_RK_TVD2) r.out = u0_idx;
        else r.out = 3 - u0_idx - cur;  // the buffer that is neither
    } else {
        r.out = u0_idx;
    }
    return r;
}

// Enqueues one stage (immersed-ghost fill + stage kernel).  P/parity/flags
// select graph mode.
int enqueue_stage(cfs_ctx* c, int stage, const Roles& r, double dt, bool graph_mode, int parity, bool first,
                  bool last, int row_lo = 0, int row_hi = 0, bool with_fill = true) {
    if (with_fill && c->ib_n > 0) CFS_CUDA(c, cfs::launch_ib_fill(c->L.elem_bytes, ib_args(c, c->S[r.in]), c->stream));
    if (c->rv && with_fill) {
        cfs::ViscArgs va{};
        va.in = c->S[r.in];
        va.rv = c->rv;
        va.L = c->L;
        va.gamma = c->cfg.gamma;
        va.dx = c->dx;
        va.dy = c->dy;
        va.inv_dx = 1.0 / c->dx;
        va.inv_dy = 1.0 / c->dy;
        va.mu = c->cfg.mu;
        va.mach2 = c->cfg.mach * c->cfg.mach;
        va.kT = c->cfg.mu / ((c->cfg.gamma - 1) * va.mach2 * c->cfg.prandtl);
        va.gm1_f = static_cast<float>(va.gamma - 1);
        va.cT_f = static_cast<float>(va.gamma * va.mach2);
        va.mu_f = static_cast<float>(va.mu);
        va.kT_f = static_cast<float>(va.kT);
        va.inv_dx_f = static_cast<float>(va.inv_dx);
        va.inv_dy_f = static_cast<float>(va.inv_dy);
        CFS_CUDA(c, cfs::launch_viscous(c->prec, va, c->stream));
    }
    cfs::StageArgs a = base_args(c);
    a.rv = c->rv;
    a.in = c->S[r.in];
    a.u0 = r.u0 >= 0 ? c->S[r.u0] : nullptr;
    a.u1 = r.u1 >= 0 ? c->S[r.u1] : nullptr;
    a.out = c->S[r.out];
    if (c->has_tmaps) {
        a.has_tmaps = 1;
        std::memcpy(a.tmap_in, c->tmaps[r.in], cfs::kTensorMapBytes);
        if (r.u0 >= 0) std::memcpy(a.tmap_u0, c->tmaps[r.u0], cfs::kTensorMapBytes);
    }
    a.rhs = c->cfg.keep_rhs ? c->rhs : nullptr;
    a.stage = stage;
    a.dt = dt;
    a.row_lo = row_lo;
    a.row_hi = row_hi;
    if (graph_mode) {
        a.P = c->P;
        a.parity = parity;
        a.first_stage = first ? 1 : 0;
        a.last_stage = last ? 1 : 0;
    }
    CFS_CUDA(c, cfs::launch_stage(c->prec, a, c->stream));
    return CFS_OK;
}

int run_stage(cfs_ctx* c, int stage, double dt) {
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    c->wmax_carry = false;
    if (stage > 0 && stage != c->next_stage)
        return fail(c, CFS_ERR_STATE, "stage " + std::to_string(stage) + " requested but the RK sequence expects stage " +
                                          std::to_string(c->next_stage));
    const Roles r = roles_for(c, stage, c->cur, c->u0_idx, c->u1_idx);
    const int rc = enqueue_stage(c, stage, r, dt, false, 0, false, false);
    if (rc != CFS_OK) return rc;
    if (stage == 0) c->u0_idx = r.u0;
    if (stage == 1) c->u1_idx = r.u1;
    c->cur = r.out;
    c->next_stage = (stage + 1) % stages_per_step(c->cfg.rk);
    if (c->next_stage == 0) ++c->steps_done;
    return CFS_OK;
}

// Upload of per-ghost data for the device fill.  Reference form: the pivoted
// LDL^T factor of each donor matrix.  Slip form: donors and weights from
// cfs::slip_donors (the given donors serve as its fallback).
int upload_ib(cfs_ctx* c, int mode, int n, const int32_t* cell, const int32_t* donor4, const double* image,
              const double* normal) {
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    release_graph(c);
    cudaFree(c->ib_cell);
    cudaFree(c->ib_donor);
    cudaFree(c->ib_perm);
    cudaFree(c->ib_img);
    cudaFree(c->ib_fac);
    c->ib_cell = c->ib_donor = c->ib_perm = nullptr;
    c->ib_img = c->ib_fac = nullptr;
    c->ib_n = 0;
    c->ib_cell_h.assign(cell, cell + n);
    c->ib_donor_h.assign(donor4, donor4 + 4 * static_cast<size_t>(n));
    c->ib_img_h.assign(image, image + 2 * static_cast<size_t>(n));
    if (n == 0) return CFS_OK;
    std::vector<uint8_t> fluid_all;
    const uint8_t* types = c->has_types ? c->types_h.data() : nullptr;
    if (!types) {
        fluid_all.assign(static_cast<size_t>(c->cfg.nx) * c->cfg.ny, 0);
        types = fluid_all.data();
    }
    std::vector<int32_t> dev_donor;
    std::vector<double> fac;
    std::vector<int> perm;
    cfs::ib_factors(mode, types, c->cfg.nx, c->cfg.ny, c->dx, c->dy, n, donor4, image, normal, dev_donor, fac, perm);
    CFS_CUDA(c, cudaMalloc(&c->ib_cell, sizeof(int) * n));
    CFS_CUDA(c, cudaMalloc(&c->ib_donor, sizeof(int) * 4 * n));
    CFS_CUDA(c, cudaMalloc(&c->ib_perm, sizeof(int) * 4 * n));
    CFS_CUDA(c, cudaMalloc(&c->ib_img, sizeof(double) * 2 * n));
    CFS_CUDA(c, cudaMalloc(&c->ib_fac, sizeof(double) * 16 * n));
    CFS_CUDA(c, cudaMemcpy(c->ib_cell, cell, sizeof(int) * n, cudaMemcpyHostToDevice));
    CFS_CUDA(c, cudaMemcpy(c->ib_donor, dev_donor.data(), sizeof(int) * 4 * n, cudaMemcpyHostToDevice));
    CFS_CUDA(c, cudaMemcpy(c->ib_perm, perm.data(), sizeof(int) * 4 * n, cudaMemcpyHostToDevice));
    CFS_CUDA(c, cudaMemcpy(c->ib_img, image, sizeof(double) * 2 * n, cudaMemcpyHostToDevice));
    CFS_CUDA(c, cudaMemcpy(c->ib_fac, fac.data(), sizeof(double) * 16 * n, cudaMemcpyHostToDevice));
    c->ib_n = n;
    c->ib_mode = mode;
    return CFS_OK;
}

}  // namespace

namespace cfs {
// Error message of a context-free entry point, read by cfs_last_error(NULL)
// (the thread's last CUDA error consumed as in fail(): on CUDA and allocation
// failures only).
void record_global_error(int code, const std::string& msg) {
    g_create_error = msg;
    if (code == CFS_ERR_CUDA || code == CFS_ERR_NOMEM) (void)cudaGetLastError();
}

cudaError_t launch_stage(Prec p, const StageArgs& a, cudaStream_t s) {
    if (p == kF64Exact) return launch_stage_exact(a, s);
    if (p == kF32Mixed) return launch_stage_f32(a, s);
    return launch_stage_f64(a, s);
}
cudaError_t launch_viscous(Prec p, const ViscArgs& a, cudaStream_t s) {
    if (p == kF32Mixed) return launch_viscous_f32(a, s);
    return launch_viscous_f64(a, s);
}
cudaError_t launch_weno_faces(Prec p, int n, const double* st, double* l, double* r, double g, double eps, cudaStream_t s) {
    if (p == kF64Exact) return launch_weno_faces_exact(n, st, l, r, g, eps, s);
    if (p == kF32Mixed) return launch_weno_faces_f32(n, st, l, r, g, eps, s);
    return launch_weno_faces_f64(n, st, l, r, g, eps, s);
}
cudaError_t launch_hll_faces(Prec p, int n, int dir, const double* L, const double* R, double* F, double g, int v,
                             cudaStream_t s) {
    if (p == kF64Exact) return launch_hll_faces_exact(n, dir, L, R, F, g, v, s);
    if (p == kF32Mixed) return launch_hll_faces_f32(n, dir, L, R, F, g, v, s);
    return launch_hll_faces_f64(n, dir, L, R, F, g, v, s);
}
}  // namespace cfs

extern "C" {

int cfs_abi_version(void) { return CFS_ABI_VERSION; }

int cfs_variant_count(void) { return cfs::kNumVariants; }

int cfs_variant_info(int v, int* rows, int* warps, int* min_blocks, int* prefetch) {
    if (v < 1 || v > cfs::kNumVariants) return fail(nullptr, CFS_ERR_INVALID, "unknown kernel variant");
    if (rows) *rows = cfs::kVariants[v - 1].rows;
    if (warps) *warps = cfs::kVariants[v - 1].warps;
    if (min_blocks) *min_blocks = cfs::kVariants[v - 1].min_blocks;
    if (prefetch) *prefetch = cfs::kVariants[v - 1].load;
    return CFS_OK;
}

void cfs_config_default(cfs_config* g) {
    if (!g) return;
    std::memset(g, 0, sizeof(*g));
    g->nx = g->ny = 64;
    g->lx = g->ly = 1.0;
    g->gamma = 1.4;
    g->weno_eps = 1e-2;
    g->precision = CFS_FP64;
    g->rk = CFS_RK_TVD3_REFERENCE;
    g->hll = CFS_HLL_REFERENCE;
    for (int s = 0; s < 4; ++s) g->bc[s] = CFS_BC_NEUMANN;
    g->viscous = CFS_VISCOUS_OFF;
    g->mu = 1e-3;
    g->prandtl = 0.72;
    g->mach = 1.0;
    g->rounding = CFS_ROUND_STOCHASTIC_ALL;
}

const char* cfs_last_error(const cfs_ctx* c) { return c ? c->err.c_str() : g_create_error.c_str(); }

int cfs_create(const cfs_config* cfg, cfs_ctx** out) {
    if (!out) return fail(nullptr, CFS_ERR_INVALID, "null output pointer");
    *out = nullptr;
    std::string msg;
    const int v = validate(cfg, msg);
    if (v != CFS_OK) return fail(nullptr, v, msg);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(nullptr, CFS_ERR_CUDA, "no CUDA device available (the engine has no CPU path)");
    if (cfg->device < 0 || cfg->device >= ndev) return fail(nullptr, CFS_ERR_INVALID, "device ordinal out of range");
    cfs_ctx* c = new (std::nothrow) cfs_ctx();
    if (!c) return fail(nullptr, CFS_ERR_NOMEM, "host allocation failed");
    c->cfg = *cfg;
    c->prec = cfg->precision == CFS_FP32_MIXED ? cfs::kF32Mixed : (cfg->precision == CFS_FP64_EXACT ? cfs::kF64Exact : cfs::kF64);
    c->L = cfs::Layout::make(cfg->nx, cfg->ny, c->prec == cfs::kF32Mixed ? 4 : 8);
    c->dx = cfg->lx / cfg->nx;  // CartesianMesh::CalCellsize (CartesianMesh.cpp:150-154)
    c->dy = cfg->ly / cfg->ny;
    for (int s = 0; s < 4; ++s) {
        c->sides.bc[s] = cfg->bc[s];
        // DirichletBoundary ghost: rho, rho u, rho v, E from p (Cylinder.cpp:22-32,
        // EulerPhase::computeEnergyfromOther, EulerPhase.cpp:124-128).
        const double rho = cfg->bc_prim[s][0], u = cfg->bc_prim[s][1], vv = cfg->bc_prim[s][2], p = cfg->bc_prim[s][3];
        const double mx = rho * u, my = rho * vv;
        const double e = p / (cfg->gamma - 1);
        c->sides.U[s][0] = rho;
        c->sides.U[s][1] = mx;
        c->sides.U[s][2] = my;
        c->sides.U[s][3] = e + 0.5 * (mx * mx + my * my) / rho;
    }
    auto bail = [&](int code) {
        const std::string m = c->err;
        cfs_destroy(c);
        return fail(nullptr, code, m);
    };
    if (cudaSetDevice(cfg->device) != cudaSuccess) { c->err = "cudaSetDevice failed"; return bail(CFS_ERR_CUDA); }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { c->err = "stream creation failed"; return bail(CFS_ERR_CUDA); }
    const size_t sb = static_cast<size_t>(c->L.bytes());
    for (int b = 0; b < 3; ++b) {
        if (cudaMalloc(&c->S[b], sb) != cudaSuccess) { c->err = "device allocation of the state failed"; return bail(CFS_ERR_NOMEM); }
        cudaMemsetAsync(c->S[b], 0, sb, c->stream);
    }
    const size_t hb = sizeof(double) * kVars * static_cast<size_t>(cfg->nx) * cfg->ny;
    if (cudaMalloc(&c->staging, hb) != cudaSuccess) { c->err = "device allocation of the staging buffer failed"; return bail(CFS_ERR_NOMEM); }
    if (cudaMalloc(&c->sums, sizeof(double) * cfs::plane_sums_scratch_doubles()) != cudaSuccess) {
        c->err = "device allocation of the sum scratch failed";
        return bail(CFS_ERR_NOMEM);
    }
    if (cfg->viscous == CFS_VISCOUS_NS) {
        const size_t vb = static_cast<size_t>(3) * cfg->nx * cfg->ny * c->L.elem_bytes;
        if (cudaMalloc(&c->rv, vb) != cudaSuccess) { c->err = "device allocation of the viscous RHS failed"; return bail(CFS_ERR_NOMEM); }
        cudaMemsetAsync(c->rv, 0, vb, c->stream);
    }
    bool physical = false;
    for (int s = 0; s < 4; ++s) physical = physical || cfg->bc[s] == CFS_BC_NEUMANN || cfg->bc[s] == CFS_BC_DIRICHLET;
    if (physical && c->prec != cfs::kF64Exact) {
        const size_t bb = static_cast<size_t>(cfs::bflux_count(c->L)) * c->L.elem_bytes;
        if (cudaMalloc(&c->bflux, bb) != cudaSuccess) { c->err = "device allocation of the boundary fluxes failed"; return bail(CFS_ERR_NOMEM); }
    }
    if (cfg->keep_rhs) {
        if (cudaMalloc(&c->rhs, hb) != cudaSuccess) { c->err = "device allocation of the RHS buffer failed"; return bail(CFS_ERR_NOMEM); }
        cudaMemsetAsync(c->rhs, 0, hb, c->stream);
    }
    if (cudaMalloc(&c->P, sizeof(cfs::DevParams)) != cudaSuccess || cudaMalloc(&c->wmax, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&c->totals, 4 * sizeof(double)) != cudaSuccess || cudaMalloc(&c->err_d, sizeof(unsigned int)) != cudaSuccess) {
        c->err = "device allocation of the reduction slots failed";
        return bail(CFS_ERR_NOMEM);
    }
    cudaMemsetAsync(c->P, 0, sizeof(cfs::DevParams), c->stream);
    cudaMemsetAsync(c->err_d, 0, sizeof(unsigned int), c->stream);
    // (without it, cfs_advance copies its parameters through pageable memory)
    if (cudaHostAlloc(&c->hp_pin, 2 * sizeof(cfs::DevParams), cudaHostAllocDefault) != cudaSuccess) {
        (void)cudaGetLastError();
        c->hp_pin = nullptr;
    }
    if (c->prec != cfs::kF64Exact) {
        // tensor maps of the three state buffers (TMA load schedule), encoded
        // on the host once (the buffers never move) and passed in each
        // stage's argument block
        for (int b = 0; b < 3; ++b) {
            if (cfs::encode_state_map(c->S[b], c->L, c->tmaps[b]) != cudaSuccess) {
                c->err = "tensor map encoding of the state buffers failed";
                return bail(CFS_ERR_CUDA);
            }
        }
        c->has_tmaps = true;
    }
    for (int b = 0; b < 3; ++b) cfs::launch_ghost_fill(c->L.elem_bytes, c->S[b], c->L, c->sides, c->stream);
    // the clears and ghost fills above are checked here, at enqueue and at completion
    cudaError_t ie = cudaStreamSynchronize(c->stream);
    if (ie == cudaSuccess) ie = cudaGetLastError();
    if (ie != cudaSuccess) { c->err = std::string("initialisation failed: ") + cudaGetErrorString(ie); return bail(CFS_ERR_CUDA); }
    *out = c;
    return CFS_OK;
}

int cfs_destroy(cfs_ctx* c) {
    if (!c) return CFS_OK;
    cudaSetDevice(c->cfg.device);  // best effort: the frees below belong to that device
    if (c->stream) cudaStreamSynchronize(c->stream);
    release_graph(c);
    for (void* p : c->S) cudaFree(p);
    cudaFree(c->rhs);
    cudaFree(c->staging);
    cudaFree(c->sums);
    if (c->host_stage) cudaFreeHost(c->host_stage);
    cudaFree(c->rv);
    cudaFree(c->types_d);
    cudaFree(c->lowo_d);
    cudaFree(c->cflags_d);
    cudaFree(c->bflux);
    cudaFree(c->ib_cell);
    cudaFree(c->ib_donor);
    cudaFree(c->ib_perm);
    cudaFree(c->ib_img);
    cudaFree(c->ib_fac);
    cudaFree(c->P);
    if (c->hp_pin) cudaFreeHost(c->hp_pin);
    cudaFree(c->wmax);
    cudaFree(c->totals);
    cudaFree(c->err_d);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return CFS_OK;
}

// Copies of caller arrays: pinned arrays and small copies go straight to the
// DMA engine; large pageable ones through the chunked pipeline of a pinned
// staging buffer (allocated on first use; without it, the plain copy).
static bool ensure_host_stage(cfs_ctx* c, size_t bytes) {
    if (c->host_stage_bytes >= bytes) return true;
    if (c->host_stage) cudaFreeHost(c->host_stage);
    c->host_stage = nullptr;
    c->host_stage_bytes = 0;
    if (cudaHostAlloc(&c->host_stage, bytes, cudaHostAllocDefault) != cudaSuccess) {
        (void)cudaGetLastError();
        c->host_stage = nullptr;
        return false;
    }
    c->host_stage_bytes = bytes;
    return true;
}

static bool staged(cfs_ctx* c, const void* host, size_t bytes) {
    return bytes >= cfs::kStagedCopyMinBytes && cfs::host_is_pageable(host) && ensure_host_stage(c, bytes);
}

static cudaError_t copy_in(cfs_ctx* c, void* dst, const void* src, size_t bytes) {
    if (staged(c, src, bytes)) return cfs::upload_staged(dst, src, bytes, c->host_stage, c->stream, c->cfg.device);
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
}

// (returns once dst holds the data)
static cudaError_t copy_out(cfs_ctx* c, void* dst, const void* src, size_t bytes) {
    if (staged(c, dst, bytes)) return cfs::download_staged(dst, src, bytes, c->host_stage, c->stream, c->cfg.device);
    const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
    return e != cudaSuccess ? e : cudaStreamSynchronize(c->stream);
}

int cfs_set_state(cfs_ctx* c, const double* U) {
    if (!c || !U) return fail(c, CFS_ERR_INVALID, "null argument");
    c->wmax_carry = false;
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    const size_t hb = sizeof(double) * kVars * static_cast<size_t>(c->cfg.nx) * c->cfg.ny;
    CFS_CUDA(c, copy_in(c, c->staging, U, hb));
    if (c->L.elem_bytes == 4) {
        // FP32 storage offsets: the FP32-rounded mean of each variable, summed
        // on the device from the uploaded state (a fixed summation order)
        const size_t n = static_cast<size_t>(c->cfg.nx) * c->cfg.ny;
        double sums[kVars] = {0, 0, 0, 0};
        if (!c->fixed_offsets) {
            CFS_CUDA(c, cfs::launch_plane_sums(c->staging, static_cast<long long>(n), c->sums, c->stream));
            CFS_CUDA(c, cudaMemcpyAsync(sums, c->sums + cfs::plane_sums_scratch_doubles() - kVars, sizeof(sums),
                                        cudaMemcpyDeviceToHost, c->stream));
            CFS_CUDA(c, cudaStreamSynchronize(c->stream));
        }
        bool changed = false;
        for (int v = 0; v < kVars; ++v) {
            float off = c->fixed_offsets ? c->fixed_off[v] : static_cast<float>(sums[v] / static_cast<double>(n));
            if (!std::isfinite(off)) off = 0.0f;
            changed = changed || off != c->L.off[v];
            c->L.off[v] = off;
        }
        if (changed) release_graph(c);
    }
    CFS_CUDA(c, cfs::launch_pack(c->L.elem_bytes, c->staging, c->S[0], c->L, c->stream));
    for (int b = 0; b < 3; ++b) CFS_CUDA(c, cfs::launch_ghost_fill(c->L.elem_bytes, c->S[b], c->L, c->sides, c->stream));
    CFS_CUDA(c, cudaStreamSynchronize(c->stream));
    c->cur = 0;
    c->u0_idx = c->u1_idx = -1;
    c->next_stage = 0;
    return CFS_OK;
}

int cfs_set_storage_offsets(cfs_ctx* c, const double* off4) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    c->fixed_offsets = off4 != nullptr;
    for (int v = 0; v < kVars; ++v) c->fixed_off[v] = off4 ? static_cast<float>(off4[v]) : 0.0f;
    return CFS_OK;
}

int cfs_get_step(cfs_ctx* c, unsigned int* step, double* cfl_max, double* off4) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    if (step) *step = c->steps_done;
    if (cfl_max) {
        double m = 0.0;
        if (c->wmax_carry) std::memcpy(&m, &c->wmax_bits, sizeof(m));
        *cfl_max = m;
    }
    if (off4)
        for (int v = 0; v < kVars; ++v) off4[v] = static_cast<double>(c->L.off[v]);
    return CFS_OK;
}

int cfs_set_step(cfs_ctx* c, unsigned int step, double cfl_max) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    if (!(cfl_max >= 0) || !std::isfinite(cfl_max)) return fail(c, CFS_ERR_INVALID, "cfl_max must be finite and >= 0");
    if (c->next_stage != 0) return fail(c, CFS_ERR_STATE, "a step is in progress (stage sequence not at stage 0)");
    c->steps_done = step;
    c->wmax_carry = cfl_max > 0;
    c->wmax_bits = 0;
    if (c->wmax_carry) std::memcpy(&c->wmax_bits, &cfl_max, sizeof(cfl_max));
    return CFS_OK;
}

int cfs_get_state(cfs_ctx* c, double* U) {
    if (!c || !U) return fail(c, CFS_ERR_INVALID, "null argument");
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    const size_t hb = sizeof(double) * kVars * static_cast<size_t>(c->cfg.nx) * c->cfg.ny;
    CFS_CUDA(c, cfs::launch_unpack(c->L.elem_bytes, c->S[c->cur], c->staging, c->L, c->stream));
    CFS_CUDA(c, copy_out(c, U, c->staging, hb));
    return check_device_errors(c);
}

int cfs_get_rhs(cfs_ctx* c, double* R) {
    if (!c || !R) return fail(c, CFS_ERR_INVALID, "null argument");
    if (!c->cfg.keep_rhs) return fail(c, CFS_ERR_STATE, "context created without keep_rhs");
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    const size_t hb = sizeof(double) * kVars * static_cast<size_t>(c->cfg.nx) * c->cfg.ny;
    CFS_CUDA(c, copy_out(c, R, c->rhs, hb));
    return CFS_OK;
}

int cfs_set_cell_types(cfs_ctx* c, const uint8_t* types) {
    if (!c || !types) return fail(c, CFS_ERR_INVALID, "null argument");
    c->wmax_carry = false;
    const size_t n = static_cast<size_t>(c->cfg.nx) * c->cfg.ny;
    for (size_t k = 0; k < n; ++k)
        if (types[k] > 2) return fail(c, CFS_ERR_INVALID, "cell type out of range at " + std::to_string(k));
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    release_graph(c);
    if (!c->types_d) CFS_CUDA(c, cudaMalloc(&c->types_d, n));
    CFS_CUDA(c, cudaMemcpy(c->types_d, types, n, cudaMemcpyHostToDevice));
    c->types_h.assign(types, types + n);
    c->has_types = true;
    std::vector<uint8_t> f;
    if (c->cfg.positivity >= CFS_POSITIVITY_BODY) {
        f = cfs::low_order_faces(types, c->cfg.nx, c->cfg.ny, c->cfg.bc);
        if (!c->lowo_d) CFS_CUDA(c, cudaMalloc(&c->lowo_d, f.size()));
        CFS_CUDA(c, cudaMemcpy(c->lowo_d, f.data(), f.size(), cudaMemcpyHostToDevice));
    }
    const std::vector<uint8_t> cf = cfs::cell_flags(types, f.empty() ? nullptr : f.data(), c->cfg.nx, c->cfg.ny);
    if (!c->cflags_d) CFS_CUDA(c, cudaMalloc(&c->cflags_d, cf.size()));
    CFS_CUDA(c, cudaMemcpy(c->cflags_d, cf.data(), cf.size(), cudaMemcpyHostToDevice));
    return CFS_OK;
}

int cfs_set_ib(cfs_ctx* c, int mode, int n, const int32_t* cell, const int32_t* donor4, const double* image_xy,
               const double* normal_xy) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    c->wmax_carry = false;
    if (mode != CFS_IB_REFERENCE && mode != CFS_IB_BILINEAR_SLIP) return fail(c, CFS_ERR_INVALID, "unknown IB mode");
    if (n < 0 || (n > 0 && (!cell || !donor4 || !image_xy))) return fail(c, CFS_ERR_INVALID, "bad IB list");
    if (n > 0 && mode == CFS_IB_BILINEAR_SLIP && !normal_xy) return fail(c, CFS_ERR_INVALID, "slip mode needs wall normals");
    const long long ncell = static_cast<long long>(c->cfg.nx) * c->cfg.ny;
    for (int g = 0; g < n; ++g) {
        if (cell[g] < 0 || cell[g] >= ncell) return fail(c, CFS_ERR_INVALID, "IB cell index out of range");
        for (int k = 0; k < 4; ++k)
            if (donor4[4 * g + k] < 0 || donor4[4 * g + k] >= ncell) return fail(c, CFS_ERR_INVALID, "IB donor index out of range");
    }
    return upload_ib(c, mode, n, cell, donor4, image_xy, normal_xy);
}

int cfs_ib_build_circle(cfs_ctx* c, double radius, double cx, double cy, int npoints, int mode) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    cfs::IbList ib;
    std::string err;
    if (!cfs::build_circle(c->cfg.nx, c->cfg.ny, c->cfg.lx, c->cfg.ly, radius, cx, cy, npoints, ib, err))
        return fail(c, CFS_ERR_INVALID, err);
    const int rc = cfs_set_cell_types(c, ib.types.data());
    if (rc != CFS_OK) return rc;
    return cfs_set_ib(c, mode, static_cast<int>(ib.cell.size()), ib.cell.data(), ib.donor.data(), ib.image.data(),
                      ib.normal.data());
}

int cfs_ib_build_circle_device(cfs_ctx* c, double radius, double cx, double cy, int npoints, int mode) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    cfs::IbList ib;
    std::string err;
    if (!cfs::build_circle_device(c->cfg.nx, c->cfg.ny, c->cfg.lx, c->cfg.ly, radius, cx, cy, npoints, c->stream, ib, err))
        return fail(c, err.rfind("device circle set-up", 0) == 0 ? CFS_ERR_CUDA : CFS_ERR_INVALID, err);
    const int rc = cfs_set_cell_types(c, ib.types.data());
    if (rc != CFS_OK) return rc;
    return cfs_set_ib(c, mode, static_cast<int>(ib.cell.size()), ib.cell.data(), ib.donor.data(), ib.image.data(),
                      ib.normal.data());
}

namespace {

int circle_setup_out(const cfs::IbList& ib, uint8_t* types, int max_n, int* n, int32_t* cell, int32_t* donor4,
                     double* image_xy, double* normal_xy) {
    if (types) std::memcpy(types, ib.types.data(), ib.types.size());
    const int total = static_cast<int>(ib.cell.size());
    if (n) *n = total;
    const int m = total < max_n ? total : max_n;
    for (int g = 0; g < m; ++g) {
        if (cell) cell[g] = ib.cell[g];
        for (int k = 0; k < 4; ++k)
            if (donor4) donor4[4 * g + k] = ib.donor[4 * g + k];
        for (int k = 0; k < 2; ++k) {
            if (image_xy) image_xy[2 * g + k] = ib.image[2 * g + k];
            if (normal_xy) normal_xy[2 * g + k] = ib.normal[2 * g + k];
        }
    }
    return CFS_OK;
}

}  // namespace

int cfs_circle_setup(int nx, int ny, double lx, double ly, double radius, double cx, double cy, int npoints,
                     uint8_t* types, int max_n, int* n, int32_t* cell, int32_t* donor4, double* image_xy,
                     double* normal_xy) {
    if (nx < 1 || ny < 1 || !(lx > 0) || !(ly > 0)) return fail(nullptr, CFS_ERR_INVALID, "bad grid");
    cfs::IbList ib;
    std::string err;
    if (!cfs::build_circle(nx, ny, lx, ly, radius, cx, cy, npoints, ib, err)) return fail(nullptr, CFS_ERR_INVALID, err);
    return circle_setup_out(ib, types, max_n, n, cell, donor4, image_xy, normal_xy);
}

int cfs_ib_build_polygon(cfs_ctx* c, int npoints, const double* xy, int mode) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    if (npoints < 3 || !xy) return fail(c, CFS_ERR_INVALID, "a polygon needs at least 3 vertices");
    cfs::IbList ib;
    std::string err;
    if (!cfs::build_polygon(c->cfg.nx, c->cfg.ny, c->cfg.lx, c->cfg.ly,
                            std::vector<double>(xy, xy + 2 * static_cast<size_t>(npoints)), ib, err))
        return fail(c, CFS_ERR_INVALID, err);
    const int rc = cfs_set_cell_types(c, ib.types.data());
    if (rc != CFS_OK) return rc;
    return cfs_set_ib(c, mode, static_cast<int>(ib.cell.size()), ib.cell.data(), ib.donor.data(), ib.image.data(),
                      ib.normal.data());
}

int cfs_polygon_setup(int nx, int ny, double lx, double ly, int npoints, const double* xy, uint8_t* types, int max_n,
                      int* n, int32_t* cell, int32_t* donor4, double* image_xy, double* normal_xy) {
    if (nx < 1 || ny < 1 || !(lx > 0) || !(ly > 0)) return fail(nullptr, CFS_ERR_INVALID, "bad grid");
    if (npoints < 3 || !xy) return fail(nullptr, CFS_ERR_INVALID, "a polygon needs at least 3 vertices");
    cfs::IbList ib;
    std::string err;
    if (!cfs::build_polygon(nx, ny, lx, ly, std::vector<double>(xy, xy + 2 * static_cast<size_t>(npoints)), ib, err))
        return fail(nullptr, CFS_ERR_INVALID, err);
    return circle_setup_out(ib, types, max_n, n, cell, donor4, image_xy, normal_xy);
}

int cfs_circle_setup_device(int device, int nx, int ny, double lx, double ly, double radius, double cx, double cy,
                            int npoints, uint8_t* types, int max_n, int* n, int32_t* cell, int32_t* donor4,
                            double* image_xy, double* normal_xy) {
    if (nx < 1 || ny < 1 || !(lx > 0) || !(ly > 0)) return fail(nullptr, CFS_ERR_INVALID, "bad grid");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(nullptr, CFS_ERR_CUDA, "no CUDA device available (the device set-up has no CPU path)");
    if (device < 0 || device >= ndev) return fail(nullptr, CFS_ERR_INVALID, "device ordinal out of range");
    if (cudaSetDevice(device) != cudaSuccess) return fail(nullptr, CFS_ERR_CUDA, "cudaSetDevice failed");
    cfs::IbList ib;
    std::string err;
    if (!cfs::build_circle_device(nx, ny, lx, ly, radius, cx, cy, npoints, nullptr, ib, err))
        return fail(nullptr, err.rfind("device circle set-up", 0) == 0 ? CFS_ERR_CUDA : CFS_ERR_INVALID, err);
    return circle_setup_out(ib, types, max_n, n, cell, donor4, image_xy, normal_xy);
}

int cfs_get_ib(cfs_ctx* c, uint8_t* types, int max_n, int* n, int32_t* cell, int32_t* donor4, double* image_xy) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    const size_t nc = static_cast<size_t>(c->cfg.nx) * c->cfg.ny;
    if (types) {
        if (c->has_types) std::memcpy(types, c->types_h.data(), nc);
        else std::memset(types, 0, nc);
    }
    const int total = static_cast<int>(c->ib_cell_h.size());
    if (n) *n = total;
    const int m = total < max_n ? total : max_n;
    for (int g = 0; g < m; ++g) {
        if (cell) cell[g] = c->ib_cell_h[g];
        for (int k = 0; k < 4; ++k)
            if (donor4) donor4[4 * g + k] = c->ib_donor_h[4 * g + k];
        if (image_xy) {
            image_xy[2 * g] = c->ib_img_h[2 * g];
            image_xy[2 * g + 1] = c->ib_img_h[2 * g + 1];
        }
    }
    return CFS_OK;
}

int cfs_ib_fill(cfs_ctx* c) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    c->wmax_carry = false;
    if (c->ib_n == 0) return CFS_OK;
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    CFS_CUDA(c, cfs::launch_ib_fill(c->L.elem_bytes, ib_args(c, c->S[c->cur]), c->stream));
    return CFS_OK;
}

int cfs_compute_dt(cfs_ctx* c, double cfl, double* dt) {
    if (!c || !dt) return fail(c, CFS_ERR_INVALID, "null argument");
    if (!(cfl > 0)) return fail(c, CFS_ERR_INVALID, "cfl must be positive");
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    CFS_CUDA(c, cudaMemsetAsync(c->wmax, 0, sizeof(unsigned long long), c->stream));
    CFS_CUDA(c, cfs::launch_wmax(c->L.elem_bytes, c->S[c->cur], c->L, c->has_types ? c->types_d : nullptr, c->cfg.gamma,
                                 c->dx, c->dy, c->wmax, c->stream));
    unsigned long long bits = 0;
    CFS_CUDA(c, cudaMemcpyAsync(&bits, c->wmax, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
    CFS_CUDA(c, cudaStreamSynchronize(c->stream));
    double m;
    std::memcpy(&m, &bits, sizeof(m));
    if (!(m > 0) || !std::isfinite(m))
        return fail(c, CFS_ERR_NUMERIC, "CFL reduction: a fluid cell is non-finite or every wave speed is 0");
    *dt = cfl / m;
    return CFS_OK;
}

int cfs_stage(cfs_ctx* c, int counter, double dt) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    if (counter < 1) return fail(c, CFS_ERR_INVALID, "loop counter starts at 1 (Run.cpp:153)");
    return run_stage(c, stage_of_counter(c->cfg.rk, counter), dt);
}

int cfs_step(cfs_ctx* c, double dt) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    if (c->next_stage != 0) return fail(c, CFS_ERR_STATE, "a step is in progress (stage sequence not at stage 0)");
    for (int s = 0; s < stages_per_step(c->cfg.rk); ++s) {
        const int rc = run_stage(c, s, dt);
        if (rc != CFS_OK) return rc;
    }
    return CFS_OK;
}

int cfs_advance(cfs_ctx* c, int nsteps, double cfl, double dt, double* t_elapsed, double* dt_last) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    if (nsteps < 0) return fail(c, CFS_ERR_INVALID, "nsteps must be non-negative");
    if (c->next_stage != 0) return fail(c, CFS_ERR_STATE, "a step is in progress (stage sequence not at stage 0)");
    if (!(cfl > 0) && !(dt > 0)) return fail(c, CFS_ERR_INVALID, "give cfl > 0 or dt > 0");
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    if (c->cur != 0) {
        CFS_CUDA(c, cudaMemcpyAsync(c->S[0], c->S[c->cur], static_cast<size_t>(c->L.bytes()), cudaMemcpyDeviceToDevice, c->stream));
        c->cur = 0;
    }
    cfs::DevParams hp{};
    hp.use_cfl = cfl > 0 ? 1 : 0;
    hp.cfl = cfl;
    hp.dt_fixed = dt;
    hp.seed[0] = hp.seed[1] = c->steps_done;
    // first step's CFL maximum: carried from the previous advance's last stage
    // while the state is unchanged (so that K calls of one step take the steps
    // one call of K steps takes), else reduced now
    const bool carry = hp.use_cfl && c->wmax_carry;
    if (carry) hp.wmax[0] = c->wmax_bits;
    // (the previous advance ended with a stream synchronisation, so the pinned
    // slot is free)
    const cfs::DevParams* hp_src = &hp;
    if (c->hp_pin) {
        c->hp_pin[0] = hp;
        hp_src = c->hp_pin;
    }
    CFS_CUDA(c, cudaMemcpyAsync(c->P, hp_src, sizeof(hp), cudaMemcpyHostToDevice, c->stream));
    if (hp.use_cfl && !carry) {
        if (c->ib_n > 0) CFS_CUDA(c, cfs::launch_ib_fill(c->L.elem_bytes, ib_args(c, c->S[0]), c->stream));
        CFS_CUDA(c, cfs::launch_wmax(c->L.elem_bytes, c->S[0], c->L, c->has_types ? c->types_d : nullptr, c->cfg.gamma,
                                     c->dx, c->dy, reinterpret_cast<unsigned long long*>(c->P), c->stream));
    }
    const int S = stages_per_step(c->cfg.rk);
    auto enqueue_step = [&](int parity) -> int {
        int cur = 0, u0 = -1, u1 = -1;
        for (int s = 0; s < S; ++s) {
            const Roles r = roles_for(c, s, cur, u0, u1);
            const int rc = enqueue_stage(c, s, r, dt, true, parity, s == 0, s == S - 1);
            if (rc != CFS_OK) return rc;
            if (s == 0) u0 = r.u0;
            if (s == 1) u1 = r.u1;
            cur = r.out;
        }
        return CFS_OK;
    };
    // CUDA graphs of two steps (parities 0, 1) and of one step (parity 0),
    // captured at first use; every launch reads dt and the CFL slots from P
    auto capture = [&](int steps, cudaGraphExec_t* exec) -> int {
        cudaGraph_t g = nullptr;
        CFS_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        int rc = CFS_OK;
        for (int k = 0; k < steps && rc == CFS_OK; ++k) rc = enqueue_step(k);
        const cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
        if (rc != CFS_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ec != cudaSuccess) return fail(c, CFS_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(ec));
        const cudaError_t ei = cudaGraphInstantiate(exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            *exec = nullptr;
            return fail(c, CFS_ERR_CUDA, std::string("graph instantiation failed: ") + cudaGetErrorString(ei));
        }
        return CFS_OK;
    };
    if (nsteps >= 2 && !c->graph2)
        if (const int rc = capture(2, &c->graph2); rc != CFS_OK) return rc;
    if (nsteps % 2 == 1 && !c->graph1)
        if (const int rc = capture(1, &c->graph1); rc != CFS_OK) return rc;
    for (int k = 0; k + 1 < nsteps; k += 2) CFS_CUDA(c, cudaGraphLaunch(c->graph2, c->stream));
    if (nsteps % 2 == 1) CFS_CUDA(c, cudaGraphLaunch(c->graph1, c->stream));
    cfs::DevParams out{};
    CFS_CUDA(c, cudaMemcpyAsync(c->hp_pin ? c->hp_pin + 1 : &out, c->P, sizeof(out), cudaMemcpyDeviceToHost, c->stream));
    CFS_CUDA(c, cudaStreamSynchronize(c->stream));
    if (c->hp_pin) out = c->hp_pin[1];
    if (t_elapsed) *t_elapsed = out.t;
    if (dt_last) *dt_last = out.dt_last;
    c->steps_done += static_cast<unsigned int>(nsteps);
    if (const int rc = check_device_errors(c); rc != CFS_OK) return rc;
    if (nsteps > 0) c->wmax_carry = false;
    if (nsteps > 0 && (!(out.dt_last > 0) || !std::isfinite(out.dt_last)))
        return fail(c, CFS_ERR_NUMERIC, "time step became non-finite or non-positive");
    if (nsteps > 0 && hp.use_cfl) {
        // the last step (parity 1 after an even count, 0 after an odd one)
        // left the maximum of the final state in wmax[1 - parity]; it is
        // +infinity when a fluid cell of that state is non-finite
        c->wmax_bits = out.wmax[nsteps % 2 == 1 ? 1 : 0];
        c->wmax_carry = c->wmax_bits != 0;
        if (c->wmax_bits == 0x7ff0000000000000ull) return fail(c, CFS_ERR_NUMERIC, "a fluid cell became non-finite");
    }
    return CFS_OK;
}

// ---- device-ordered stepping of decomposed grids
int cfs_steps_begin(cfs_ctx* c, double cfl, double dt) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    if (c->in_steps) return fail(c, CFS_ERR_STATE, "cfs_steps_begin inside a run of steps");
    if (c->next_stage != 0) return fail(c, CFS_ERR_STATE, "a step is in progress (stage sequence not at stage 0)");
    if (!(cfl > 0) && !(dt > 0)) return fail(c, CFS_ERR_INVALID, "give cfl > 0 or dt > 0");
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    cfs::DevParams hp{};
    hp.use_cfl = cfl > 0 ? 1 : 0;
    hp.cfl = cfl;
    hp.dt_fixed = dt;
    hp.seed[0] = hp.seed[1] = c->steps_done;
    const bool carry = hp.use_cfl && c->wmax_carry;
    if (carry) hp.wmax[0] = c->wmax_bits;
    CFS_CUDA(c, cudaMemcpyAsync(c->P, &hp, sizeof(hp), cudaMemcpyHostToDevice, c->stream));
    if (hp.use_cfl && !carry) {
        if (c->ib_n > 0) CFS_CUDA(c, cfs::launch_ib_fill(c->L.elem_bytes, ib_args(c, c->S[c->cur]), c->stream));
        CFS_CUDA(c, cfs::launch_wmax(c->L.elem_bytes, c->S[c->cur], c->L, c->has_types ? c->types_d : nullptr, c->cfg.gamma,
                                     c->dx, c->dy, reinterpret_cast<unsigned long long*>(c->P), c->stream));
    }
    c->wmax_carry = false;
    c->in_steps = true;
    c->steps_cfl = hp.use_cfl != 0;
    c->steps_parity = 0;
    c->steps_part = CFS_PART_ALL;
    return CFS_OK;
}

int cfs_steps_stage(cfs_ctx* c, int part) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    if (!c->in_steps) return fail(c, CFS_ERR_STATE, "cfs_steps_stage outside cfs_steps_begin / cfs_steps_end");
    if (part != CFS_PART_ALL && part != CFS_PART_INTERIOR && part != CFS_PART_EDGES)
        return fail(c, CFS_ERR_INVALID, "unknown stage part");
    const bool split = part != CFS_PART_ALL;
    if (split && (c->prec == cfs::kF64Exact || c->rv || c->ib_n > 0 || c->cfg.nx < 2 * cfs::kGhost))
        return fail(c, CFS_ERR_INVALID, "interior/edge parts need a throughput form, no viscous terms, no immersed "
                                        "boundary and nx >= 6");
    if (part == CFS_PART_EDGES && c->steps_part != CFS_PART_INTERIOR)
        return fail(c, CFS_ERR_STATE, "the edge part follows the interior part of the same stage");
    if (part != CFS_PART_EDGES && c->steps_part == CFS_PART_INTERIOR)
        return fail(c, CFS_ERR_STATE, "the interior part of this stage awaits its edge part");
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    const int S = stages_per_step(c->cfg.rk);
    const int stage = c->next_stage;
    const Roles r = roles_for(c, stage, c->cur, c->u0_idx, c->u1_idx);
    // the step's first-stage bookkeeping (t, dt, CFL slot reset) runs in
    // exactly one launch: the full stage or its interior part; the
    // immersed-ghost fill and viscous RHS run with the full stage only (the
    // split parts refuse both above)
    const bool first = stage == 0 && part != CFS_PART_EDGES;
    const bool last = stage == S - 1;
    if (part == CFS_PART_ALL) {
        const int rc = enqueue_stage(c, stage, r, 0.0, true, c->steps_parity, first, last, 0, 0, true);
        if (rc != CFS_OK) return rc;
    } else if (part == CFS_PART_INTERIOR) {
        const int rc = enqueue_stage(c, stage, r, 0.0, true, c->steps_parity, first, last, cfs::kGhost,
                                     c->cfg.nx - cfs::kGhost, false);
        if (rc != CFS_OK) return rc;
    } else {
        int rc = enqueue_stage(c, stage, r, 0.0, true, c->steps_parity, first, last, 0, cfs::kGhost, false);
        if (rc == CFS_OK)
            rc = enqueue_stage(c, stage, r, 0.0, true, c->steps_parity, first, last, c->cfg.nx - cfs::kGhost,
                               c->cfg.nx, false);
        if (rc != CFS_OK) return rc;
    }
    c->steps_part = part;
    if (part == CFS_PART_INTERIOR) return CFS_OK;
    if (stage == 0) c->u0_idx = r.u0;
    if (stage == 1) c->u1_idx = r.u1;
    c->cur = r.out;
    c->next_stage = (stage + 1) % S;
    if (c->next_stage == 0) {
        ++c->steps_done;
        c->steps_parity ^= 1;
    }
    return CFS_OK;
}

int cfs_cfl_export(cfs_ctx* c, void* dev_dst) {
    if (!c || !dev_dst) return fail(c, CFS_ERR_INVALID, "null argument");
    if (!c->in_steps || c->next_stage != 0) return fail(c, CFS_ERR_STATE, "the CFL slot is exchanged between steps");
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    CFS_CUDA(c, cudaMemcpyAsync(dev_dst, &c->P->wmax[c->steps_parity], sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                c->stream));
    return CFS_OK;
}

int cfs_cfl_import(cfs_ctx* c, const void* dev_src) {
    if (!c || !dev_src) return fail(c, CFS_ERR_INVALID, "null argument");
    if (!c->in_steps || c->next_stage != 0) return fail(c, CFS_ERR_STATE, "the CFL slot is exchanged between steps");
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    CFS_CUDA(c, cudaMemcpyAsync(&c->P->wmax[c->steps_parity], dev_src, sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                c->stream));
    return CFS_OK;
}

int cfs_steps_end(cfs_ctx* c, double* t_elapsed, double* dt_last) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    if (!c->in_steps) return fail(c, CFS_ERR_STATE, "cfs_steps_end without cfs_steps_begin");
    if (c->next_stage != 0) return fail(c, CFS_ERR_STATE, "a step is in progress (stage sequence not at stage 0)");
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    cfs::DevParams out{};
    CFS_CUDA(c, cudaMemcpyAsync(&out, c->P, sizeof(out), cudaMemcpyDeviceToHost, c->stream));
    CFS_CUDA(c, cudaStreamSynchronize(c->stream));
    c->in_steps = false;
    if (const int rc = check_device_errors(c); rc != CFS_OK) return rc;
    if (t_elapsed) *t_elapsed = out.t;
    if (dt_last) *dt_last = out.dt_last;
    if (out.t > 0 && (!(out.dt_last > 0) || !std::isfinite(out.dt_last)))
        return fail(c, CFS_ERR_NUMERIC, "time step became non-finite or non-positive");
    if (c->steps_cfl && out.t > 0) {
        c->wmax_bits = out.wmax[c->steps_parity];
        c->wmax_carry = c->wmax_bits != 0;
        if (c->wmax_bits == 0x7ff0000000000000ull) return fail(c, CFS_ERR_NUMERIC, "a fluid cell became non-finite");
    }
    return CFS_OK;
}

int cfs_synchronize(cfs_ctx* c) {
    if (!c) return fail(c, CFS_ERR_INVALID, "null context");
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    CFS_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_device_errors(c);
}

void* cfs_get_stream(cfs_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

int cfs_halo_bytes(cfs_ctx* c, long long* bytes) {
    if (!c || !bytes) return fail(c, CFS_ERR_INVALID, "null argument");
    *bytes = cfs::kGhost * c->L.row_bytes();
    return CFS_OK;
}

// Rows hold whole cells and are contiguous in the padded layout: one side's 3
// rows are one block of 3 * row_bytes, so a message is one plain copy.
int cfs_halo_pack(cfs_ctx* c, int side, void* dst) {
    if (!c || !dst || (side != 0 && side != 1)) return fail(c, CFS_ERR_INVALID, "bad halo pack arguments");
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    const size_t row_bytes = static_cast<size_t>(c->L.row_bytes());
    const int first = side == 0 ? 0 : c->cfg.nx - cfs::kGhost;
    const char* src = static_cast<const char*>(c->S[c->cur]) + static_cast<size_t>(first + cfs::kGhost) * row_bytes;
    CFS_CUDA(c, cudaMemcpyAsync(dst, src, cfs::kGhost * row_bytes, cudaMemcpyDeviceToDevice, c->stream));
    return CFS_OK;
}

int cfs_halo_unpack(cfs_ctx* c, int side, const void* src) {
    if (!c || !src || (side != 0 && side != 1)) return fail(c, CFS_ERR_INVALID, "bad halo unpack arguments");
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    c->wmax_carry = false;
    const size_t row_bytes = static_cast<size_t>(c->L.row_bytes());
    const int first = side == 0 ? -cfs::kGhost : c->cfg.nx;
    char* dst = static_cast<char*>(c->S[c->cur]) + static_cast<size_t>(first + cfs::kGhost) * row_bytes;
    CFS_CUDA(c, cudaMemcpyAsync(dst, src, cfs::kGhost * row_bytes, cudaMemcpyDeviceToDevice, c->stream));
    return CFS_OK;
}

int cfs_conserved_totals(cfs_ctx* c, double totals[4]) {
    if (!c || !totals) return fail(c, CFS_ERR_INVALID, "null argument");
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    CFS_CUDA(c, cfs::launch_totals(c->L.elem_bytes, c->S[c->cur], c->L, c->has_types ? c->types_d : nullptr, c->sums,
                                   c->totals, c->stream));
    CFS_CUDA(c, cudaMemcpyAsync(totals, c->totals, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CFS_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int v = 0; v < 4; ++v) totals[v] *= c->dx * c->dy;
    return CFS_OK;
}

int cfs_weno5_faces(cfs_ctx* c, int n, const double* st, double* left, double* right) {
    if (!c || n < 0 || (n > 0 && (!st || !left || !right))) return fail(c, CFS_ERR_INVALID, "bad argument");
    if (n == 0) return CFS_OK;
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    DeviceScratch d_st, d_l, d_r;
    cudaError_t e = d_st.alloc(sizeof(double) * 24 * n);
    if (e == cudaSuccess) e = d_l.alloc(sizeof(double) * 5 * n);
    if (e == cudaSuccess) e = d_r.alloc(sizeof(double) * 5 * n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_st.p, st, sizeof(double) * 24 * n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cfs::launch_weno_faces(c->prec, n, d_st.get<double>(), d_l.get<double>(), d_r.get<double>(), c->cfg.gamma,
                                   c->cfg.weno_eps, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(left, d_l.p, sizeof(double) * 5 * n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(right, d_r.p, sizeof(double) * 5 * n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return fail(c, CFS_ERR_CUDA, std::string("weno5 faces: ") + cudaGetErrorString(e));
    return CFS_OK;
}

int cfs_hll_faces(cfs_ctx* c, int n, int dir, const double* L, const double* R, double* F) {
    if (!c || n < 0 || (dir != 0 && dir != 1) || (n > 0 && (!L || !R || !F))) return fail(c, CFS_ERR_INVALID, "bad argument");
    if (n == 0) return CFS_OK;
    CFS_CUDA(c, cudaSetDevice(c->cfg.device));
    DeviceScratch d_l, d_r, d_f;
    cudaError_t e = d_l.alloc(sizeof(double) * 4 * n);
    if (e == cudaSuccess) e = d_r.alloc(sizeof(double) * 4 * n);
    if (e == cudaSuccess) e = d_f.alloc(sizeof(double) * 4 * n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_l.p, L, sizeof(double) * 4 * n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_r.p, R, sizeof(double) * 4 * n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cfs::launch_hll_faces(c->prec, n, dir, d_l.get<double>(), d_r.get<double>(), d_f.get<double>(), c->cfg.gamma,
                                  c->cfg.hll, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(F, d_f.p, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return fail(c, CFS_ERR_CUDA, std::string("hll faces: ") + cudaGetErrorString(e));
    return CFS_OK;
}

}  // extern "C"
