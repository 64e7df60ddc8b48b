// Device grid layout and kernel argument blocks shared by the host code and the
// kernels.  Plain C++ (no CUDA syntax) so that g++-compiled host files can use it.
//
// State: cells interleaved, (nx + 6) rows of `pitch` cells, each cell the four
// conserved variables (rho, rho u, rho v, E) side by side -- one 16-byte
// vector per cell in FP32, two in FP64.  Row r = i + 3 holds x index i
// (i = -3 .. nx+2); cell j of a row (j = -3 .. ny+2) sits at column joff + j,
// where joff is one 128-byte block so that every interior row starts 128-byte
// aligned.  A stage reads and writes whole cells, so one vector access (or one
// TMA box per row of a tile) moves all four variables.  The three ghost
// layers per side are maintained by the kernels (Neumann copies, periodic
// wraps) or set once (Dirichlet states), so a stage kernel reads a tile plus
// its 3-cell halo with no boundary logic in the load path.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define CFS_HD __host__ __device__ __forceinline__
#else
#define CFS_HD inline
#endif

namespace cfs {

constexpr int kGhost = 3;
constexpr int kVars = 4;

enum BcKind : int { kNeumann = 0, kDirichlet = 1, kPeriodic = 2, kHalo = 3 };

struct Layout {
    int nx, ny;
    int pitch;           // cells per row
    int joff;            // column of j = 0
    long long cells;     // cells per state buffer ((nx + 6) * pitch)
    int elem_bytes;      // bytes per variable: 8 (FP64) or 4 (FP32)
    // FP32 storage keeps value - off[v] (off = an FP32 value near the variable's
    // mean), so the rounding step of the stored state scales with the variation
    // of the field rather than its magnitude.  Always 0 for FP64 storage.
    float off[4];

    static Layout make(int nx, int ny, int elem_bytes) {
        Layout L;
        L.nx = nx;
        L.ny = ny;
        L.elem_bytes = elem_bytes;
        const int blk = 128 / (elem_bytes * kVars);  // cells per 128-byte block
        L.joff = blk;
        const int need = L.joff + ny + kGhost;
        L.pitch = ((need + blk - 1) / blk) * blk;
        L.cells = static_cast<long long>(nx + 2 * kGhost) * L.pitch;
        for (int v = 0; v < 4; ++v) L.off[v] = 0.0f;
        return L;
    }
    // cell index of (i, j) and element index of variable v of a cell
    CFS_HD long long offset(int i, int j) const { return static_cast<long long>(i + kGhost) * pitch + joff + j; }
    CFS_HD static long long at(long long cell, int v) { return cell * kVars + v; }
    CFS_HD long long row_bytes() const { return static_cast<long long>(pitch) * kVars * elem_bytes; }
    long long bytes() const { return cells * kVars * elem_bytes; }
};

// Boundary kinds of the four sides (left, right, bottom, top) and the
// conserved ghost state of each Dirichlet side.
struct BcSides {
    int bc[4];
    double U[4][4];
};

// Device-resident step parameters used by graph-replayed steps.
struct DevParams {
    unsigned long long wmax[2];   // max wave-speed sums (FP64 bit patterns), ping-pong per step
    double dt_fixed;
    double cfl;
    double t;                     // simulated time advanced
    double dt_last;
    int use_cfl;
    int pad;
    unsigned int seed[2];         // stochastic-rounding step counter, ping-pong per step
};

struct StageArgs {
    const void* in;        // state differentiated this stage (tile + halo reads)
    const void* u0;        // RK stage-0 copy (pointwise reads), stage >= 1
    const void* u1;        // RK stage-1 copy, TVD3-as-written stage 2
    void* out;             // new state (interior + ghost copies)
    double* rhs;           // optional RHS, [4][nx][ny]
    const uint8_t* types;  // optional cell types [nx][ny]; null = all fluid
    Layout L;
    int bc[4];
    double gamma, eps, dx, dy;
    int stage, rk, hll;
    int viscous;
    double mu, prandtl, mach;
    double dt;             // used when P is null
    DevParams* P;          // graph mode: dt from P (fixed or CFL), t accounting
    int parity;            // graph mode: which wmax slot holds this step's max
    int last_stage;        // 1: accumulate the CFL max of the new state into P->wmax[1-parity]
    int first_stage;       // 1: reset P->wmax[1-parity], advance P->t
    const void* rv;        // optional viscous RHS (rho u, rho v, E) [3][nx][ny], storage type
    int variant;           // throughput-form kernel variant (1-based; 0 = default)
    int positivity;        // 0 off, 1 face-state fallback, 2 also first order near the body, 3 also floors
    const uint8_t* lowo;   // positivity 2: [nx+1][ny+1] face flags, bit 0 x-face (i-1/2, j),
                           // bit 1 y-face (i, j-1/2): stencil holds a non-fluid cell
    int rounding;          // FP32 storage: 0 stochastic, 1 to nearest
    unsigned int seed;     // stochastic-rounding step counter when P is null
    const uint8_t* cflags; // throughput forms: per-cell flag bytes (kCell* bits) of cells
                           // i = -1..nx, j = -1..ny, [nx+2][ny+2]; null = all fluid, no low-order faces
    void* bflux;           // throughput forms: fluxes through the physical boundary faces
                           // (bflux_side_offset), arithmetic type of the form
    int row_lo, row_hi;    // throughput forms: the launch updates cells of rows [row_lo, row_hi)
                           // (row_hi 0: up to nx); a decomposed grid updates its interior
                           // rows while the halo exchange is in flight, then its edge rows
    int rows;              // row march: rows of one warp's work item (0: the launcher chooses)
    unsigned int* err;     // device error flags (kErr* bits), set instead of waiting forever
    int has_tmaps;         // 1: tmap_in (and, stage >= 1, tmap_u0) hold encoded tensor maps
    // TMA load schedule: tensor maps (CUtensorMap) of the `in` and `u0` buffers,
    // box of 4 variables x 36 cells x 1 row.  Kernels that read them take the
    // arguments as a __grid_constant__ parameter, so the copies address the
    // maps in parameter space.
    alignas(64) unsigned char tmap_in[128];
    alignas(64) unsigned char tmap_u0[128];
};

// Bits of *StageArgs::err.
constexpr unsigned int kErrTmaTimeout = 1u;  // a TMA copy did not land within its bounded wait
constexpr unsigned int kErrTmaAlign = 2u;    // a TMA copy's shared-memory row was not 128-byte aligned (not issued)

// Rows [lo, hi) a stage launch updates.
CFS_HD int stage_row_lo(const StageArgs& a) { return a.row_lo; }
CFS_HD int stage_row_hi(const StageArgs& a) { return a.row_hi > 0 ? a.row_hi : a.L.nx; }

// Bits of StageArgs::cflags.  The x-faces of cell (i, j) are (i-1/2, j) (lo)
// and (i+1/2, j) (hi), its y-faces (i, j-1/2) and (i, j+1/2); a low-order face
// has a non-fluid cell in its reconstruction stencil (CFS_POSITIVITY_BODY).
constexpr uint8_t kCellSolid = 1;   // non-fluid cell: keeps its state
constexpr uint8_t kCellLowXlo = 2;
constexpr uint8_t kCellLowXhi = 4;
constexpr uint8_t kCellLowYlo = 8;
constexpr uint8_t kCellLowYhi = 16;

// Boundary-face flux layout (StageArgs::bflux): sides 0 (face i = 0) and 1
// (i = nx) hold [4][ny], sides 2 (j = 0) and 3 (j = ny) hold [4][nx].
CFS_HD long long bflux_side_offset(const Layout& L, int s) {
    return s == 0 ? 0 : s == 1 ? 4LL * L.ny : s == 2 ? 8LL * L.ny : 8LL * L.ny + 4LL * L.nx;
}
CFS_HD long long bflux_count(const Layout& L) { return 8LL * (L.nx + L.ny); }

// Sides whose faces take the reference's boundary stencil.
CFS_HD bool physical_side(const StageArgs& a, int s) { return a.bc[s] == kNeumann || a.bc[s] == kDirichlet; }

// Row-march instantiation features, chosen per launch:
constexpr int kFeatPos = 1;    // positivity fallbacks and floors (StageArgs::positivity != 0)
constexpr int kFeatExtra = 2;  // RHS copy (StageArgs::rhs) and viscous RHS (StageArgs::rv)
constexpr int kFeatEdge = 4;   // physical sides (boundary-face fluxes) or cell flags (StageArgs::cflags)
CFS_HD int march_features(const StageArgs& a) {
    bool edge = a.cflags != nullptr;
    for (int s = 0; s < 4; ++s) edge = edge || physical_side(a, s);
    return (a.positivity ? kFeatPos : 0) | ((a.rhs || a.rv) ? kFeatExtra : 0) | (edge ? kFeatEdge : 0);
}

// Viscous (Navier-Stokes) RHS of one state: (dFv/dx + dGv/dy) for the momentum
// and energy equations, written to rv[3][nx][ny].
struct ViscArgs {
    const void* in;
    void* rv;
    Layout L;
    double gamma, dx, dy, mu, kT, mach2;
    double inv_dx, inv_dy;  // 1/dx, 1/dy (formed once on the host: a thread here covers about one cell)
    // the FP32 form's constants, rounded once on the host: gamma - 1,
    // gamma Ma^2, mu, kT, 1/dx, 1/dy
    float gm1_f, cT_f, mu_f, kT_f, inv_dx_f, inv_dy_f;
};

struct IbArgs {
    void* U;               // state to fill in place
    Layout L;
    int n;
    int mode;              // 0 reference LDLT replay, 1 bilinear + slip
    const int* cell;       // [n] linear index i*ny + j
    const int* donor;      // [4n] linear index i*ny + j
    const double* image;   // [2n]
    const double* fac;     // [16n] reference: l10 l20 l21 l30 l31 l32 d0..d3 (10); bilinear: w0..w3 nx ny
    const int* perm;       // [4n] reference pivot order
};

}  // namespace cfs
