/* cfs.h - C ABI of the B200 (sm_100a) compressible-flow stage engine.
 *
 * One context owns one device-resident Cartesian grid (nx by ny cells on
 * [0,lx] x [0,ly]) with three ghost layers per side, and runs the per-RK-stage
 * hot path of the reference solver (xinxiangsama/2d_Compressible_Flow_Solver)
 * as fused CUDA kernels: immersed-ghost fill, WENO5 reconstruction of the
 * conserved variables, HLL interface flux, flux difference, TVD Runge-Kutta
 * update of fluid cells, physical-boundary ghost refresh and the CFL step.
 *
 * Host arrays use the reference's cell order: U[v][i][j], v = (rho, rho u,
 * rho v, E), i = x index (outer), j = y index (inner), as cells[i][j]
 * (CartesianMesh.cpp:3-9) and the HDF5 datasets (Output.cpp:60).
 *
 * Every call returns CFS_OK (0) or a positive error code; the message of the
 * last failure of a context is cfs_last_error(ctx) (cfs_last_error(NULL) after
 * a failed cfs_create).  A failed call leaves no CUDA error pending on the
 * calling thread (a refused allocation does not fail the next call's launch
 * checks, on this context or another).  Calls on one context come from one
 * host thread; all work of a context is ordered on the context's CUDA stream.
 * There is no CPU fallback: without a usable CUDA device cfs_create fails with
 * CFS_ERR_CUDA.
 */
#ifndef CFS_H
#define CFS_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CFS_ABI_VERSION 3

enum cfs_status {
    CFS_OK = 0,
    CFS_ERR_INVALID = 1,    /* bad argument or configuration */
    CFS_ERR_CUDA = 2,       /* a CUDA call failed (message has the CUDA error) */
    CFS_ERR_NOMEM = 3,      /* device or host allocation failed */
    CFS_ERR_STATE = 4,      /* call not valid in the context's current state */
    CFS_ERR_NUMERIC = 5     /* the CFL reduction met a non-finite fluid cell (a blow-up), or
                               gave a non-positive dt */
};

enum cfs_precision {
    CFS_FP64 = 0,        /* FP64 state and arithmetic, FMA-contracted kernels */
    CFS_FP32_MIXED = 1,  /* FP32 state/WENO/HLL; FP64 p and c where kinetic energy
                            exceeds 90% of E, FP64 dt and conservation sums */
    CFS_FP64_EXACT = 2   /* FP64 in the reference's operation order, no FMA:
                            bit-identical to the reference built without fast-math */
};

enum cfs_rk {
    CFS_RK_TVD2 = 0,            /* TVD2rdRK (TVD2rdRK.cpp:3-31), the driver's choice (Run.cpp:47) */
    CFS_RK_TVD3_REFERENCE = 1,  /* TVD3rdRK as written (TVD3rdRK.cpp:3-48): stage 3 uses U1 */
    CFS_RK_SSP3 = 2             /* Shu-Osher SSP-RK3 (no reference counterpart) */
};

enum cfs_hll {
    CFS_HLL_REFERENCE = 0,  /* RiemmanSolverHLL::Solver (RiemmanSolverHLL.cpp:5-75), wave bounds as written */
    CFS_HLL_DAVIS = 1       /* Davis bounds min/max(u_L -+ a_L, u_R -+ a_R) (no reference counterpart) */
};

enum cfs_bc {
    CFS_BC_NEUMANN = 0,    /* NeummanBoundary (NeummanBoundary.cpp:31-45): ghost = adjacent cell */
    CFS_BC_DIRICHLET = 1,  /* DirichletBoundary (DirichletBoundary.cpp:32-46): fixed state */
    CFS_BC_PERIODIC = 2,   /* no reference counterpart */
    CFS_BC_HALO = 3        /* left/right only: ghost rows filled by the caller from a neighbouring
                              subdomain (cfs_halo_unpack), as CartesianParallel::exchangedata fills
                              the process-boundary ghost cells (CartesianParallel.cpp:172-427) */
};

enum cfs_cell_type { CFS_CELL_FLUID = 0, CFS_CELL_SOLID = 1, CFS_CELL_IMMERSED_GHOST = 2 };

enum cfs_ib_mode {
    CFS_IB_REFERENCE = 0,      /* ImagePoint::InterpolatePhase (ImagePoint.cpp:20-82): LDLT of the
                                  donor matrix's lower triangle, both momenta negated (Cell.cpp:172-181) */
    CFS_IB_BILINEAR_SLIP = 1   /* bilinear weights over the 2 x 2 cell block around the image point
                                  (fluid cells only, renormalised; inverse-distance weights over the
                                  given donors when that block has no fluid weight), only the
                                  wall-normal momentum reflected (slip wall) */
};

enum cfs_viscous { CFS_VISCOUS_OFF = 0, CFS_VISCOUS_NS = 1 };

/* Face-state positivity fallbacks of the throughput forms (no reference
 * counterpart: the reference's WENO5-on-conserved + HLL scheme has none and
 * reaches negative pressure on strong inflow past a body).  FP64_EXACT accepts
 * CFS_POSITIVITY_OFF only. */
enum cfs_positivity {
    CFS_POSITIVITY_OFF = 0,   /* reconstructed states used as they come (the reference) */
    CFS_POSITIVITY_FACE = 1,  /* a face state with rho <= 0 or p <= 0 (or NaN) is replaced by the
                                 value of the cell next to the face on its side (first order) */
    CFS_POSITIVITY_BODY = 2,  /* FACE, and both states of every face whose 6-cell stencil holds an
                                 immersed-ghost or solid cell are first order */
    CFS_POSITIVITY_FLOOR = 3  /* BODY, and floors on every fluid cell's new state: rho <= 1e-6 (or a
                                 NaN) gives the floor state at rest (rho = p = 1e-6, no momentum);
                                 p <= 1e-6 raises E so that p = 1e-6, momentum kept.  Not
                                 conservative where it acts (near-vacuum cells) */
};

/* Rounding of the FP32 state storage of CFS_FP32_MIXED (no reference
 * counterpart; the FP64 forms round to nearest).  cfs_config_default selects
 * CFS_ROUND_STOCHASTIC_ALL. */
enum cfs_rounding {
    CFS_ROUND_STOCHASTIC = 0,  /* the state that ends each RK step is rounded to one of its two
                                  neighbouring floats with probability by nearness (random bits
                                  hashed from cell and step): an unbiased error that does not build
                                  up; intermediate stage states round to nearest */
    CFS_ROUND_NEAREST = 1,     /* FP32 FMA update, round to nearest */
    CFS_ROUND_STOCHASTIC_ALL = 2 /* as CFS_ROUND_STOCHASTIC in every stage, intermediate ones included:
                                    rounding an intermediate stage to nearest leaves a small mass bias
                                    per step (its increments lie on a coarse lattice of the stored
                                    grid); stochastically, the mass error stays a random walk */
};

typedef struct cfs_config {
    int nx, ny;              /* cells; CartesianMesh::setnumberCellsX/YGlobal (Run.cpp:17-18) */
    double lx, ly;           /* domain lengths; setGlobalLengthX/Y (Run.cpp:19-20) */
    double gamma;            /* Gamma, param.h:5 (1.4) */
    double weno_eps;         /* Weno5th.cpp:5 (1e-2) */
    int precision;           /* enum cfs_precision */
    int rk;                  /* enum cfs_rk */
    int hll;                 /* enum cfs_hll */
    int bc[4];               /* enum cfs_bc for left, right, bottom, top (Cylinder.cpp:19-40 order) */
    double bc_prim[4][4];    /* Dirichlet (rho, u, v, p) per side, applied as Cylinder.cpp:22-32 */
    int viscous;             /* enum cfs_viscous */
    double mu, prandtl, mach;/* Navier-Stokes constants (constant viscosity, T = gamma Ma^2 p / rho) */
    int keep_rhs;            /* 1: keep the last stage's RHS for cfs_get_rhs (Cell::comRHS m_flux) */
    int device;              /* CUDA device ordinal */
    int variant;             /* stage-kernel variant of the throughput forms (tile rows x warps x
                                occupancy target, see cfs_variant_info); 0 = the tuned default */
    int positivity;          /* enum cfs_positivity */
    int rounding;            /* enum cfs_rounding (CFS_FP32_MIXED) */
    int march_rows;          /* throughput forms: rows of one warp's work item in the row march;
                                0 = chosen at each launch so the blocks fill whole waves of the
                                GPU's resident blocks (the tuned default), > 0 = fixed (<= 4096) */
} cfs_config;

typedef struct cfs_ctx cfs_ctx;

/* Number of stage-kernel variants of the throughput forms, and the shape of
 * variant v (1-based): rows marched per warp, warps per block, minimum resident
 * blocks per SM requested from the compiler, and the row march's load schedule
 * (0: loads at their use; 1: issued early in each row's iteration; 2: two rows
 * ahead; 3: rows staged in shared memory by asynchronous copies).
 * Returns CFS_ERR_INVALID for an unknown v. */
int cfs_variant_count(void);
int cfs_variant_info(int v, int* rows, int* warps, int* min_blocks, int* prefetch);

/* Fills a config with the reference's defaults: gamma 1.4, eps 1e-2, FP64,
 * TVD3 as written, reference HLL, Neumann sides, inviscid. */
void cfs_config_default(cfs_config* cfg);

/* Creates a context and allocates the device grid.
 * Replaces Run::initialize's mesh/plugin set-up (Run.cpp:10-90): the plugin
 * selection point Run.cpp:41-48 maps to cfg->{rk,hll,weno_eps,bc}. */
int cfs_create(const cfs_config* cfg, cfs_ctx** out);
int cfs_destroy(cfs_ctx* ctx);
const char* cfs_last_error(const cfs_ctx* ctx);
int cfs_abi_version(void);

/* Conserved state in and out (host U[4][nx][ny]).
 * set: Initialcondition::fillIn (Initialcondition.h:11) over all cells, then
 *      the physical-boundary ghost fill (CartesianMesh::ApplyBoundaryCondition,
 *      CartesianMesh.cpp:280-305, called at Run.cpp:128).
 * get: the cell phases Output::WriteToHDF5 reads (Output.cpp:58-75).
 * U may be pinned or pageable host memory.  A pageable array of 32 MB or more
 * is copied in 16 chunks through a pinned staging buffer of the state's size,
 * allocated by the first such call and kept until cfs_destroy, with host
 * threads (up to 16) moving each chunk while the DMA engine moves the one
 * before (after) it; the bytes are the same as a direct copy's. */
int cfs_set_state(cfs_ctx* ctx, const double* U);
int cfs_get_state(cfs_ctx* ctx, double* U);

/* RHS R = -(dF/dx + dG/dy) of the last stage (Cell::comRHS, Cell.cpp:110-162,
 * stored in Cell::m_flux and written as FluxRho/FluxMu/FluxMv/FluxEnergy by
 * Output.cpp:38-41).  Requires cfg.keep_rhs = 1.  Host R[4][nx][ny]. */
int cfs_get_rhs(cfs_ctx* ctx, double* R);

/* Cell types (enum cfs_cell_type), host types[nx][ny]; default all fluid.
 * Only fluid cells are advanced (Run.cpp:193-200). */
int cfs_set_cell_types(cfs_ctx* ctx, const uint8_t* types);

/* Immersed-ghost list: n cells (i*ny + j), 4 fluid donors each (i*ny + j, in
 * the reference's nearest-first order), the image point (x, y) of each, and
 * for CFS_IB_BILINEAR_SLIP the unit wall normal.  Replaces the ImagePoint
 * objects Circle::SetImagepoint builds (Circle.cpp:105-138).  Set the cell
 * types first: the slip form picks its donors among fluid cells. */
int cfs_set_ib(cfs_ctx* ctx, int mode, int n, const int32_t* cell, const int32_t* donor4,
               const double* image_xy, const double* normal_xy);

/* Circle immersed boundary built on the host exactly as the reference does it:
 * Circle::Initialize (Circle.cpp:12-41) with npoints vertices,
 * DistinguishWallandFluid (:43-51), SetGhostcell(cells, 3) (:53-103),
 * SetImagepoint (:105-138) and FindNearest4FluidCellsIndexed (:160-215);
 * then cfs_set_cell_types + cfs_set_ib.  Fails with CFS_ERR_INVALID when an
 * immersed-ghost cell finds fewer than 4 fluid donors (the reference then reads
 * past its donor list, ImagePoint.cpp:25). */
int cfs_ib_build_circle(cfs_ctx* ctx, double radius, double cx, double cy, int npoints, int mode);

/* The same circle set-up as cfs_ib_build_circle, host only (no context, no
 * device): writes types[nx][ny] and, for the first min(n, max_n) immersed-ghost
 * cells (i outer, j inner order), cell index, 4 donors, image point and unit
 * normal (from the ghost centre to its image point).  *n receives the total. */
int cfs_circle_setup(int nx, int ny, double lx, double ly, double radius, double cx, double cy, int npoints,
                     uint8_t* types, int max_n, int* n, int32_t* cell, int32_t* donor4, double* image_xy,
                     double* normal_xy);

/* The same circle set-up with its per-cell work on the device (no counterpart
 * in the reference, whose set-up is host code): classification, ghost marking
 * and image points run as kernels built without FMA contraction, so types,
 * ghost list, image points and normals are bit for bit those of the host
 * set-up; the donors are chosen on the host from the read-back types (the
 * reference's sort and tie order).  cfs_ib_build_circle_device uses the
 * context's device and stream; cfs_circle_setup_device the given device and
 * its default stream, with cfs_circle_setup's outputs.  Errors as
 * cfs_ib_build_circle, plus CFS_ERR_CUDA for a device failure. */
int cfs_ib_build_circle_device(cfs_ctx* ctx, double radius, double cx, double cy, int npoints, int mode);
int cfs_circle_setup_device(int device, int nx, int ny, double lx, double ly, double radius, double cx, double cy,
                            int npoints, uint8_t* types, int max_n, int* n, int32_t* cell, int32_t* donor4,
                            double* image_xy, double* normal_xy);

/* A closed polygon body (no counterpart in the reference, whose only
 * ImmersedBoundary shape is the circle): npoints vertices xy[2*npoints] in
 * order, either orientation, non-convex allowed.  A cell is solid when its
 * centre is inside (even-odd rule); ghost cells are marked as SetGhostcell
 * marks them (Circle.cpp:53-103); a ghost's image point mirrors its centre in
 * the nearest point of the polygon's boundary; donors as for the circle
 * (FindNearest4FluidCellsIndexed, Circle.cpp:160-215).  cfs_ib_build_polygon
 * installs it in a context (types + cfs_set_ib with `mode`);
 * cfs_polygon_setup returns the lists on the host as cfs_circle_setup does.
 * CFS_ERR_INVALID for fewer than 3 vertices, non-finite vertices or a ghost
 * with fewer than 4 fluid donors. */
int cfs_ib_build_polygon(cfs_ctx* ctx, int npoints, const double* xy, int mode);
int cfs_polygon_setup(int nx, int ny, double lx, double ly, int npoints, const double* xy, uint8_t* types, int max_n,
                      int* n, int32_t* cell, int32_t* donor4, double* image_xy, double* normal_xy);

/* Read-back of the immersed-boundary set-up: types[nx][ny], and for the first
 * min(n, max_n) immersed-ghost cells (i outer, j inner order) their cell
 * index, donors and image point.  *n receives the total count. */
int cfs_get_ib(cfs_ctx* ctx, uint8_t* types, int max_n, int* n, int32_t* cell, int32_t* donor4, double* image_xy);

/* Fills immersed-ghost cells from their image points now
 * (Cell::comImmersedGhostPhase over IG cells, Run.cpp:107-113,156-162). */
int cfs_ib_fill(cfs_ctx* ctx);

/* CFL step on the current state: dt = cfl / max over fluid cells of
 * (|u|+a)/dx + (|v|+a)/dy.  No reference counterpart (the reference fixes dt,
 * param.h:20, set by Explicit::setTimeStep at Run.cpp:95).  Warp-shuffle max
 * reduction; the max is exact, so dt is the same on every launch.  A fluid
 * cell whose wave-speed sum is not finite (NaN from a negative pressure or
 * density) makes the maximum +infinity: CFS_ERR_NUMERIC. */
int cfs_compute_dt(cfs_ctx* ctx, double cfl, double* dt);

/* One iteration of Run::solver's loop (Run.cpp:153-203) with loop counter
 * `counter` (1, 2, 3, ...), whose stage is derived as TVD2rdRK.cpp:11 /
 * TVD3rdRK.cpp:15 do: immersed-ghost fill, reconstruction + HLL on every face
 * (Interpolation::comLeftPhase/comRightPhase, Interpolation.h:14-15;
 * RiemmanSolver::Solver, RiemmanSolver.h:12), Explicit::advance of every fluid
 * cell (Explicit.h:10) with time step dt, physical-boundary ghost refresh
 * (Boundary::EnforceBoundary, Boundary.h:11). */
int cfs_stage(cfs_ctx* ctx, int counter, double dt);

/* One full RK step (2 or 3 cfs_stage calls) with time step dt. */
int cfs_step(cfs_ctx* ctx, double dt);

/* nsteps full RK steps, the stage launches replayed from a CUDA graph.
 * cfl > 0: dt of every step comes from the CFL reduction of the step's
 * initial state, computed on the device inside the previous step's last stage
 * (no host round trip) -- also across calls, while nothing but cfs_advance has
 * touched the state since (so K calls of one step take the steps one call of
 * K steps takes); otherwise the first step's reduction runs at the call's
 * start.  cfl <= 0: fixed dt.  *t_elapsed (optional) receives the simulated
 * time advanced, *dt_last the last dt.  With cfl > 0, a fluid cell that turns
 * non-finite in any step makes every later dt 0, and the call returns
 * CFS_ERR_NUMERIC (also when it happens in the last step: the final stage's
 * CFL maximum is then +infinity). */
int cfs_advance(cfs_ctx* ctx, int nsteps, double cfl, double dt, double* t_elapsed, double* dt_last);

/* Halo exchange of a slab decomposition along x (the reference's process
 * boundaries, CartesianParallel.cpp:62-148).  side 0 = left (low x), 1 = right.
 * cfs_halo_bytes: size of one side's message (3 rows x 4 variables, ghost
 * columns included, the state's storage type).  pack: the 3 interior rows next
 * to `side` of the current state -> dev_dst (device memory).  unpack: dev_src ->
 * the 3 ghost rows of `side`.  Both are ordered on the context's stream.
 * Messages carry stored values: in CFS_FP32_MIXED every context of one
 * decomposed grid must store against the same offsets (cfs_set_storage_offsets). */
int cfs_halo_bytes(cfs_ctx* ctx, long long* bytes);
int cfs_halo_pack(cfs_ctx* ctx, int side, void* dev_dst);
int cfs_halo_unpack(cfs_ctx* ctx, int side, const void* dev_src);

/* CFS_FP32_MIXED stores each variable as (value - offset) in FP32.  By default
 * cfs_set_state takes the offsets from the state (each variable's mean, rounded
 * to FP32).  This call fixes them (FP32-rounded) for the following
 * cfs_set_state calls; off = NULL returns to the default.  No effect on the
 * FP64 forms.  (No reference counterpart.) */
int cfs_set_storage_offsets(cfs_ctx* ctx, const double* off4);

/* Run counters, for resuming a run bit for bit from a snapshot in a new
 * context (no reference counterpart: the reference writes snapshots but never
 * reads them back, Output.cpp:20).
 * get: *step = completed RK steps (the counter the FP32-mixed stochastic
 *   rounding hashes with each cell); *cfl_max = the CFL maximum of the current
 *   state that the next cfs_advance will use (left by the last advance's final
 *   stage), 0 when none is carried; off4[4] = the FP32-mixed storage offsets
 *   (cfs_set_storage_offsets; 0 in the FP64 forms).  Any pointer may be NULL.
 * set: after cfs_set_state, installs step and cfl_max (0: the next
 *   cfs_advance reduces the maximum afresh).  CFS_ERR_STATE inside a step.
 * Resume = cfs_set_storage_offsets(off4), cfs_set_state(U), cfs_set_step(step,
 * cfl_max): the following steps are then the bits the uninterrupted run takes. */
int cfs_get_step(cfs_ctx* ctx, unsigned int* step, double* cfl_max, double* off4);
int cfs_set_step(cfs_ctx* ctx, unsigned int step, double cfl_max);

/* Device-ordered stepping, for a grid decomposed over several contexts (the
 * reference's MPI decomposition, CartesianParallel.cpp:3-60, whose halo
 * exchange :172-427 posts Irecv/Isend per stage and waits).  Nothing here
 * waits on the host between begin and end: dt comes from the device (CFL
 * maximum fused into each step's last stage, as cfs_advance), and every call
 * only enqueues work on the context's stream, so the caller orders its halo
 * exchange (cfs_halo_pack/unpack and its own transfers) and the CFL
 * reduction across contexts on that stream, or on streams it joins to it.
 *   cfs_steps_begin: starts a run of steps with cfl > 0 (device CFL dt) or a
 *     fixed dt; reduces the first step's CFL maximum unless one is carried.
 *   cfs_steps_stage: enqueues the next stage of the running step (the stage
 *     sequence of cfs_stage), or one part of it: CFS_PART_INTERIOR updates
 *     rows 3 .. nx-4, which read no ghost row, so it may run while the ghost
 *     rows of its input are still being exchanged; CFS_PART_EDGES then updates
 *     rows 0..2 and nx-3..nx-1.  The parts need a throughput form, no viscous
 *     terms, no immersed boundary and nx >= 6.
 *   cfs_cfl_export / cfs_cfl_import: between steps, copy the CFL maximum the
 *     next step will use (8 bytes, FP64 bits of a non-negative value, so an
 *     integer MAX orders it) to / from caller device memory, ordered on the
 *     stream: export, a MAX all-reduce over the contexts, import.
 *   cfs_steps_end: waits for the stream; *t_elapsed and *dt_last as
 *     cfs_advance; CFS_ERR_NUMERIC on a non-finite step or fluid cell. */
enum cfs_stage_part { CFS_PART_ALL = 0, CFS_PART_INTERIOR = 1, CFS_PART_EDGES = 2 };
int cfs_steps_begin(cfs_ctx* ctx, double cfl, double dt);
int cfs_steps_stage(cfs_ctx* ctx, int part);
int cfs_cfl_export(cfs_ctx* ctx, void* dev_dst);
int cfs_cfl_import(cfs_ctx* ctx, const void* dev_src);
int cfs_steps_end(cfs_ctx* ctx, double* t_elapsed, double* dt_last);

/* Waits for the context's stream. */
int cfs_synchronize(cfs_ctx* ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work (events, copies, collectives) against the engine's. */
void* cfs_get_stream(cfs_ctx* ctx);

/* Sums over fluid cells of rho, rho u, rho v and E times the cell area,
 * accumulated in FP64 (conservation check). */
int cfs_conserved_totals(cfs_ctx* ctx, double totals[4]);

/* ---- Batched cases -------------------------------------------------------
 * Hundreds of independent grids of uneven size advanced together: every stage
 * of every case runs in ONE persistent launch whose warps pull work items
 * (case, 30-column segment, row chunk) from a device counter, largest cases first;
 * each case keeps its own CFL time step, computed on the device; whole steps
 * are replayed from a CUDA graph.  Throughput forms only (CFS_FP32_MIXED,
 * CFS_FP64).  No reference counterpart (the reference runs one grid). */
typedef struct cfs_case {
    int nx, ny;
    double lx, ly;
    int bc[4];
    double bc_prim[4][4];
    int circle;              /* 1: circle immersed boundary (cfs_ib_build_circle) */
    double radius, cx, cy;
    int npoints;
    int ib_mode;             /* enum cfs_ib_mode */
    int rows;                /* row chunk of a work item (0: the default, 64 rows) */
    int edge_code;           /* 1: run this case with the row march's edge code even where it
                                needs none (no physical side, no body): its work items join the
                                launch of the cases that need it, one launch fewer per stage when
                                it is the only case without; 0: the code path the case needs */
} cfs_case;

typedef struct cfs_batch cfs_batch;

/* common supplies precision, rk, hll, gamma, weno_eps, positivity, rounding and device. */
int cfs_batch_create(const cfs_config* common, int ncases, const cfs_case* cases, cfs_batch** out);
int cfs_batch_destroy(cfs_batch* b);
const char* cfs_batch_last_error(const cfs_batch* b);
int cfs_batch_set_state(cfs_batch* b, int c, const double* U);
int cfs_batch_get_state(cfs_batch* b, int c, double* U);
/* nsteps RK steps of every case with per-case CFL dt (cfl > 0) or a common
 * fixed dt; t (optional, [ncases]) receives each case's simulated time.
 * With cfl > 0, a fluid cell of some case that turns non-finite gives
 * CFS_ERR_NUMERIC (its CFL maximum becomes +infinity). */
int cfs_batch_advance(cfs_batch* b, int nsteps, double cfl, double dt, double* t);
/* nsteps RK steps with a fixed dt per case (dt_case[ncases], finite and
 * positive): replays another run's time steps, e.g. an FP64 batch's CFL steps
 * on an FP32-mixed batch of the same cases.  t as cfs_batch_advance. */
int cfs_batch_advance_dt(cfs_batch* b, int nsteps, const double* dt_case, double* t);
/* Per case, the dt of the last step taken (dt[ncases]; 0 before any step). */
int cfs_batch_dt_last(const cfs_batch* b, double* dt);
/* The batch's CUDA stream (a cudaStream_t), for callers that time or order
 * their own work against it. */
void* cfs_batch_get_stream(cfs_batch* b);
/* Total cells of the batch and the number of work items of one stage launch. */
int cfs_batch_info(const cfs_batch* b, long long* cells, int* items);

/* CFL step of a caller-owned device state, for callers that cannot allocate
 * device memory (no counterpart in the reference).  For a state held by a
 * CFS_FP64 or CFS_FP64_EXACT context, the same dt, bit for bit, as
 * cfs_compute_dt on that context (a CFS_FP32_MIXED context reduces its
 * FP32-rounded, offset storage, so its dt can differ in the last bits); needs
 * no context and calls no cudaMalloc, cudaFree or allocating library routine.
 * U: device array U[4][nx][ny] (reference order, FP64); types: device uint8
 * [nx][ny] (0 = fluid) or NULL for all fluid; stream: a cudaStream_t or NULL;
 * *dt: host output.  Runs on the current device.
 * Scratch is a fixed static device array, so nx*ny is limited to 16,777,216
 * cells (4096 x 4096); larger grids are refused with CFS_ERR_INVALID.  The first
 * call on a device looks up that array's device address (cudaGetSymbolAddress).
 * Every call copies dt to the host (pageable memory) and waits for `stream`,
 * so no call may be made on a stream that is being captured into a CUDA graph.
 * All calls share the array: calls that overlap on the GPU (other streams,
 * other host threads) race and must be serialised by the caller.  A fluid cell
 * whose wave-speed sum is not finite gives CFS_ERR_NUMERIC, as in
 * cfs_compute_dt.  Errors: cfs_last_error(NULL). */
int cfs_compute_dt_static(const double* U, const uint8_t* types, int nx, int ny, double lx, double ly,
                          double gamma, double cfl, void* stream, double* dt);

/* Measured arithmetic peaks of a device's CUDA cores (a diagnostic with no
 * counterpart in the reference): FP32 FFMA, packed FP32 FFMA2 and FP64 DFMA
 * throughput in TFLOP/s (2 flops per fused multiply-add), from independent
 * multiply-add chains filling every SM, best of three timed launches.  The
 * stage kernels are bound by instruction issue and these pipes, so this is
 * the denominator of their floating-point roofline.  Takes a few ms and 2.4 MB
 * of device memory.  Errors: cfs_last_error(NULL). */
int cfs_fp_peaks(int device, double* fp32_tflops, double* fp32x2_tflops, double* fp64_tflops);

/* Unit-level entry points (device batch, host buffers), mirroring one plugin
 * call each, for parity tests:
 * cfs_weno5_faces: Weno5th::comLeftPhase + comRightPhase (Weno5th.cpp:57-81) on
 *   n six-cell stencils st[n][6][4] -> left[n][5], right[n][5] = (rho, mx, my, E, p).
 * cfs_hll_faces: EulerMod::comFlux + RiemmanSolverHLL::Solver
 *   (CellInterface.cpp:68-89) on n face states L[n][4], R[n][4] -> F[n][4].
 * Both use the context's precision, hll variant, gamma and eps. */
int cfs_weno5_faces(cfs_ctx* ctx, int n, const double* st, double* left, double* right);
int cfs_hll_faces(cfs_ctx* ctx, int n, int dir, const double* L, const double* R, double* F);

#ifdef __cplusplus
}
#endif
#endif /* CFS_H */
