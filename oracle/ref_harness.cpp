// Test infrastructure (oracle only).  Drives the reference solver's OWN numerical
// classes -- compiled unmodified from the reference tree against the shims in
// oracle/shim -- the way Run::initialize / Run::solver do (Run.cpp:10-90,93-236),
// with the grid, boundary conditions, integrator, immersed circle and initial
// state taken from a config instead of literals.  Built by oracle/Makefile into
// oracle/_ref/ (never shipped, never linked by the product).
//
// Additions that are NOT in the reference and are marked as such:
//   * an optional CFL time step recomputed at the first stage of each RK step
//     (the reference keeps dt fixed, param.h:20, Run.cpp:95);
//   * read-out helpers (state, RHS, IB lists, unit-level WENO/HLL/viscous calls).
#include "meshes/CartesianMesh.h"
#include "parallel/CartesianParallel.h"
#include "model/EulerMod.h"
#include "interpolation/Weno5th.h"
#include "flux/RiemmanSolverHLL.h"
#include "timeadvance/TVD3rdRK.h"
#include "gradient/FourthOrderCS.h"
#include "object/Circle.h"
#include "initialcondition/Initialcondition.h"

#include <chrono>
#include <cmath>
#include <cstring>

#ifdef CFS_WITH_GPU_PLUGINS
#include "cfs_plugins.h"
#endif

// The four process globals the reference's mesh objects reach through `extern`
// (Run.cpp:5-8).
std::shared_ptr<Model> model;
std::shared_ptr<Interpolation> interpolation;
std::shared_ptr<RiemmanSolver> riemmansolver;
std::shared_ptr<ForthOrderCS> gradient;

extern "C" {
struct ref_config {
    int nx, ny;
    double lx, ly;
    int integrator;       // 2 = TVD2rdRK (Run.cpp:47), 3 = TVD3rdRK
    double dt;            // fixed time step (param.h:20 style)
    double cfl;           // > 0: harness recomputes dt at each step start (addition)
    int bc_type[4];       // left, right, bottom, top: 0 Neumann, 1 Dirichlet
    double bc_prim[4][4]; // Dirichlet (rho, u, v, p) per side
    int circle;           // 1: Circle immersed boundary
    double radius, cx, cy;
    int npoints;          // polygon vertices (CartesianMesh.cpp:360 uses 400)
};
}

namespace {

// Initial condition through the reference's Initialcondition interface
// (Initialcondition.h:6-15): conserved state from an array [4][nx][ny].
class ArrayIC : public Initialcondition {
public:
    ArrayIC(const ref_config& c, const double* U) : m_c(c), m_U(U) {}
    void fillIn(Cell* cell) const override {
        const auto& idx = cell->getElement()->getIndex();
        const int i = static_cast<int>(idx[0]), j = static_cast<int>(idx[1]);
        const size_t n = static_cast<size_t>(m_c.nx) * m_c.ny, k = static_cast<size_t>(i) * m_c.ny + j;
        auto& ph = cell->getPhase();
        ph->setDensity(m_U[k]);
        ph->setU(m_U[n + k]);
        ph->setV(m_U[2 * n + k]);
        ph->setTotalEnergy(m_U[3 * n + k]);
        ph->computePressurefromOther();
    }
    void setBounbdaryCondition(std::vector<std::shared_ptr<Boundary>>& b) override {
        static const double normals[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
        for (int s = 0; s < 4; ++s) {
            if (m_c.bc_type[s] == 1) {
                const double rho = m_c.bc_prim[s][0], u = m_c.bc_prim[s][1], v = m_c.bc_prim[s][2], p = m_c.bc_prim[s][3];
                // Same body as the reference's Dirichlet lambda (Cylinder.cpp:22-32).
                b.push_back(std::make_shared<DirichletBoundary>(normals[s][0], normals[s][1], [rho, u, v, p](Phase& phase) {
                    phase.setDensity(rho);
                    phase.setU(rho * u);
                    phase.setV(rho * v);
                    phase.setPressure(p);
                    phase.computeEnergyfromOther();
                }));
            } else {
                b.push_back(std::make_shared<NeummanBoundary>(normals[s][0], normals[s][1]));
            }
        }
    }

private:
    ref_config m_c;
    const double* m_U;
};

struct Sim {
    std::shared_ptr<Mesh> mesh;
    std::vector<std::vector<Cell>> cells;
    std::vector<std::shared_ptr<Cell>> ghosts, cpuGhosts;
    std::vector<CellInterface> faces;
    std::vector<std::shared_ptr<CellInterface>> ghostFaces;
    std::shared_ptr<Parallel> parallel;
    std::shared_ptr<Explicit> rk;
    std::shared_ptr<ImmersedBoundary> ib;
    std::shared_ptr<Initialcondition> ic;
    int integrator = 3;
};

// Silences the reference's progress prints on std::cout (CartesianParallel.cpp:9-11,
// 22-25,43-44,55-59; Run.cpp:75-78) while the harness sets a grid up.
struct QuietCout {
    std::streambuf* old;
    QuietCout() : old(std::cout.rdbuf(nullptr)) {}
    ~QuietCout() { std::cout.rdbuf(old); std::cout.clear(); }
};

// Run::initialize (Run.cpp:10-90) with config values.
void initialize(Sim& s, const ref_config& c, const double* U) {
    QuietCout quiet;
    auto cm = std::make_shared<CartesianMesh>();
    s.mesh = cm;
    s.mesh->setnumberCellsXGlobal(c.nx);
    s.mesh->setnumberCellsYGlobal(c.ny);
    s.mesh->setGlobalLengthX(c.lx);
    s.mesh->setGlobalLengthY(c.ly);

    s.parallel = std::make_shared<CartesianParallel>();
    s.parallel->setIdAndNumprocs(0, 1);
    s.parallel->setMesh(s.mesh);
    s.parallel->ZoneDcomposition();
    s.parallel->setNeibours();

    s.mesh->allocateCells(s.cells);
    s.mesh->allocateCellInterfaces(s.faces);
    s.mesh->CalCellsize();
    s.mesh->BindCellInterfacesWithCells(s.cells, s.faces);
    s.mesh->SetElement(s.cells);
    s.mesh->SetFace(s.faces);

    model = std::make_shared<EulerMod>();
    interpolation = std::make_shared<Weno5th>();
    gradient = std::make_shared<ForthOrderCS>();
    riemmansolver = std::make_shared<RiemmanSolverHLL>();
    s.ic = std::make_shared<ArrayIC>(c, U);
    s.integrator = c.integrator;
    if (c.integrator == 2) s.rk = std::make_shared<TVD2rdRK>();
    else s.rk = std::make_shared<TVD3rdRK>();
    if (c.circle) {
        s.ib = std::make_shared<Circle>(c.radius, Eigen::Vector2d(c.cx, c.cy));
        // CartesianMesh::setImmersedBoundary (CartesianMesh.cpp:357-374) with the
        // polygon size as a parameter.
        s.ib->Initialize(static_cast<size_t>(c.npoints));
        for (auto& col : s.cells)
            for (auto& cell : col) s.ib->DistinguishWallandFluid(&cell);
        s.ib->SetGhostcell(s.cells, 3);
        for (auto& col : s.cells)
            for (auto& cell : col)
                if (cell.isImmersedGhost()) s.ib->SetImagepoint(&cell, s.cells);
    }
    for (auto& col : s.cells)
        for (auto& cell : col) cell.allocateVar();
    for (auto& f : s.faces) f.allocateVar();

    s.ic->setBounbdaryCondition(s.mesh->getBoundarys());
    s.mesh->InsertBoundaryGhostCells(s.faces, s.ghosts, s.ghostFaces);
    for (auto& g : s.ghosts) g->allocateVar();
    s.parallel->InsertCpuBoundaryGhostCells(s.faces, s.cpuGhosts, s.ghostFaces);
    for (auto& g : s.cpuGhosts) g->allocateVar();
    for (auto& f : s.faces) f.DistinguishType();
}

// Run::solver pre-loop (Run.cpp:95-128), without the HDF5 write.
void preloop(Sim& s, double dt) {
    s.rk->setTimeStep(dt);
    for (auto& col : s.cells)
        for (auto& cell : col)
            if (cell.isFluid()) s.ic->fillIn(&cell);
    for (auto& col : s.cells)
        for (auto& cell : col)
            if (cell.isImmersedGhost()) cell.comImmersedGhostPhase();
    s.parallel->FillSendcellBuffer(s.faces);
    s.parallel->WriteRecvcellBuffer(s.faces);
    for (auto& f : s.faces) f.collectCells();
    for (auto& col : s.cells)
        for (auto& cell : col) {
            cell.collectStencilCells(Direction::X, 5);
            cell.collectStencilCells(Direction::Y, 5);
        }
    s.mesh->ApplyBoundaryCondition(s.faces);
}

// CFL step (addition, no reference counterpart): dt = cfl / max over fluid
// cells of (|u|+c)/dx + (|v|+c)/dy with p from EulerPhase.cpp:132's formula.
double cfl_dt(Sim& s, const ref_config& c) {
    const double dx = c.lx / c.nx, dy = c.ly / c.ny;
    double m = 0.0;
    for (auto& col : s.cells)
        for (auto& cell : col) {
            if (!cell.isFluid()) continue;
            const auto& ph = cell.getPhase();
            const double rho = ph->getDensity(), mx = ph->getU(), my = ph->getV(), E = ph->getTotalEnergy();
            const double p = (Gamma - 1) * (E - 0.5 * (mx * mx + my * my) / rho);
            const double a = std::sqrt(Gamma * p / rho);
            const double u = mx / rho, v = my / rho;
            double w = (std::fabs(u) + a) / dx + (std::fabs(v) + a) / dy;
            if (!(w == w)) w = HUGE_VAL;  // a blown-up cell: dt = 0, as the engine and the oracle take it
            if (w > m) m = w;
        }
    return c.cfl / m;
}

// One loop iteration of Run::solver (Run.cpp:153-233) = one RK stage.
void stage(Sim& s, int i) {
    for (auto& col : s.cells)
        for (auto& cell : col)
            if (cell.isImmersedGhost()) cell.comImmersedGhostPhase();
    s.parallel->exchangedata();
    for (auto& f : s.faces) f.comInterpolationPhase();
    for (auto& f : s.faces) f.computeFlux();
    for (auto& col : s.cells)
        for (auto& cell : col)
            if (cell.isFluid()) s.rk->advance(&cell, i);
    s.mesh->ApplyBoundaryCondition(s.faces);
}

bool step_start(const Sim& s, int i) { return s.integrator == 2 ? (i % 2 == 1) : (i % 3 == 1); }

void dump_state(Sim& s, const ref_config& c, double* U) {
    const size_t n = static_cast<size_t>(c.nx) * c.ny;
    for (int i = 0; i < c.nx; ++i)
        for (int j = 0; j < c.ny; ++j) {
            const auto& ph = s.cells[i][j].getPhase();
            const size_t k = static_cast<size_t>(i) * c.ny + j;
            U[k] = ph->getDensity();
            U[n + k] = ph->getU();
            U[2 * n + k] = ph->getV();
            U[3 * n + k] = ph->getTotalEnergy();
        }
}

void reset_globals() {
    model.reset();
    interpolation.reset();
    riemmansolver.reset();
    gradient.reset();
}

// Reads ImagePoint's protected donor list (ImagePoint.h:25), which has no getter.
struct DonorPeek : ImagePoint {
    static const std::vector<Cell*>& donors(const ImagePoint& p) { return p.*(&DonorPeek::m_cells); }
};

}  // namespace

extern "C" {

// Runs `nstages` loop iterations of Run::solver from the conserved state U_in
// ([4][nx][ny], i = x outer, j = y inner as in Output.cpp:60).  Writes the final
// state (all cells), the last RHS held in each cell's m_flux (Cell.cpp:135-137),
// and the dt used at each stage.  Returns 0.
int ref_run(const ref_config* c, const double* U_in, int nstages, double* U_out, double* rhs_out, double* dt_log) {
    Sim s;
    initialize(s, *c, U_in);
    preloop(s, c->dt);
    double dt = c->dt;
    for (int i = 1; i <= nstages; ++i) {
        if (c->cfl > 0.0 && step_start(s, i)) {
            dt = cfl_dt(s, *c);
            s.rk->setTimeStep(dt);
        }
        if (dt_log) dt_log[i - 1] = dt;
        stage(s, i);
    }
    if (U_out) dump_state(s, *c, U_out);
    if (rhs_out) {
        const size_t n = static_cast<size_t>(c->nx) * c->ny;
        for (int i = 0; i < c->nx; ++i)
            for (int j = 0; j < c->ny; ++j) {
                const auto& f = s.cells[i][j].getFlux();
                const size_t k = static_cast<size_t>(i) * c->ny + j;
                rhs_out[k] = f->getMass();
                rhs_out[n + k] = f->getMomentum()[0];
                rhs_out[2 * n + k] = f->getMomentum()[1];
                rhs_out[3 * n + k] = f->getEnergy();
            }
    }
    reset_globals();
    return 0;
}

// A grid kept between timing calls (one per process: the reference's plugins
// are process globals): create builds it as Run::initialize does, each
// ref_session_stages call runs the next `nstages` solver iterations and
// returns their wall-clock seconds, destroy frees it.
struct RefSession {
    Sim s;
    int next = 1;  // loop counter of the next iteration
};

void* ref_session_create(const ref_config* c, const double* U_in) {
    auto* r = new RefSession();
    initialize(r->s, *c, U_in);
    preloop(r->s, c->dt);
    return r;
}

double ref_session_stages(void* h, int nstages) {
    auto* r = static_cast<RefSession*>(h);
    const auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < nstages; ++k) stage(r->s, r->next++);
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

void ref_session_destroy(void* h) {
    delete static_cast<RefSession*>(h);
    reset_globals();
}

// Wall-clock seconds of `nstages` solver iterations (setup excluded).
double ref_time_stages(const ref_config* c, const double* U_in, int nstages) {
    Sim s;
    initialize(s, *c, U_in);
    preloop(s, c->dt);
    const auto t0 = std::chrono::steady_clock::now();
    for (int i = 1; i <= nstages; ++i) stage(s, i);
    const auto t1 = std::chrono::steady_clock::now();
    reset_globals();
    return std::chrono::duration<double>(t1 - t0).count();
}

// Immersed-boundary set-up as the reference computes it: cell types
// (0 fluid, 1 solid, 2 immersed ghost) in [nx][ny] order, and for each
// immersed-ghost cell in (i outer, j inner) order its (i,j), image point and the
// (i,j) of its donors.  Returns the number of immersed-ghost cells, or -1 when
// more than max_ig.  n_donors < 4 reproduces the reference's short list.
int ref_ib_info(const ref_config* c, int* types, int max_ig, int* ig_ij, double* image_xy, int* donor_ij, int* n_donors) {
    std::vector<double> U(4 * static_cast<size_t>(c->nx) * c->ny, 1.0);
    Sim s;
    initialize(s, *c, U.data());
    int n = 0;
    for (int i = 0; i < c->nx; ++i)
        for (int j = 0; j < c->ny; ++j) {
            Cell& cell = s.cells[i][j];
            types[static_cast<size_t>(i) * c->ny + j] = cell.isFluid() ? 0 : (cell.isSolid() ? 1 : 2);
            if (!cell.isImmersedGhost()) continue;
            if (n >= max_ig) { reset_globals(); return -1; }
            ig_ij[2 * n] = i;
            ig_ij[2 * n + 1] = j;
            const auto& ip = cell.getImagepoint();
            image_xy[2 * n] = ip->getPosition().x();
            image_xy[2 * n + 1] = ip->getPosition().y();
            const auto& d = DonorPeek::donors(*ip);
            n_donors[n] = static_cast<int>(d.size());
            for (size_t k = 0; k < 4; ++k) {
                if (k < d.size()) {
                    donor_ij[8 * n + 2 * k] = static_cast<int>(d[k]->getElement()->getIndex()[0]);
                    donor_ij[8 * n + 2 * k + 1] = static_cast<int>(d[k]->getElement()->getIndex()[1]);
                } else {
                    donor_ij[8 * n + 2 * k] = -1;
                    donor_ij[8 * n + 2 * k + 1] = -1;
                }
            }
            ++n;
        }
    reset_globals();
    return n;
}

// One face through Weno5th::comLeftPhase/comRightPhase (Weno5th.cpp:57-81):
// cells[k][0..3] = (rho, mx, my, E) of the 6-cell stencil (i-3 .. i+2).
// Outputs (rho, mx, my, E, p) of the left and right states.
int ref_weno_face(const double* cells, double* left, double* right) {
    model = std::make_shared<EulerMod>();
    std::vector<Cell> cs(6);
    std::list<Cell*> lst;
    for (int k = 0; k < 6; ++k) {
        cs[k].allocateVar();
        auto& ph = cs[k].getPhase();
        ph->setDensity(cells[4 * k]);
        ph->setU(cells[4 * k + 1]);
        ph->setV(cells[4 * k + 2]);
        ph->setTotalEnergy(cells[4 * k + 3]);
        lst.push_back(&cs[k]);
    }
    Weno5th w;
    std::unique_ptr<Phase> L, R;
    model->allocatePhase(L);
    model->allocatePhase(R);
    w.comLeftPhase(lst, L);
    w.comRightPhase(lst, R);
    const Phase* ps[2] = {L.get(), R.get()};
    double* outs[2] = {left, right};
    for (int s = 0; s < 2; ++s) {
        outs[s][0] = ps[s]->getDensity();
        outs[s][1] = ps[s]->getU();
        outs[s][2] = ps[s]->getV();
        outs[s][3] = ps[s]->getTotalEnergy();
        outs[s][4] = ps[s]->getPressure();
    }
    reset_globals();
    return 0;
}

// One face through EulerMod::comFlux + RiemmanSolverHLL::Solver
// (CellInterface.cpp:68-89).  L, R = (rho, mx, my, E); dir 0 = X, 1 = Y.
int ref_hll(const double* L, const double* R, int dir, double* flux) {
    model = std::make_shared<EulerMod>();
    riemmansolver = std::make_shared<RiemmanSolverHLL>();
    std::unique_ptr<Phase> pl, pr;
    model->allocatePhase(pl);
    model->allocatePhase(pr);
    const double* src[2] = {L, R};
    std::unique_ptr<Phase>* dst[2] = {&pl, &pr};
    for (int s = 0; s < 2; ++s) {
        (*dst[s])->setDensity(src[s][0]);
        (*dst[s])->setU(src[s][1]);
        (*dst[s])->setV(src[s][2]);
        (*dst[s])->setTotalEnergy(src[s][3]);
        (*dst[s])->computePressurefromOther();
    }
    const Direction d = dir == 0 ? Direction::X : Direction::Y;
    auto fl = model->comFlux(pl, d);
    auto fr = model->comFlux(pr, d);
    auto res = riemmansolver->Solver(pl, pr, fl, fr, d);
    flux[0] = res->getMass();
    flux[1] = res->getMomentum()[0];
    flux[2] = res->getMomentum()[1];
    flux[3] = res->getEnergy();
    reset_globals();
    return 0;
}

// The reference's (unwired) viscous path on a grid state: after the pre-loop,
// temperature T = Gamma Ma^2 p / rho (EulerPhase.cpp:135-138) is computed for
// every interior and physical ghost cell (the reference never calls it), then
// Cell::comPrimitiveGradient on every cell (Cell.cpp:164-170) and
// CellInterface::comviscousflux on every face (CellInterface.cpp:115-119).
// grad_out: [6][nx][ny] = (u_x, u_y, v_x, v_y, T_x, T_y).
// fvx_out: [4][nx+1][ny] x-normal faces, fvy_out: [4][nx][ny+1] y-normal faces,
// indexed by the face's (i, j) as in CartesianMesh.cpp:27-31,50-54.
int ref_viscous(const ref_config* c, const double* U_in, double* grad_out, double* fvx_out, double* fvy_out) {
    Sim s;
    initialize(s, *c, U_in);
    preloop(s, c->dt);
    for (auto& col : s.cells)
        for (auto& cell : col) cell.getPhase()->computeTemperaturefromOther();
    s.mesh->ApplyBoundaryCondition(s.faces);
    for (auto& g : s.ghosts) g->getPhase()->computeTemperaturefromOther();
    for (auto& col : s.cells)
        for (auto& cell : col) cell.comPrimitiveGradient();
    for (auto& f : s.faces) f.comviscousflux();
    const int nx = c->nx, ny = c->ny;
    const size_t n = static_cast<size_t>(nx) * ny;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            const auto& g = s.cells[i][j].getGradient();
            const size_t k = static_cast<size_t>(i) * ny + j;
            grad_out[k] = g->getUGradient()[0];
            grad_out[n + k] = g->getUGradient()[1];
            grad_out[2 * n + k] = g->getVGradient()[0];
            grad_out[3 * n + k] = g->getVGradient()[1];
            grad_out[4 * n + k] = g->getTGradient()[0];
            grad_out[5 * n + k] = g->getTGradient()[1];
        }
    const size_t nfx = static_cast<size_t>(nx + 1) * ny, nfy = static_cast<size_t>(nx) * (ny + 1);
    for (int i = 0; i <= nx; ++i)
        for (int j = 0; j < ny; ++j) {
            const auto& f = s.faces[i + j * (nx + 1)].getvisflux();
            const size_t k = static_cast<size_t>(i) * ny + j;
            fvx_out[k] = f->getMass();
            fvx_out[nfx + k] = f->getMomentum()[0];
            fvx_out[2 * nfx + k] = f->getMomentum()[1];
            fvx_out[3 * nfx + k] = f->getEnergy();
        }
    const size_t nh = static_cast<size_t>(nx + 1) * ny;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j <= ny; ++j) {
            const auto& f = s.faces[nh + i + static_cast<size_t>(j) * nx].getvisflux();
            const size_t k = static_cast<size_t>(i) * (ny + 1) + j;
            fvy_out[k] = f->getMass();
            fvy_out[nfy + k] = f->getMomentum()[0];
            fvy_out[2 * nfy + k] = f->getMomentum()[1];
            fvy_out[3 * nfy + k] = f->getEnergy();
        }
    reset_globals();
    return 0;
}

#ifdef CFS_WITH_GPU_PLUGINS
// ref_run's loop with the product's GPU plugins registered in place of the
// reference's (the drop-in at Run.cpp:41-48): EulerMod, Weno5th, HLL and the
// RK class are swapped for cfs_plugins' subclasses before the pre-loop, so the
// reference's own loop drives one cfs_stage per iteration.  precision:
// cfs_precision.  Fixed dt only.  Returns 0, or -1 with the message in err.
int ref_gpu_run(const ref_config* c, const double* U_in, int nstages, int precision, double* U_out, char* err,
                int err_len) {
    try {
        Sim s;
        initialize(s, *c, U_in);
        cfs_config cfg;
        cfs_config_default(&cfg);
        cfg.nx = c->nx;
        cfg.ny = c->ny;
        cfg.lx = c->lx;
        cfg.ly = c->ly;
        cfg.precision = precision;
        cfg.rk = c->integrator == 2 ? CFS_RK_TVD2 : CFS_RK_TVD3_REFERENCE;
        cfg.hll = CFS_HLL_REFERENCE;
        for (int k = 0; k < 4; ++k) {
            cfg.bc[k] = c->bc_type[k] == 1 ? CFS_BC_DIRICHLET : CFS_BC_NEUMANN;
            for (int q = 0; q < 4; ++q) cfg.bc_prim[k][q] = c->bc_prim[k][q];
        }
        auto gpu = std::make_shared<cfs_plugins::Session>(cfg, s.cells);
        if (c->circle) gpu->set_circle(c->radius, c->cx, c->cy, c->npoints);
        gpu->set_sync_interval(0);
        model = std::make_shared<cfs_plugins::GpuModel>();
        interpolation = std::make_shared<cfs_plugins::GpuInterpolation>();
        riemmansolver = std::make_shared<cfs_plugins::GpuRiemannSolver>();
        gradient = std::make_shared<cfs_plugins::GpuGradient>();
        s.rk = std::make_shared<cfs_plugins::GpuExplicit>(gpu);
        preloop(s, c->dt);
        for (int i = 1; i <= nstages; ++i) stage(s, i);
        gpu->sync_to_host();
        if (U_out) dump_state(s, *c, U_out);
        const long long ran = gpu->stages_run();
        s.rk.reset();
        reset_globals();
        return ran == nstages ? 0 : -1;
    } catch (const std::exception& e) {
        if (err && err_len > 0) {
            std::strncpy(err, e.what(), static_cast<size_t>(err_len - 1));
            err[err_len - 1] = 0;
        }
        reset_globals();
        return -1;
    }
}
#endif

}  // extern "C"
