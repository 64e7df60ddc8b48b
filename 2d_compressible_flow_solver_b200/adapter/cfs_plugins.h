// GPU plugins for the reference program: drop-in subclasses of its plugin
// interfaces, registered where Run::initialize selects its plugins
// (Run.cpp:41-48 and the process globals of Run.cpp:5-8 / 49-52).
//
// The reference's loop (Run.cpp:153-233) keeps calling its per-face and
// per-cell plugin methods.  With these plugins:
//   * Interpolation::comLeftPhase/comRightPhase (Interpolation.h:14-15),
//     Model::comFlux (model.h) and RiemmanSolver::Solver (RiemmanSolver.h:12)
//     do nothing (the solver hands back one shared zero flux);
//   * the first Explicit::advance call of each loop iteration (Explicit.h:10)
//     runs that iteration's whole stage on the GPU through the C ABI
//     (cfs_stage with the loop counter: immersed-ghost fill, WENO5 + HLL on
//     every face, RHS and RK update of every fluid cell, boundary ghosts); the
//     remaining calls of the iteration are counted and return;
//   * after the last call of an iteration i with i % sync_every == 0 the
//     device state is copied back into every Cell's phase, ahead of
//     Output::WriteToHDF5 (Run.cpp:205-207 writes every 50 iterations).
// The state is uploaded from the Cells at the first advance call, i.e. after
// the initial condition and the first immersed-ghost fill (Run.cpp:97-110).
// Host-side work the loop still does (immersed-ghost fill on the host copy,
// boundary copies, the per-element virtual calls) no longer feeds the result.
//
// Errors: the reference has no error convention; a failing cfs_* call throws
// std::runtime_error carrying cfs_last_error.
//
// Integration in Run.cpp:
//     auto gpu = std::make_shared<cfs_plugins::Session>(cfg, m_cellsLv1);
//     gpu->set_circle(0.1, 0.5, 1.0, 400);          // the Circle of Run.cpp:48
//     m_model = std::make_shared<cfs_plugins::GpuModel>();
//     m_interpolation = std::make_shared<cfs_plugins::GpuInterpolation>();
//     m_riemmansolver = std::make_shared<cfs_plugins::GpuRiemannSolver>();
//     m_timeadvance = std::make_shared<cfs_plugins::GpuExplicit>(gpu);
//     gradient = std::make_shared<cfs_plugins::GpuGradient>();  // Run.cpp:8, if used
// and gpu->sync_to_host() before the final Output::WriteToHDF5 (Run.cpp:235).
#pragma once

#include "cfs.h"

#include "flux/EulerFlux.h"
// RiemmanSolver.h has no working include guard ("#pragma ocne", RiemmanSolver.h:1),
// so it is reached only through the guarded RiemmanSolverHLL.h, as the
// reference's own sources do.
#include "flux/RiemmanSolverHLL.h"
#include "gradient/FourthOrderCS.h"
#include "interpolation/Interpolation.h"
#include "meshes/Cell.h"
#include "model/EulerMod.h"
#include "timeadvance/Explicit.h"

#include <memory>
#include <vector>

namespace cfs_plugins {

class Session {
public:
    // cfg: grid, sides, precision and integrator of the run (cfg.rk must match
    // the Explicit plugin the reference would have used: CFS_RK_TVD2 for
    // TVD2rdRK, CFS_RK_TVD3_REFERENCE for TVD3rdRK).  cells: the rank's
    // Cell grid (Run::m_cellsLv1), cells[i][j] with i along x.
    Session(const cfs_config& cfg, std::vector<std::vector<Cell>>& cells);
    ~Session();
    Session(const Session&) = delete;
    Session& operator=(const Session&) = delete;

    // Circle immersed boundary with the reference's classification, image
    // points and donors (Circle.cpp) and its LDLT fill (CFS_IB_REFERENCE).
    void set_circle(double radius, double cx, double cy, int npoints);
    // Copy the device state to the Cells after iterations i % every == 0
    // (0: never; sync_to_host on demand).
    void set_sync_interval(int every) { sync_every_ = every; }

    // Explicit::advance of one fluid cell in loop iteration `step`.
    void on_advance(int step, double dt);
    // Device state -> every Cell's phase (pressure recomputed from the
    // conserved variables, EulerPhase.cpp:130-133); with cfg.keep_rhs, the
    // last stage's RHS -> every fluid Cell's flux (Cell.cpp:135-137).
    void sync_to_host();

    cfs_ctx* context() { return ctx_; }
    long long stages_run() const { return stages_; }

private:
    void check(int rc) const;
    void upload();

    cfs_config cfg_{};
    std::vector<std::vector<Cell>>& cells_;
    cfs_ctx* ctx_ = nullptr;
    long long fluid_cells_ = 0;
    long long calls_ = 0;
    long long stages_ = 0;
    int current_step_ = -1;
    int sync_every_ = 50;
    bool uploaded_ = false;
};

// Interpolation plugin: reconstruction runs inside the GPU stage.
class GpuInterpolation : public Interpolation {
public:
    void comLeftPhase(std::list<Cell*>&, std::unique_ptr<Phase>&) override {}
    void comRightPhase(std::list<Cell*>&, std::unique_ptr<Phase>&) override {}
};

// Model plugin: EulerMod's allocation of phases and fluxes, no flux evaluation.
class GpuModel : public EulerMod {
public:
    std::shared_ptr<Flux> comFlux(const std::unique_ptr<Phase>&, Direction) override;

private:
    std::shared_ptr<Flux> zero_ = std::make_shared<EulerFlux>(0.0, Flux::Coord(0.0, 0.0), 0.0);
};

// Riemann-solver plugin: the HLL flux is computed inside the GPU stage.
class GpuRiemannSolver : public RiemmanSolver {
public:
    std::shared_ptr<Flux> Solver(std::unique_ptr<Phase>&, std::unique_ptr<Phase>&, std::shared_ptr<Flux>,
                                 std::shared_ptr<Flux>&, Direction) override;
    void info() override;

private:
    std::shared_ptr<Flux> zero_ = std::make_shared<EulerFlux>(0.0, Flux::Coord(0.0, 0.0), 0.0);
};

// Gradient plugin (ForthOrderCS, FourthOrderCS.h:15-16): the viscous
// derivatives and face fluxes are computed inside the GPU stage when the
// session's config selects CFS_VISCOUS_NS (cfg.mu, cfg.prandtl, cfg.mach), so
// the per-face and per-cell calls, which the reference's loop makes only if its
// commented-out gradient calls (Run.cpp:175-179, 188) are restored, do nothing.
class GpuGradient : public ForthOrderCS {
public:
    void comviscousfluxForcellinterface(CellInterface*, std::list<Cell*>&, Direction) override {}
    void comprimitivederivativeForcell(Cell*, std::vector<Cell*>&, Direction) override {}
};

// Explicit (time-advance) plugin: one GPU stage per loop iteration.
class GpuExplicit : public Explicit {
public:
    explicit GpuExplicit(std::shared_ptr<Session> s) : s_(std::move(s)) { m_dt = 0.0; }
    void advance(Cell*, const int& step) override { s_->on_advance(step, m_dt); }
    void setTimeStep(const double& dt) override { m_dt = dt; }
    const double& getTimeStep() const override { return m_dt; }

private:
    std::shared_ptr<Session> s_;
};

}  // namespace cfs_plugins
