// GPU plugins for the reference program (see cfs_plugins.h).
#include "cfs_plugins.h"

#include <stdexcept>
#include <string>

namespace cfs_plugins {

Session::Session(const cfs_config& cfg, std::vector<std::vector<Cell>>& cells) : cfg_(cfg), cells_(cells) {
    if (static_cast<int>(cells.size()) != cfg.nx || cells.empty() || static_cast<int>(cells[0].size()) != cfg.ny)
        throw std::runtime_error("cfs_plugins::Session: the Cell grid is not nx x ny");
    check(cfs_create(&cfg_, &ctx_));
}

Session::~Session() {
    if (ctx_) cfs_destroy(ctx_);
}

void Session::check(int rc) const {
    if (rc != CFS_OK) throw std::runtime_error(std::string("cfs error ") + std::to_string(rc) + ": " + cfs_last_error(ctx_));
}

void Session::set_circle(double radius, double cx, double cy, int npoints) {
    check(cfs_ib_build_circle(ctx_, radius, cx, cy, npoints, CFS_IB_REFERENCE));
}

// Cells -> device, reference order U[4][nx][ny] (Output.cpp:60).
void Session::upload() {
    const int nx = cfg_.nx, ny = cfg_.ny;
    const size_t n = static_cast<size_t>(nx) * ny;
    std::vector<double> U(4 * n);
    fluid_cells_ = 0;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            Cell& c = cells_[i][j];
            const auto& ph = c.getPhase();
            const size_t k = static_cast<size_t>(i) * ny + j;
            U[k] = ph->getDensity();
            U[n + k] = ph->getU();
            U[2 * n + k] = ph->getV();
            U[3 * n + k] = ph->getTotalEnergy();
            if (c.isFluid()) ++fluid_cells_;
        }
    check(cfs_set_state(ctx_, U.data()));
    uploaded_ = true;
}

void Session::on_advance(int step, double dt) {
    if (step != current_step_) {
        if (!uploaded_) upload();
        check(cfs_stage(ctx_, step, dt));
        ++stages_;
        current_step_ = step;
        calls_ = 0;
    }
    if (++calls_ == fluid_cells_ && sync_every_ > 0 && step % sync_every_ == 0) sync_to_host();
}

void Session::sync_to_host() {
    if (!uploaded_) return;
    const int nx = cfg_.nx, ny = cfg_.ny;
    const size_t n = static_cast<size_t>(nx) * ny;
    std::vector<double> U(4 * n);
    check(cfs_get_state(ctx_, U.data()));
    std::vector<double> R;
    if (cfg_.keep_rhs && stages_ > 0) {
        R.resize(4 * n);
        check(cfs_get_rhs(ctx_, R.data()));
    }
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            Cell& c = cells_[i][j];
            auto& ph = c.getPhase();
            const size_t k = static_cast<size_t>(i) * ny + j;
            ph->setDensity(U[k]);
            ph->setU(U[n + k]);
            ph->setV(U[2 * n + k]);
            ph->setTotalEnergy(U[3 * n + k]);
            ph->computePressurefromOther();
            if (!R.empty() && c.isFluid()) {
                auto& f = c.getFlux();
                f->setMass(R[k]);
                f->setMomentum(Flux::Coord(R[n + k], R[2 * n + k]));
                f->setEnergy(R[3 * n + k]);
            }
        }
}

std::shared_ptr<Flux> GpuModel::comFlux(const std::unique_ptr<Phase>&, Direction) { return zero_; }

std::shared_ptr<Flux> GpuRiemannSolver::Solver(std::unique_ptr<Phase>&, std::unique_ptr<Phase>&, std::shared_ptr<Flux>,
                                               std::shared_ptr<Flux>&, Direction) {
    return zero_;
}

void GpuRiemannSolver::info() { std::cout << "HLL on the GPU (cfs_stage)" << std::endl; }

}  // namespace cfs_plugins
