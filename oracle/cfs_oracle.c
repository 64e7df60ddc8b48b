/* Test infrastructure (oracle only) -- see cfs_oracle.h.
 *
 * The "reference" variants evaluate every expression in the operation order of
 * the reference source they cite, so that, built with -ffp-contract=off and no
 * fast-math, they reproduce the reference's doubles bit for bit (checked
 * against oracle/_ref/libref_strict.so by tests/test_oracle.py).  The other
 * variants have no reference counterpart and are the checker for the features
 * the reference cannot express.
 */
#include "cfs_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NV 4

static inline size_t ncell(const orc_config* c) { return (size_t)c->nx * (size_t)c->ny; }

/* Value of variable v of cell (i, j), where i or j may lie up to 3 cells
 * outside the grid.  A physical side repeats ONE ghost cell for all three
 * stencil slots, because CellInterface::collectCells (CellInterface.cpp:147-179)
 * stops walking at a boundary face; the Neumann ghost is a copy of the adjacent
 * interior cell (NeummanBoundary.cpp:31-45), the Dirichlet ghost a fixed state
 * (DirichletBoundary.cpp:32-46).  Periodic sides wrap (no reference). */
static inline double cval(const orc_config* c, const double* U, int v, int i, int j) {
    if (i < 0) {
        if (c->bc[0] == ORC_BC_DIRICHLET) return c->bc_U[0][v];
        i = (c->bc[0] == ORC_BC_PERIODIC) ? i + c->nx : 0;
    } else if (i >= c->nx) {
        if (c->bc[1] == ORC_BC_DIRICHLET) return c->bc_U[1][v];
        i = (c->bc[1] == ORC_BC_PERIODIC) ? i - c->nx : c->nx - 1;
    }
    if (j < 0) {
        if (c->bc[2] == ORC_BC_DIRICHLET) return c->bc_U[2][v];
        j = (c->bc[2] == ORC_BC_PERIODIC) ? j + c->ny : 0;
    } else if (j >= c->ny) {
        if (c->bc[3] == ORC_BC_DIRICHLET) return c->bc_U[3][v];
        j = (c->bc[3] == ORC_BC_PERIODIC) ? j - c->ny : c->ny - 1;
    }
    return U[(size_t)v * ncell(c) + (size_t)i * c->ny + j];
}

/* Cell index at stencil slot k (0..5) of the face between cells a-1 and a of a
 * line of n cells, i.e. nominally a-3+k.  CellInterface::collectCells
 * (CellInterface.cpp:147-179) stops BOTH of its walkers when the face itself is
 * a physical boundary face (:172-178 test the face it stands on), so on such a
 * face every interior slot repeats the first interior cell: the left boundary
 * face reads [g, g, g, c0, c0, c0] and the right one [c, c, c, g, g, g]. */
static inline int face_slot(int a, int k, int n, int lo_periodic, int hi_periodic) {
    int i = a - 3 + k;
    if (a == 0 && !lo_periodic && k >= 3) i = 0;
    if (a == n && !hi_periodic && k <= 2) i = n - 1;
    return i;
}

/* True when (i, j) is a physical ghost position (outside a non-periodic side). */
static inline int is_phys_ghost(const orc_config* c, int i, int j) {
    if (i < 0) return c->bc[0] != ORC_BC_PERIODIC;
    if (i >= c->nx) return c->bc[1] != ORC_BC_PERIODIC;
    if (j < 0) return c->bc[2] != ORC_BC_PERIODIC;
    if (j >= c->ny) return c->bc[3] != ORC_BC_PERIODIC;
    return 0;
}

/* Weno5th::weno5Interpolation, Weno5th.cpp:4-28 (eps is 1e-2 there). */
double orc_weno5(const double v[5], double eps) {
    double beta0 = (13.0 / 12.0) * ((v[0] - 2 * v[1] + v[2]) * (v[0] - 2 * v[1] + v[2]))
                 + 0.25 * ((v[0] - 4 * v[1] + 3 * v[2]) * (v[0] - 4 * v[1] + 3 * v[2]));
    double beta1 = (13.0 / 12.0) * ((v[1] - 2 * v[2] + v[3]) * (v[1] - 2 * v[2] + v[3]))
                 + 0.25 * ((v[1] - v[3]) * (v[1] - v[3]));
    double beta2 = (13.0 / 12.0) * ((v[2] - 2 * v[3] + v[4]) * (v[2] - 2 * v[3] + v[4]))
                 + 0.25 * ((3 * v[2] - 4 * v[3] + v[4]) * (3 * v[2] - 4 * v[3] + v[4]));
    double alpha0 = 0.1 / ((eps + beta0) * (eps + beta0));
    double alpha1 = 0.6 / ((eps + beta1) * (eps + beta1));
    double alpha2 = 0.3 / ((eps + beta2) * (eps + beta2));
    double sum_alpha = alpha0 + alpha1 + alpha2;
    double omega0 = alpha0 / sum_alpha;
    double omega1 = alpha1 / sum_alpha;
    double omega2 = alpha2 / sum_alpha;
    return omega0 * (v[0] / 3.0 - 7.0 * v[1] / 6.0 + 11.0 * v[2] / 6.0)
         + omega1 * (-v[1] / 6.0 + 5.0 * v[2] / 6.0 + v[3] / 3.0)
         + omega2 * (v[2] / 3.0 + 5.0 * v[3] / 6.0 - v[4] / 6.0);
}

/* EulerPhase::computePressurefromOther, EulerPhase.cpp:130-133. */
static inline double pressure(double g, double rho, double mx, double my, double E) {
    return (g - 1) * (E - 0.5 * (mx * mx + my * my) / rho);
}

/* Weno5th::comInterpolation on the 5 cells of one side (Weno5th.cpp:30-55):
 * P = (rho, mx, my, E, p). */
static void reconstruct(const orc_config* c, const double s[5][NV], double P[5]) {
    double v[5];
    for (int q = 0; q < NV; ++q) {
        for (int k = 0; k < 5; ++k) v[k] = s[k][q];
        P[q] = orc_weno5(v, c->weno_eps);
    }
    P[4] = pressure(c->gamma, P[0], P[1], P[2], P[3]);
}

/* EulerMod::comFlux, EulerMod.cpp:33-54 (dir 0 = X, 1 = Y). */
static void phys_flux(const double P[5], int dir, double F[4]) {
    const double rho = P[0], u = P[1], v = P[2], E = P[3], p = P[4];
    if (dir == 0) {
        F[0] = u;
        F[1] = u * u / rho + p;
        F[2] = u * v / rho;
        F[3] = (E + p) * (u / rho);
    } else {
        F[0] = v;
        F[1] = u * v / rho;
        F[2] = v * v / rho + p;
        F[3] = (E + p) * (v / rho);
    }
}

static inline double min_ref(double a, double b) { return (b < a) ? b : a; } /* std::min */
static inline double max_ref(double a, double b) { return (a < b) ? b : a; } /* std::max */

/* RiemmanSolverHLL::Solver, RiemmanSolverHLL.cpp:5-75, including its wave-speed
 * choice (left momentum in both bounds, :41-42).  ORC_HLL_DAVIS uses the Davis
 * bounds min/max(u_L -+ a_L, u_R -+ a_R) from velocities (no reference). */
static void hll(const orc_config* c, const double L[5], const double R[5], int dir, double F[4]) {
    const double g = c->gamma;
    double FL[4], FR[4];
    phys_flux(L, dir, FL);
    phys_flux(R, dir, FR);
    const double rhoL = L[0], pL = L[4], EL = L[3];
    const double rhoR = R[0], pR = R[4], ER = R[3];
    const double aL = sqrt(g * pL / rhoL);
    const double aR = sqrt(g * pR / rhoR);
    const int idx = (dir == 0) ? 1 : 2;
    const double qL = L[idx], qR = R[idx];
    double SL, SR;
    if (c->hll == ORC_HLL_REFERENCE) {
        double a_ave = 0.5 * (aL + aR);
        double rho_ave = 0.5 * (rhoL + rhoR);
        double p_star = 0.5 * (pL + pR) - 0.5 * (qR / rhoR - qL / rhoL) * rho_ave * a_ave;
        double u_star = 0.5 * (qR / rhoR + qL / rhoL) - 0.5 * (pR - pL) / (rho_ave * a_ave);
        double rho_star_L = rhoL + (qL / rhoL - u_star) * rho_ave / a_ave;
        double rho_star_R = rhoR - (qR / rhoR - u_star) * rho_ave / a_ave;
        double a_star_L = sqrt(g * p_star / rho_star_L);
        double a_star_R = sqrt(g * p_star / rho_star_R);
        SL = min_ref(qL - aL, u_star - a_star_L);
        SR = max_ref(qL + aL, u_star + a_star_R);
    } else {
        const double uL = qL / rhoL, uR = qR / rhoR;
        SL = min_ref(uL - aL, uR - aR);
        SR = max_ref(uL + aL, uR + aR);
    }
    if (SL >= 0) {
        for (int q = 0; q < 4; ++q) F[q] = FL[q];
    } else if (SR <= 0) {
        for (int q = 0; q < 4; ++q) F[q] = FR[q];
    } else {
        double inv_SR_SL = 1.0 / (SR - SL);
        F[0] = (SR * FL[0] - SL * FR[0] + SL * SR * (rhoR - rhoL)) * inv_SR_SL;
        F[1] = (SR * FL[1] - SL * FR[1] + SL * SR * (R[1] - L[1])) * inv_SR_SL;
        F[2] = (SR * FL[2] - SL * FR[2] + SL * SR * (R[2] - L[2])) * inv_SR_SL;
        F[3] = (SR * FL[3] - SL * FR[3] + SL * SR * (ER - EL)) * inv_SR_SL;
    }
}

int orc_hll(const orc_config* c, const double L4[4], const double R4[4], int dir, double F[4]) {
    double L[5] = {L4[0], L4[1], L4[2], L4[3], pressure(c->gamma, L4[0], L4[1], L4[2], L4[3])};
    double R[5] = {R4[0], R4[1], R4[2], R4[3], pressure(c->gamma, R4[0], R4[1], R4[2], R4[3])};
    hll(c, L, R, dir, F);
    return 0;
}

/* Interface flux from the 6-cell stencil s[0..5] = cells (a-3 .. a+2) across the
 * face between cells a-1 and a: left state from s[0..4], right state from the
 * reversed s[5..1] (Weno5th.cpp:57-81), then HLL (CellInterface.cpp:68-89).
 * Positivity fallbacks (no reference counterpart): ORC_POS_FACE replaces a
 * state with rho <= 0 or p <= 0 (or NaN) by the cell next to the face on its
 * side; ORC_POS_BODY also takes both cells' values (first order) when lowo,
 * i.e. the stencil holds an immersed-ghost or solid cell. */
static void face_flux(const orc_config* c, const double s[6][NV], int dir, double F[4], int lowo) {
    double sl[5][NV], sr[5][NV], L[5], R[5];
    for (int k = 0; k < 5; ++k)
        for (int q = 0; q < NV; ++q) {
            sl[k][q] = s[k][q];
            sr[k][q] = s[5 - k][q];
        }
    reconstruct(c, sl, L);
    reconstruct(c, sr, R);
    if (c->positivity) {
        /* first-order fallback of a non-physical WENO state: the cell next to
         * the face on that side (s[2] left, s[3] right) */
        if (lowo || !(L[0] > 0) || !(L[4] > 0)) {
            for (int q = 0; q < NV; ++q) L[q] = s[2][q];
            L[4] = pressure(c->gamma, L[0], L[1], L[2], L[3]);
        }
        if (lowo || !(R[0] > 0) || !(R[4] > 0)) {
            for (int q = 0; q < NV; ++q) R[q] = s[3][q];
            R[4] = pressure(c->gamma, R[0], R[1], R[2], R[3]);
        }
    }
    hll(c, L, R, dir, F);
}

/* ---- Pivoted LDL^T of the lower triangle (the Eigen-API shim's algorithm,
 * oracle/shim/eigen_shim.h), used by the reference's immersed-boundary fill. */
typedef struct {
    double l[4][4], d[4];
    int perm[4];
} ldlt4;

static void ldlt4_factor(const double a[4][4], ldlt4* f) {
    double w[4][4];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            w[r][c] = (r >= c) ? a[r][c] : a[c][r];
            f->l[r][c] = 0.0;
        }
    for (int k = 0; k < 4; ++k) f->perm[k] = k;
    for (int k = 0; k < 4; ++k) {
        int p = k;
        double best = fabs(w[k][k]);
        for (int i = k + 1; i < 4; ++i) {
            const double v = fabs(w[i][i]);
            if (v > best) { best = v; p = i; }
        }
        if (p != k) {
            for (int c = 0; c < 4; ++c) { double t = w[k][c]; w[k][c] = w[p][c]; w[p][c] = t; }
            for (int r = 0; r < 4; ++r) { double t = w[r][k]; w[r][k] = w[r][p]; w[r][p] = t; }
            for (int c = 0; c < k; ++c) { double t = f->l[k][c]; f->l[k][c] = f->l[p][c]; f->l[p][c] = t; }
            int t = f->perm[k]; f->perm[k] = f->perm[p]; f->perm[p] = t;
        }
        const double d = w[k][k];
        f->d[k] = d;
        const int usable = fabs(d) > DBL_MIN;
        for (int i = k + 1; i < 4; ++i) f->l[i][k] = usable ? w[i][k] / d : 0.0;
        for (int i = k + 1; i < 4; ++i)
            for (int j = k + 1; j < 4; ++j) w[i][j] = w[i][j] - f->l[i][k] * d * f->l[j][k];
    }
}

static void ldlt4_solve(const ldlt4* f, const double b[4], double x[4]) {
    double y[4];
    for (int k = 0; k < 4; ++k) y[k] = b[f->perm[k]];
    for (int i = 0; i < 4; ++i)
        for (int k = 0; k < i; ++k) y[i] -= f->l[i][k] * y[k];
    for (int i = 0; i < 4; ++i) y[i] = (fabs(f->d[i]) > DBL_MIN) ? y[i] / f->d[i] : 0.0;
    for (int i = 3; i >= 0; --i)
        for (int k = i + 1; k < 4; ++k) y[i] -= f->l[k][i] * y[k];
    for (int k = 0; k < 4; ++k) x[f->perm[k]] = y[k];
}

/* Slip-form donors (no reference counterpart): bilinear tensor weights over the
 * 2 x 2 block of cell centres around (X, Y), restricted to fluid cells and
 * renormalised; inverse-squared-distance weights over the given donors when the
 * block keeps less than 1e-3 of the weight. */
static void slip_weights(const orc_config* c, const uint8_t* types, double X, double Y, const int32_t fb[4],
                         int32_t d[4], double w[4]) {
    const int nx = c->nx, ny = c->ny;
    const double dx = c->lx / nx, dy = c->ly / ny;
    const double fx = (X - 0.5 * dx) / dx, fy = (Y - 0.5 * dy) / dy;
    const int i0 = (int)floor(fx), j0 = (int)floor(fy);
    const double tx = fx - i0, ty = fy - j0;
    double sum = 0.0;
    int keep = -1;
    for (int k = 0; k < 4; ++k) {
        const int i = i0 + (k & 1), j = j0 + (k >> 1);
        const double wk = ((k & 1) ? tx : 1 - tx) * ((k >> 1) ? ty : 1 - ty);
        const int ok = i >= 0 && i < nx && j >= 0 && j < ny && (!types || types[(size_t)i * ny + j] == ORC_CELL_FLUID);
        d[k] = ok ? i * ny + j : -1;
        w[k] = ok ? wk : 0.0;
        if (ok) {
            sum += wk;
            if (keep < 0) keep = k;
        }
    }
    if (sum > 1e-3) {
        for (int k = 0; k < 4; ++k) {
            if (d[k] < 0) d[k] = d[keep];
            w[k] /= sum;
        }
        return;
    }
    double s = 0.0;
    for (int k = 0; k < 4; ++k) {
        const int i = fb[k] / ny, j = fb[k] % ny;
        const double ex = (i + 0.5) * dx - X, ey = (j + 0.5) * dy - Y;
        w[k] = 1.0 / (ex * ex + ey * ey + 1e-300);
        d[k] = fb[k];
        s += w[k];
    }
    for (int k = 0; k < 4; ++k) w[k] /= s;
}

/* Cell::comImmersedGhostPhase -> ImagePoint::InterpolatePhase
 * (Cell.cpp:172-181, ImagePoint.cpp:20-82): donor rows [x y, x, y, 1] with cell
 * centres x = (i + 0.5) dx (CartesianMesh.cpp:92), LDLT of that matrix, four
 * solves, value = W0 X Y + W1 X + W2 Y + W3 at the image point, then
 * (rho, -mx, -my, E).  ORC_IB_BILINEAR_SLIP: bilinear weights and only the wall-
 * normal momentum reflected (no reference counterpart). */
int orc_ib_fill(const orc_config* c, const orc_ib* ib, double* U) {
    if (!ib || ib->n <= 0) return 0;
    const size_t n = ncell(c);
    const double dx = c->lx / c->nx, dy = c->ly / c->ny;
    for (int g = 0; g < ib->n; ++g) {
        double M[4][4], f[4][4];
        for (int k = 0; k < 4; ++k) {
            const int d = ib->donor[4 * g + k];
            const int i = d / c->ny, j = d % c->ny;
            const double x = (i + 0.5) * dx, y = (j + 0.5) * dy;
            M[k][0] = x * y;
            M[k][1] = x;
            M[k][2] = y;
            M[k][3] = 1.0;
            for (int q = 0; q < NV; ++q) f[q][k] = U[(size_t)q * n + (size_t)d];
        }
        const double X = ib->image[2 * g], Y = ib->image[2 * g + 1];
        double val[4];
        if (ib->mode == ORC_IB_REFERENCE) {
            ldlt4 fac;
            ldlt4_factor(M, &fac);
            for (int q = 0; q < NV; ++q) {
                double W[4];
                ldlt4_solve(&fac, f[q], W);
                val[q] = W[0] * X * Y + W[1] * X + W[2] * Y + W[3];
            }
            val[1] = -val[1];
            val[2] = -val[2];
        } else {
            int32_t d[4];
            double w[4];
            slip_weights(c, ib->types, X, Y, &ib->donor[4 * g], d, w);
            for (int q = 0; q < NV; ++q) {
                val[q] = 0.0;
                for (int k = 0; k < 4; ++k) val[q] += w[k] * U[(size_t)q * n + (size_t)d[k]];
            }
            const double nx_ = ib->normal[2 * g], ny_ = ib->normal[2 * g + 1];
            const double mn = val[1] * nx_ + val[2] * ny_;
            val[1] = val[1] - 2.0 * mn * nx_;
            val[2] = val[2] - 2.0 * mn * ny_;
        }
        const size_t cell = (size_t)ib->cell[g];
        for (int q = 0; q < NV; ++q) U[(size_t)q * n + cell] = val[q];
    }
    return 0;
}

double orc_cfl_dt(const orc_config* c, const uint8_t* types, const double* U, double cfl) {
    const size_t n = ncell(c);
    const double dx = c->lx / c->nx, dy = c->ly / c->ny, g = c->gamma;
    double m = 0.0;
#pragma omp parallel for reduction(max : m) num_threads(c->nthreads > 0 ? c->nthreads : omp_get_max_threads())
    for (long k = 0; k < (long)n; ++k) {
        if (types && types[k] != ORC_CELL_FLUID) continue;
        const double rho = U[k], mx = U[n + k], my = U[2 * n + k], E = U[3 * n + k];
        const double p = (g - 1) * (E - 0.5 * (mx * mx + my * my) / rho);
        const double a = sqrt(g * p / rho);
        const double u = mx / rho, v = my / rho;
        double w = (fabs(u) + a) / dx + (fabs(v) + a) / dy;
        if (!(w == w)) w = INFINITY; /* a blown-up cell: dt = 0, as the engine reports it */
        if (w > m) m = w;
    }
    return cfl / m;
}

/* Reference stencil tables, FourthOrderCS.h:28-42. */
static const double THETA_R[3][6] = {
    {71.0 / 1920, -141.0 / 128, 69.0 / 64, 1.0 / 192, -3.0 / 128, 3.0 / 640},
    {-3.0 / 640, 25.0 / 384, -75.0 / 64, 75.0 / 64, -25.0 / 384, 3.0 / 640},
    {-3.0 / 640, 3.0 / 128, -1.0 / 192, -69.0 / 64, 141.0 / 128, -71.0 / 1920}};
static const double THETA_C[5] = {1.0 / 12, -8.0 / 12, 0.0, 8.0 / 12, -1.0 / 12};
static const double ZETA_R[3][4] = {
    {5.0 / 16, 15.0 / 16, -15.0 / 16, 1.0 / 16},
    {-1.0 / 16, 9.0 / 16, 9.0 / 16, -1.0 / 16},
    {1.0 / 16, -5.0 / 16, 15.0 / 16, 5.0 / 16}};

/* Primitive (u, v, T) of cell (i, j) through the ghost rule; T = gamma Ma^2 p / rho
 * (EulerPhase.cpp:135-138). */
static inline void prim(const orc_config* c, const double* U, int i, int j, double* u, double* v, double* T) {
    const double rho = cval(c, U, 0, i, j), mx = cval(c, U, 1, i, j), my = cval(c, U, 2, i, j), E = cval(c, U, 3, i, j);
    const double p = pressure(c->gamma, rho, mx, my, E);
    *u = mx / rho;
    *v = my / rho;
    *T = c->gamma * (c->mach * c->mach) * p / rho;
}

/* Navier-Stokes terms (no reference counterpart; the reference computes but
 * never adds its viscous flux, Cell.cpp:128-133, Run.cpp:188).  Normal
 * derivative at the face from THETA_R[1] over 6 cells, cross derivative from
 * cell-centred THETA_C gradients interpolated with ZETA_R[1], face u, v from
 * ZETA_R[1]; sigma_11 = mu (4/3 u_x - 2/3 v_y), sigma_12 = mu (u_y + v_x),
 * heat flux k T_x with k = mu / ((gamma-1) Ma^2 Pr).  Adds (Fv_r - Fv_l)/dx +
 * (Gv_t - Gv_b)/dy to rhs of every cell. */
static void add_ns_terms(const orc_config* c, const double* U, double* rhs) {
    const int nx = c->nx, ny = c->ny;
    const size_t n = ncell(c);
    const double dx = c->lx / nx, dy = c->ly / ny, mu = c->mu;
    const double kT = mu / ((c->gamma - 1) * (c->mach * c->mach) * c->prandtl);
    const int W = 3;  /* primitive halo */
    const int px = nx + 2 * W, py = ny + 2 * W;
    double* P = (double*)malloc(sizeof(double) * 3 * (size_t)px * py);
    double* Gx = (double*)malloc(sizeof(double) * 3 * (size_t)px * py); /* d/dx of u,v,T */
    double* Gy = (double*)malloc(sizeof(double) * 3 * (size_t)px * py); /* d/dy of u,v,T */
    const size_t pn = (size_t)px * py;
#define PI(q, i, j) P[(size_t)(q) * pn + (size_t)((i) + W) * py + ((j) + W)]
#define GXI(q, i, j) Gx[(size_t)(q) * pn + (size_t)((i) + W) * py + ((j) + W)]
#define GYI(q, i, j) Gy[(size_t)(q) * pn + (size_t)((i) + W) * py + ((j) + W)]
#pragma omp parallel for num_threads(c->nthreads > 0 ? c->nthreads : omp_get_max_threads())
    for (int i = -W; i < nx + W; ++i)
        for (int j = -W; j < ny + W; ++j) {
            double u, v, T;
            /* corner ghosts take the x-side rule first, then the y-side rule */
            prim(c, U, i, j, &u, &v, &T);
            PI(0, i, j) = u;
            PI(1, i, j) = v;
            PI(2, i, j) = T;
        }
    /* d/dy at cells i = -2 .. nx+1 (x-face cross derivatives reach two cells
     * past the grid along x), d/dx at j = -2 .. ny+1 likewise. */
#pragma omp parallel for num_threads(c->nthreads > 0 ? c->nthreads : omp_get_max_threads())
    for (int i = -2; i < nx + 2; ++i)
        for (int j = 0; j < ny; ++j)
            for (int q = 0; q < 3; ++q) {
                double sy = 0.0;
                for (int m = 0; m < 5; ++m) sy += THETA_C[m] * PI(q, i, j - 2 + m);
                GYI(q, i, j) = sy / dy;
            }
#pragma omp parallel for num_threads(c->nthreads > 0 ? c->nthreads : omp_get_max_threads())
    for (int i = 0; i < nx; ++i)
        for (int j = -2; j < ny + 2; ++j)
            for (int q = 0; q < 3; ++q) {
                double sx = 0.0;
                for (int m = 0; m < 5; ++m) sx += THETA_C[m] * PI(q, i - 2 + m, j);
                GXI(q, i, j) = sx / dx;
            }
#pragma omp parallel for num_threads(c->nthreads > 0 ? c->nthreads : omp_get_max_threads())
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            double fv[4][3]; /* faces: left, right, bottom, top ; (mx, my, E) */
            for (int f = 0; f < 4; ++f) {
                const int dir = f >> 1;
                const int a_i = (f == 1) ? i + 1 : i, a_j = (f == 3) ? j + 1 : j; /* cell on the + side */
                double dn[3] = {0, 0, 0}, cr[3] = {0, 0, 0}, uf = 0.0, vf = 0.0;
                for (int q = 0; q < 3; ++q) {
                    double s = 0.0;
                    for (int k = 0; k < 6; ++k)
                        s += THETA_R[1][k] * (dir == 0 ? PI(q, a_i - 3 + k, a_j) : PI(q, a_i, a_j - 3 + k));
                    dn[q] = s / (dir == 0 ? dx : dy);
                    double t = 0.0;
                    for (int k = 0; k < 4; ++k)
                        t += ZETA_R[1][k] * (dir == 0 ? GYI(q, a_i - 2 + k, a_j) : GXI(q, a_i, a_j - 2 + k));
                    cr[q] = t;
                }
                for (int k = 0; k < 4; ++k) {
                    uf += ZETA_R[1][k] * (dir == 0 ? PI(0, a_i - 2 + k, a_j) : PI(0, a_i, a_j - 2 + k));
                    vf += ZETA_R[1][k] * (dir == 0 ? PI(1, a_i - 2 + k, a_j) : PI(1, a_i, a_j - 2 + k));
                }
                if (dir == 0) { /* u_x = dn0, v_x = dn1, T_x = dn2; u_y = cr0, v_y = cr1 */
                    const double s11 = mu * (4.0 / 3.0 * dn[0] - 2.0 / 3.0 * cr[1]);
                    const double s12 = mu * (cr[0] + dn[1]);
                    fv[f][0] = s11;
                    fv[f][1] = s12;
                    fv[f][2] = uf * s11 + vf * s12 + kT * dn[2];
                } else {        /* v_y = dn1, u_y = dn0, T_y = dn2; u_x = cr0, v_x = cr1 */
                    const double s22 = mu * (4.0 / 3.0 * dn[1] - 2.0 / 3.0 * cr[0]);
                    const double s21 = mu * (dn[0] + cr[1]);
                    fv[f][0] = s21;
                    fv[f][1] = s22;
                    fv[f][2] = uf * s21 + vf * s22 + kT * dn[2];
                }
            }
            const size_t k = (size_t)i * ny + j;
            for (int q = 0; q < 3; ++q)
                rhs[(size_t)(q + 1) * n + k] += (fv[1][q] - fv[0][q]) / dx + (fv[3][q] - fv[2][q]) / dy;
        }
#undef PI
#undef GXI
#undef GYI
    free(P);
    free(Gx);
    free(Gy);
}

/* rhs[v][i][j] = Cell::comRHS (Cell.cpp:110-126) for every cell, from all face
 * fluxes of the current state (faces ordered left, right, bottom, top, Cell.h:71). */
static void compute_rhs(const orc_config* c, const uint8_t* types, const double* U, double* rhs) {
    const int nx = c->nx, ny = c->ny;
    const size_t n = ncell(c);
    const double dx = c->lx / nx, dy = c->ly / ny;
    const size_t nfx = (size_t)(nx + 1) * ny, nfy = (size_t)nx * (ny + 1);
    double* FX = (double*)malloc(sizeof(double) * NV * nfx);
    double* FY = (double*)malloc(sizeof(double) * NV * nfy);
#pragma omp parallel for num_threads(c->nthreads > 0 ? c->nthreads : omp_get_max_threads())
    for (int a = 0; a <= nx; ++a)
        for (int j = 0; j < ny; ++j) {
            double s[6][NV], F[4];
            int lowo = 0;
            for (int k = 0; k < 6; ++k) {
                const int ii = face_slot(a, k, nx, c->bc[0] == ORC_BC_PERIODIC, c->bc[1] == ORC_BC_PERIODIC);
                for (int q = 0; q < NV; ++q) s[k][q] = cval(c, U, q, ii, j);
                if (c->positivity >= ORC_POS_BODY && types && ii >= 0 && ii < nx && types[(size_t)ii * ny + j]) lowo = 1;
            }
            face_flux(c, s, 0, F, lowo);
            for (int q = 0; q < NV; ++q) FX[(size_t)q * nfx + (size_t)a * ny + j] = F[q];
        }
#pragma omp parallel for num_threads(c->nthreads > 0 ? c->nthreads : omp_get_max_threads())
    for (int i = 0; i < nx; ++i)
        for (int a = 0; a <= ny; ++a) {
            double s[6][NV], F[4];
            int lowo = 0;
            for (int k = 0; k < 6; ++k) {
                const int jj = face_slot(a, k, ny, c->bc[2] == ORC_BC_PERIODIC, c->bc[3] == ORC_BC_PERIODIC);
                for (int q = 0; q < NV; ++q) s[k][q] = cval(c, U, q, i, jj);
                if (c->positivity >= ORC_POS_BODY && types && jj >= 0 && jj < ny && types[(size_t)i * ny + jj]) lowo = 1;
            }
            face_flux(c, s, 1, F, lowo);
            for (int q = 0; q < NV; ++q) FY[(size_t)q * nfy + (size_t)i * (ny + 1) + a] = F[q];
        }
#pragma omp parallel for num_threads(c->nthreads > 0 ? c->nthreads : omp_get_max_threads())
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            const size_t k = (size_t)i * ny + j;
            for (int q = 0; q < NV; ++q) {
                const double f0 = FX[(size_t)q * nfx + (size_t)i * ny + j];
                const double f1 = FX[(size_t)q * nfx + (size_t)(i + 1) * ny + j];
                const double f2 = FY[(size_t)q * nfy + (size_t)i * (ny + 1) + j];
                const double f3 = FY[(size_t)q * nfy + (size_t)i * (ny + 1) + j + 1];
                rhs[(size_t)q * n + k] = -(f1 - f0) / dx - (f3 - f2) / dy;
            }
        }
    free(FX);
    free(FY);
    if (c->viscous) add_ns_terms(c, U, rhs);
}

/* TVD2rdRK::advance (TVD2rdRK.cpp:3-31, coef TVD2rdRK.h:16-19) and
 * TVD3rdRK::advance (TVD3rdRK.cpp:3-48, coef TVD3rdRK.h:14-18; stage 2 uses the
 * saved stage-1 input U1).  ORC_RK_SSP3 stage 2 uses the current state instead
 * (Shu-Osher; no reference counterpart). */
/* ORC_POS_FLOOR (no reference counterpart): a fluid cell whose new state has
 * rho <= ORC_RHO_FLOOR (or a NaN) becomes the floor state at rest (rho and p at
 * their floors, no momentum: keeping the velocity of a near-zero density would
 * blow it up); one with p <= ORC_P_FLOOR gets E raised so that p is at its
 * floor, momentum kept. */
static void floor_cell(const orc_config* c, double* U, size_t n, size_t k) {
    double rho = U[k], mx = U[n + k], my = U[2 * n + k], E = U[3 * n + k];
    if (!(rho > ORC_RHO_FLOOR) || !(mx == mx) || !(my == my) || !(E == E)) {
        rho = ORC_RHO_FLOOR;
        mx = my = 0.0;
        E = ORC_P_FLOOR / (c->gamma - 1);
    }
    const double ke = 0.5 * (mx * mx + my * my) / rho;
    if (!((c->gamma - 1) * (E - ke) > ORC_P_FLOOR)) E = ORC_P_FLOOR / (c->gamma - 1) + ke;
    U[k] = rho;
    U[n + k] = mx;
    U[2 * n + k] = my;
    U[3 * n + k] = E;
}

int orc_stage(const orc_config* c, const uint8_t* types, const orc_ib* ib, int stage,
              double dt, double* U, double* U0, double* U1, double* rhs_out) {
    const size_t n = ncell(c);
    orc_ib_fill(c, ib, U);
    double* R = rhs_out ? rhs_out : (double*)malloc(sizeof(double) * NV * n);
    compute_rhs(c, types, U, R);
    const int tvd2 = c->rk == ORC_RK_TVD2;
#pragma omp parallel for num_threads(c->nthreads > 0 ? c->nthreads : omp_get_max_threads())
    for (long k = 0; k < (long)n; ++k) {
        if (types && types[k] != ORC_CELL_FLUID) continue;
        for (int q = 0; q < NV; ++q) {
            const size_t e = (size_t)q * n + (size_t)k;
            const double r = R[e];
            if (tvd2) {
                if (stage == 0) {
                    U0[e] = U[e];
                    U[e] = 1.0 * U0[e] + 1.0 * dt * r;
                } else {
                    U[e] = 0.5 * U0[e] + 0.5 * U[e] + 0.5 * dt * r;
                }
            } else if (stage == 0) {
                U0[e] = U[e];
                U[e] = 1.0 * U0[e] + 1.0 * dt * r;
            } else if (stage == 1) {
                U1[e] = U[e];
                U[e] = 0.75 * U0[e] + 0.25 * U1[e] + 0.25 * dt * r;
            } else if (c->rk == ORC_RK_TVD3_REFERENCE) {
                U[e] = (1.0 / 3.0) * U0[e] + (2.0 / 3.0) * U1[e] + (2.0 / 3.0) * dt * r;
            } else {
                U[e] = (1.0 / 3.0) * U0[e] + (2.0 / 3.0) * U[e] + (2.0 / 3.0) * dt * r;
            }
        }
        if (c->positivity >= ORC_POS_FLOOR) floor_cell(c, U, n, (size_t)k);
    }
    if (!rhs_out) free(R);
    return 0;
}

static int stage_of(const orc_config* c, int counter) {
    if (c->rk == ORC_RK_TVD2) return (counter % 2 == 0) ? 1 : 0;
    return (counter % 3 == 0) ? 2 : (counter % 3 == 1) ? 0 : 1;
}

int orc_run(const orc_config* c, const uint8_t* types, const orc_ib* ib, double* U,
            int first, int count, double dt, double cfl, double* dt_log) {
    const size_t n = ncell(c);
    double* U0 = (double*)calloc(NV * n, sizeof(double));
    double* U1 = (double*)calloc(NV * n, sizeof(double));
    if (!U0 || !U1) { free(U0); free(U1); return -1; }
    for (int k = first; k < first + count; ++k) {
        const int st = stage_of(c, k);
        if (cfl > 0.0 && st == 0) dt = orc_cfl_dt(c, types, U, cfl);
        if (dt_log) dt_log[k - first] = dt;
        orc_stage(c, types, ib, st, dt, U, U0, U1, NULL);
    }
    free(U0);
    free(U1);
    return 0;
}

/* ForthOrderCS::comprimitivederivativeForcell + comviscousfluxForcellinterface
 * (FourthOrderCS.cpp:16-151) with their constants: dx = 0.002 in the face
 * routine (:32), mu = c->mu, sigma_11 = 2 mu (2/3) u_x, sigma_12 = mu (u_y + v_y)
 * for X (and the mirror for Y), q = -mu/((gamma-1) Ma^2) T_n, combination
 * (-1/24, 26/24, -1/24) of the three point values (:106-108).  Ghost cells carry
 * zero gradients (the reference never computes theirs). */
int orc_viscous_reference(const orc_config* c, const double* U, double* grad, double* fvx, double* fvy) {
    const int nx = c->nx, ny = c->ny;
    const size_t n = ncell(c);
    const double dx = c->lx / nx, dy = c->ly / ny;
    const double mu = c->mu, g = c->gamma, ma2 = c->mach * c->mach;
    /* cell gradients */
#pragma omp parallel for num_threads(c->nthreads > 0 ? c->nthreads : omp_get_max_threads())
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            for (int dir = 0; dir < 2; ++dir) {
                double su = 0.0, sv = 0.0, sT = 0.0;
                for (int m = 0; m < 5; ++m) {
                    const int ii = dir == 0 ? i - 2 + m : i, jj = dir == 0 ? j : j - 2 + m;
                    const double rho = cval(c, U, 0, ii, jj), mx = cval(c, U, 1, ii, jj), my = cval(c, U, 2, ii, jj), E = cval(c, U, 3, ii, jj);
                    const double p = pressure(g, rho, mx, my, E);
                    const double T = g * ma2 * p / rho;
                    su += THETA_C[m] * (mx / rho);
                    sv += THETA_C[m] * (my / rho);
                    sT += THETA_C[m] * T;
                }
                const double h = dir == 0 ? dx : dy;
                const size_t k = (size_t)i * ny + j;
                grad[(size_t)(0 + dir) * n + k] = su / h;
                grad[(size_t)(2 + dir) * n + k] = sv / h;
                grad[(size_t)(4 + dir) * n + k] = sT / h;
            }
        }
    const double hq = 0.002;
    for (int dir = 0; dir < 2; ++dir) {
        const int fa = dir == 0 ? nx + 1 : nx, fb = dir == 0 ? ny : ny + 1;
        const size_t nf = (size_t)fa * fb;
        double* out = dir == 0 ? fvx : fvy;
#pragma omp parallel for num_threads(c->nthreads > 0 ? c->nthreads : omp_get_max_threads())
        for (int a = 0; a < fa; ++a)
            for (int b = 0; b < fb; ++b) {
                double u[6], v[6], T[6], ud[4], vd[4], Td[4], u4[4], v4[4];
                for (int k = 0; k < 6; ++k) {
                    const int ii = dir == 0 ? face_slot(a, k, nx, c->bc[0] == ORC_BC_PERIODIC, c->bc[1] == ORC_BC_PERIODIC) : a;
                    const int jj = dir == 0 ? b : face_slot(b, k, ny, c->bc[2] == ORC_BC_PERIODIC, c->bc[3] == ORC_BC_PERIODIC);
                    const double rho = cval(c, U, 0, ii, jj), mx = cval(c, U, 1, ii, jj), my = cval(c, U, 2, ii, jj), E = cval(c, U, 3, ii, jj);
                    const double p = pressure(g, rho, mx, my, E);
                    u[k] = mx / rho;
                    v[k] = my / rho;
                    T[k] = g * ma2 * p / rho;
                    if (k >= 1 && k <= 4) {
                        const int cross = 1 - dir;
                        if (is_phys_ghost(c, ii, jj)) {
                            ud[k - 1] = 0.0; vd[k - 1] = 0.0; Td[k - 1] = 0.0;
                        } else {
                            const size_t e = (size_t)ii * ny + jj;
                            ud[k - 1] = grad[(size_t)(0 + cross) * n + e];
                            vd[k - 1] = grad[(size_t)(2 + cross) * n + e];
                            Td[k - 1] = grad[(size_t)(4 + cross) * n + e];
                        }
                        u4[k - 1] = u[k];
                        v4[k - 1] = v[k];
                    }
                }
                double vMu[3], vMv[3], vE[3];
                for (int r = 0; r < 3; ++r) {
                    double dum = 0.0, dvm = 0.0, dTm = 0.0, duc = 0.0, dvc = 0.0, dTc = 0.0, uc = 0.0, vc = 0.0;
                    for (int k = 0; k < 6; ++k) { dum += THETA_R[r][k] * u[k]; }
                    for (int k = 0; k < 6; ++k) { dvm += THETA_R[r][k] * v[k]; }
                    for (int k = 0; k < 6; ++k) { dTm += THETA_R[r][k] * T[k]; }
                    dum = dum / hq;
                    dvm = dvm / hq;
                    dTm = dTm / hq;
                    for (int k = 0; k < 4; ++k) duc += ZETA_R[r][k] * ud[k];
                    for (int k = 0; k < 4; ++k) dvc += ZETA_R[r][k] * vd[k];
                    for (int k = 0; k < 4; ++k) dTc += ZETA_R[r][k] * Td[k];
                    for (int k = 0; k < 4; ++k) uc += ZETA_R[r][k] * u4[k];
                    for (int k = 0; k < 4; ++k) vc += ZETA_R[r][k] * v4[k];
                    (void)dTc;
                    if (dir == 0) {
                        double s11 = 2 * mu * (2.0 / 3.0) * dum;
                        double s12 = mu * (duc + dvc);
                        double q1 = (-mu / ((g - 1) * ma2)) * dTm;
                        vMu[r] = s11;
                        vMv[r] = s12;
                        vE[r] = s11 * uc + s12 * vc + q1;
                    } else {
                        double s22 = 2 * mu * (2.0 / 3.0) * dvm;
                        double s21 = mu * (duc + dvc);
                        double q2 = (-mu / ((g - 1) * ma2)) * dTm;
                        vMu[r] = s21;
                        vMv[r] = s22;
                        vE[r] = s21 * uc + s22 * vc + q2;
                    }
                }
                const size_t e = (size_t)a * fb + b;
                out[e] = 0.0;
                out[nf + e] = (-1.0 / 24.0) * vMu[0] + (26.0 / 24.0) * vMu[1] + (-1.0 / 24.0) * vMu[2];
                out[2 * nf + e] = (-1.0 / 24.0) * vMv[0] + (26.0 / 24.0) * vMv[1] + (-1.0 / 24.0) * vMv[2];
                out[3 * nf + e] = (-1.0 / 24.0) * vE[0] + (26.0 / 24.0) * vE[1] + (-1.0 / 24.0) * vE[2];
            }
    }
    return 0;
}
