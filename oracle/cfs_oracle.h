/* Test infrastructure (oracle only): CPU restatement, in plain C, of the
 * reference solver's per-stage hot path, plus the variants the reference cannot
 * express (periodic sides, Davis HLL, Shu-Osher RK3, bilinear/slip IB, CFL dt,
 * Navier-Stokes terms).  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU baseline load it, as the checker.  Built by oracle/Makefile.
 *
 * State layout: U[v][i][j], v = (rho, m_x, m_y, E), i = x index (outer),
 * j = y index (inner), the cells[i][j] / Output.cpp:60 order of the reference.
 */
#ifndef CFS_ORACLE_H
#define CFS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_RK_TVD2 = 0, ORC_RK_TVD3_REFERENCE = 1, ORC_RK_SSP3 = 2 };
enum { ORC_HLL_REFERENCE = 0, ORC_HLL_DAVIS = 1 };
enum { ORC_BC_NEUMANN = 0, ORC_BC_DIRICHLET = 1, ORC_BC_PERIODIC = 2 };
enum { ORC_CELL_FLUID = 0, ORC_CELL_SOLID = 1, ORC_CELL_GHOST = 2 };
enum { ORC_IB_REFERENCE = 0, ORC_IB_BILINEAR_SLIP = 1 };
enum { ORC_POS_OFF = 0, ORC_POS_FACE = 1, ORC_POS_BODY = 2, ORC_POS_FLOOR = 3 };
#define ORC_RHO_FLOOR 1e-6
#define ORC_P_FLOOR 1e-6

typedef struct {
    int nx, ny;
    double lx, ly;
    double gamma;
    double weno_eps;
    int rk;
    int hll;
    int bc[4];            /* left, right, bottom, top */
    double bc_U[4][4];    /* conserved ghost state of a Dirichlet side */
    int viscous;          /* 0 off, 1 Navier-Stokes terms added to the RHS */
    double mu, prandtl, mach;
    int nthreads;         /* 0 = OpenMP default */
    int positivity;       /* ORC_POS_* (face-state fallbacks, see face_flux) */
} orc_config;

typedef struct {
    int n;
    const int32_t* cell;   /* [n]  i*ny + j of each immersed-ghost cell */
    const int32_t* donor;  /* [4n] i*ny + j of its four fluid donors */
    const double* image;   /* [2n] image point (x, y) */
    const double* normal;  /* [2n] unit wall normal, used by ORC_IB_BILINEAR_SLIP */
    int mode;
    const uint8_t* types;  /* [nx*ny] cell types, used by ORC_IB_BILINEAR_SLIP (NULL: all fluid) */
} orc_ib;

/* One RK stage, in the order of one Run::solver iteration (Run.cpp:153-203):
 * immersed-ghost fill, interface reconstruction + flux, RHS, RK update of fluid
 * cells.  stage = 0, 1, 2 (already mapped from the loop counter as
 * TVD2rdRK.cpp:11 / TVD3rdRK.cpp:15 do).  U0 and U1 hold the stage copies the
 * reference keeps in TVD2rdRK::m_Phase / TVD3rdRK::m_Phase0,m_Phase1.
 * rhs (optional) receives R = -(dF/dx + dG/dy) of every fluid cell. */
int orc_stage(const orc_config* c, const uint8_t* types, const orc_ib* ib, int stage,
              double dt, double* U, double* U0, double* U1, double* rhs);

/* Runs loop iterations first..first+count-1 of the reference's counter.
 * cfl > 0 recomputes dt with orc_cfl_dt at the first stage of every step. */
int orc_run(const orc_config* c, const uint8_t* types, const orc_ib* ib, double* U,
            int first, int count, double dt, double cfl, double* dt_log);

/* CFL step: cfl / max over fluid cells of (|u|+a)/dx + (|v|+a)/dy. */
double orc_cfl_dt(const orc_config* c, const uint8_t* types, const double* U, double cfl);

/* Immersed-ghost fill alone (Cell::comImmersedGhostPhase, Cell.cpp:172-181). */
int orc_ib_fill(const orc_config* c, const orc_ib* ib, double* U);

/* Unit-level pieces, for kernel tests. */
double orc_weno5(const double v[5], double eps);
int orc_hll(const orc_config* c, const double L[4], const double R[4], int dir, double F[4]);

/* The reference's viscous routines (FourthOrderCS.cpp:16-142) on a grid state,
 * with temperature T = gamma Ma^2 p / rho and zero gradients on the physical
 * ghost cells, as ref_harness's ref_viscous sets them up.  Neumann/Dirichlet
 * sides only.  grad [6][nx][ny]; fvx [4][nx+1][ny]; fvy [4][nx][ny+1]. */
int orc_viscous_reference(const orc_config* c, const double* U, double* grad, double* fvx, double* fvy);

#ifdef __cplusplus
}
#endif
#endif
