/*
 * CPU FP64 oracle for the nse2d channel time step. TEST INFRASTRUCTURE ONLY.
 *
 * This library is the checker: a plain restatement, in C++17 with OpenMP, of the
 * reference's FP64 algorithm (xupingxie/nse2d-channel-gpu, files cited per function
 * in nse2d_oracle.cpp). Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline / reference arm may load it. The product (the CUDA library under
 * nse2d-channel-gpu_b200/) never links or calls it.
 *
 * Parity pin: the oracle driver reproduces the deterministic t = 0 rows and the
 * early rows of the reference's committed test outputs
 * (tests/reference/output/<case>/diagnostics.csv) and the values of
 * tests/reference/reference.json; see tests/golden/ and tests/test_oracle_golden.py.
 *
 * Arrays are row-major [Ny][Nx] (x fastest), FP64, host memory.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- run configuration: the reference's Grid + Params (src/common.cuh:42-114) ---- */
typedef struct or_config {
    int    Nx, Ny;
    double Lx, h;
    int    stretch;        /* 0 = none/uniform, 1 = tanh */
    double beta;
    double Ub, Reb, nu_override;
    double dt_init, dt_max, cfl, cvisc;
    int    adapt;
    double t_end;
    double F0;
    int    nforce;
    double lin_drag;
    int    free_slip;      /* compile-time FREE_SLIP_WALLS in the reference */
    int    mms;
    double mms_A0, mms_eps, mms_Om;
    int    mms_kx;
    int    closure_diag;
} or_config;

/* ---- grid metrics, src/grid.cu:7-94 ---- */
int or_grid_metrics(int Nx, int Ny, double Lx, double h, int stretch, double beta,
                    double* y, double* a_node, double* a_edge, double* dy_edge, double* w_node);

/* ---- operators, src/ops.cu ---- */
void or_uv_from_psi(const double* psi, double* u, double* v, int Nx, int Ny,
                    double inv_dx, double inv_deta, const double* a_node);
void or_omega_from_psi_interior(double* w, const double* psi, int Nx, int Ny,
                                double inv_dx2, double inv_deta2,
                                const double* a_node, const double* a_edge);
void or_thom(double* w, const double* psi, int Nx, int Ny, const double* dy_edge,
             double psi_bot, double psi_top, int free_slip);
void or_arakawa(const double* psi, const double* w, double* J, int Nx, int Ny,
                double inv_dx, double inv_deta, const double* a_node);
void or_adv_from_uv(const double* u, const double* v, const double* w, double* J, int Nx, int Ny,
                    double inv_dx, double inv_deta, const double* a_node);
void or_adv_flux(const double* u, const double* v, const double* w, double* J, int Nx, int Ny,
                 double inv_dx, double inv_deta, const double* a_node);
void or_arakawa_split(const double* psi, const double* w, double* J1, double* J2, double* J3,
                      double* Jadv, int Nx, int Ny, double inv_dx, double inv_deta,
                      const double* a_node);
void or_laplacian(const double* q, double* out, int Nx, int Ny, double inv_dx2, double inv_deta2,
                  const double* a_node, const double* a_edge);
void or_rhs(const double* J, const double* lap, const double* w, double* rhs, int Nx, int Ny,
            double nu, double F0, int nforce, double h, double lin_drag, const double* y);
void or_mms_add(double* rhs, int Nx, int Ny, double Lx, double h, double t, double nu, double r,
                double A0, double eps, double Om, int kx_mode, const double* y);
void or_axpy(double* out, const double* x, const double* r, double dt, int64_t N);
void or_ssprk2(double* w2, const double* w, const double* w1, const double* r, double dt, int64_t N);
void or_ssprk3(double* wn, const double* w, const double* w2, const double* r, double dt, int64_t N);

/* ---- Poisson solve, src/poisson.cu:16-133 and src/poisson.cuh:83-118 ---- */
void or_poisson_solve(const double* w, double* psi, int Nx, int Ny, double Lx,
                      const double* a_node, const double* a_edge, double inv_deta,
                      double psi_bot, double psi_top);
/* the elimination table cp[k][r] of the reference, k = 0..Nx-1, r = 0..Ny-3 */
void or_poisson_cp(double* cp, int Nx, int Ny, double Lx, const double* a_node,
                   const double* a_edge, double inv_deta);
/* forward half spectrum (unnormalised, e^{-i}) of each row: out[j][k], k = 0..Nx/2 (re,im) */
void or_rfft_rows(const double* in, double* out, int Nx, int Ny);

/* ---- reductions, src/diag.cu ---- */
void or_max_uv(const double* psi, int Nx, int Ny, double inv_dx, double inv_deta,
               const double* a_node, double out3[3]);
/* all diagnostics.csv reductions at one state; see nse2d_oracle.cpp for the list */
void or_diag_sums(const double* psi, const double* w, const double* rhs, const double* J,
                  int Nx, int Ny, double inv_dx, double inv_deta, double h, double F0, int nforce,
                  const double* a_node, const double* a_edge, const double* y,
                  const double* w_node, double* out /* OR_NSUM */);
enum { OR_S_K = 0, OR_S_W2, OR_S_GW2, OR_S_WWY_BOT, OR_S_WWY_TOP, OR_S_WRHS, OR_S_PIN, OR_S_EPS,
       OR_S_POM, OR_S_MOB, OR_S_MOT,
       /* closure_diag sums (need rhs and J at the same state) */
       OR_S_W2_INT, OR_S_GW2_INT, OR_S_T2_D, OR_S_T2_J, OR_S_T2_W2, OR_S_T2_G2, OR_S_T2_P,
       OR_S_T2_ETA, OR_S_T2_PHI, OR_S_WALL_WRHS,
       OR_NSUM };
void or_row_moments(const double* psi, int Nx, int Ny, double inv_dx, double inv_deta,
                    const double* a_node, double* su, double* sv, double* su2, double* sv2,
                    double* suv);

/* ---- whole solver (the time loop of src/main.cu:434-551) ---- */
typedef struct or_solver or_solver;
or_solver* or_create(const or_config* cfg);
void   or_destroy(or_solver* s);
int    or_nx(const or_solver* s);
int    or_ny(const or_solver* s);
double or_nu(const or_solver* s);
/* set omega (full field incl. walls), then initial Poisson solve + Thom (main.cu:210-213) */
void   or_set_omega(or_solver* s, const double* w);
void   or_get_fields(const or_solver* s, double* w, double* psi);
void   or_set_fields(or_solver* s, const double* w, const double* psi);
const double* or_metric(const or_solver* s, int which /* 0 y,1 a_node,2 a_edge,3 dy_edge,4 w_node */);
/* adaptive dt from max|u|,|v| (main.cu:439-464); returns dt; fills umax/vmax/vmaxm */
double or_adapt_dt(or_solver* s, double* umax3);
/* one SSPRK(3,3) step of size dt at time t (main.cu:482-538) */
void   or_step(or_solver* s, double t, double dt);
/* diagnostics row values (the 19 + 13 columns of main.cu:681-687, minus step/t/dt) */
void   or_diag_row(or_solver* s, double t, int t0_row, double* out32);
double or_jwall(const or_solver* s, int stage);
void   or_set_threads(int n);
int    or_get_threads(void);

#ifdef __cplusplus
}
#endif
