// The reference's diagnostic launchers with C++ linkage (src/diag.cuh:12-113 of the reference)
// and its Spectra1D accumulator (src/diag.cuh:123-191). Same names, arguments and outputs: the
// sums are device scalars (zeroed by the launcher, then accumulated by atomic adds of per-CTA
// partials, as in the reference, so they agree with it to round-off); the row moments and the wall
// means are written per row / per wall. No static scratch: the Laplacian of
// launch_enstrophy_diss_balance_mapped is evaluated in the reduction, and the maxima of
// launch_max_uv_from_psi_mapped are combined by atomic maxima in the caller's three scalars.
#pragma once
#include <string>

#include "ops.hpp"

void launch_enstrophy_diss_mapped(const Real* omg, int Nx, int Ny, Real inv_dx, Real inv_deta, const Real* d_a_node,
                                  const Real* d_w_node, Real* d_sum_w2, Real* d_sum_gw2, cudaStream_t s = 0);
void launch_enstrophy_diss_mapped_full(const Real* omg, int Nx, int Ny, Real inv_dx, Real inv_deta,
                                       const Real* d_a_node, const Real* d_w_node, Real* d_sum_w2_full,
                                       Real* d_sum_gw2_full, cudaStream_t s = 0);
void launch_enstrophy_sbp_mapped(const Real* omg, int Nx, int Ny, Real inv_dx, Real inv_deta, const Real* d_a_edge,
                                 const Real* d_wt_node, Real* d_sum_eta_h, Real* d_sum_phi_h, cudaStream_t s = 0);
void launch_kinetic_energy_mapped(const Real* psi, int Nx, int Ny, Real inv_dx, Real inv_deta, const Real* d_a_node,
                                  const Real* d_w_node, Real* d_sum, cudaStream_t s = 0);
void launch_energy_dissipation_mapped(const Real* d_psi, const Real* d_omega, int Nx, int Ny, Real inv_dx,
                                      Real inv_deta, const Real* d_a_node, const Real* d_a_edge, const Real* d_w_node,
                                      Real* d_sum_eps, cudaStream_t s);
void launch_power_input_mapped(const Real* psi, int Nx, int Ny, Real inv_deta, Real h, Real F0, int nforce,
                               const Real* d_a_node, const Real* d_y_node, const Real* d_w_node, Real* d_sum,
                               cudaStream_t s = 0);
void launch_enstrophy_input_mapped_full(const Real* omega, int Nx, int Ny, Real h, Real F0, int nforce,
                                        const Real* d_y_node, const Real* d_w_node, Real* d_sum, cudaStream_t s = 0);
void launch_enstrophy_input_mapped(const Real* omega, int Nx, int Ny, Real h, Real F0, int nforce,
                                   const Real* d_y_node, const Real* d_w_node, Real* d_sum, cudaStream_t s = 0);
void launch_row_moments_from_psi_mapped(const Real* psi, int Nx, int Ny, Real inv_dx, Real inv_deta,
                                        const Real* d_a_node, Real* su, Real* sv, Real* su2, Real* sv2, Real* suv,
                                        cudaStream_t s = 0);
void launch_mean_wall_omega(const Real* omega, int Nx, int Ny, Real* d_mean_bot, Real* d_mean_top, cudaStream_t s = 0);
void launch_mean_wall_omega_omegay_mapped(const Real* omega, int Nx, int Ny, Real inv_deta, const Real* d_a_node,
                                          Real* d_mean_bot, Real* d_mean_top, cudaStream_t s = 0);
void launch_enstrophy_diss_balance_mapped(const Real* d_omega, int Nx, int Ny, Real inv_dx2, Real inv_deta2,
                                          const Real* d_a_node, const Real* d_a_edge, const Real* d_w_node,
                                          Real* d_sum_w2, Real* d_sum_eta, cudaStream_t s = 0);
void launch_omega_rhs_balance_mapped(const Real* d_omega, const Real* d_rhs, int Nx, int Ny, const Real* d_w_node,
                                     Real* d_sum_omega_rhs, cudaStream_t stream = 0);
void launch_max_uv_from_psi_mapped(const Real* d_psi, int Nx, int Ny, Real inv_dx, Real inv_deta,
                                   const Real* d_a_node, Real* d_umax, Real* d_vmax, Real* d_vmaxm,
                                   cudaStream_t stream = 0);

// Time-averaged 1-D energy spectra E_u(kx), E_v(kx) (src/diag.cuh:123-191), with this library's
// real row transform instead of cuFFT D2Z: init(G), accumulate(d_u, d_v) (device [Ny][Nx]),
// write_csv(path) with the reference's header and format. Owns its workspace.
struct Spectra1D {
    int Nx{0}, Ny{0}, Nxc{0};
    int samples{0};
    void* impl{nullptr};
    void init(const Grid& G);
    void accumulate(Real* d_u, Real* d_v);
    void write_csv(const std::string& path);
    ~Spectra1D();
};
