// The reference's spatial-operator launchers with C++ linkage (src/ops.cuh:12-81 of the
// reference): same names, argument order and meaning, defaults and stream semantics
// (asynchronous on s; every pointer caller-owned device memory; metrics [Ny] / [Ny-1]). Like the
// reference, a CUDA error prints and aborts, unless nse2d_set_abort_on_error(0) (nse2d.h) keeps it
// for nse2d_last_error(). The wall closure follows nse2d_testapi_set_free_slip (no-slip Thom by
// default; the reference fixes it with FREE_SLIP_WALLS at compile time).
#pragma once
#include <cstddef>

#include "grid.hpp"

typedef struct CUstream_st* cudaStream_t;

void launch_uv_from_psi_mapped(const Real* psi, Real* u, Real* v, int Nx, int Ny, Real inv_dx, Real inv_deta,
                               const Real* d_a_node, cudaStream_t s = 0);
void launch_omega_from_psi_interior_mapped(Real* w, const Real* psi, int Nx, int Ny, Real inv_dx2, Real inv_deta2,
                                           const Real* d_a_node, const Real* d_a_edge, cudaStream_t s = 0);
void launch_thom_wall_vorticity_mapped(Real* w, const Real* psi, int Nx, int Ny, const Real* d_dy_edge, Real psi_bot,
                                       Real psi_top, cudaStream_t s = 0);
void launch_arakawa_J_mapped(const Real* psi, const Real* omg, Real* J, int Nx, int Ny, Real inv_dx, Real inv_deta,
                             const Real* d_a_node, cudaStream_t s = 0);
void launch_laplacian_fd_mapped(const Real* d_q, Real* d_out, int Nx, int Ny, Real inv_dx2, Real inv_deta2,
                                const Real* d_a_node, const Real* d_a_edge, cudaStream_t s = 0);
void launch_rhs_mapped(const Real* J, const Real* lap, const Real* omg, Real* rhs, int Nx, int Ny, Real nu, Real F0,
                       int nforce, Real h, Real lin_drag, const Real* d_y_node, cudaStream_t s = 0);
void launch_mms_add_forcing(Real* d_rhs, int Nx, int Ny, Real Lx, Real h, Real t, Real nu, Real r, Real A0, Real eps,
                            Real Om, int kx_mode, const Real* d_y_node, cudaStream_t s = 0);
void launch_axpy(Real* y, const Real* x, const Real* r, Real dt, size_t N, cudaStream_t s = 0);
void launch_ssprk2(Real* w2, const Real* w, const Real* w1, const Real* rhs, Real dt, size_t N, cudaStream_t s = 0);
void launch_ssprk3(Real* wnp1, const Real* w, const Real* w2, const Real* rhs, Real dt, size_t N, cudaStream_t s = 0);
