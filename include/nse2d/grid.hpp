// The reference's C++ grid and parameter types, for code written against the reference's
// driver-side API (src/common.cuh:42-114 of the reference). Field names, types and defaults are
// the reference's, so that a driver that fills them builds unchanged against libnse2d_b200.so.
// Host-side C++ (std::vector / std::string members); not part of the C ABI.
#pragma once
#include <string>
#include <vector>

#ifndef NSE2D_HD
#if defined(__CUDACC__)
#define NSE2D_HD __host__ __device__
#else
#define NSE2D_HD
#endif
#endif

using Real = double;

// src/common.cuh:42-57
struct Grid {
    int Nx{1024};
    int Ny{1025};
    Real Lx{12.566370612};
    Real h{1.0};
    std::vector<Real> y;        // Ny
    std::vector<Real> a_node;   // Ny   (a_j = 1 / y_eta at nodes)
    std::vector<Real> a_edge;   // Ny-1 (a at j+1/2)
    std::vector<Real> dy_edge;  // Ny-1 (y_{j+1} - y_j)
    std::vector<Real> w_node;   // Ny   (trapezoid weights)
    NSE2D_HD inline Real dx() const { return Lx / (Real)Nx; }
    NSE2D_HD inline Real dy() const { return (2.0 * h) / (Real)(Ny - 1); }
    NSE2D_HD inline Real Ly() const { return 2.0 * h; }
};

// src/common.cuh:58-114
struct Params {
    Real Ub{1.0};
    std::string stretch{"none"};       // "none" | "tanh" | "table"
    std::string ytable{"none"};        // HDF5 file with dataset /y for stretch "table"
    Real beta{0.0};
    std::string integrator{"imex3"};   // parsed, unused: the time step is always SSPRK(3,3)
    Real Reb{10000.0};
    Real nu_override{-1};              // < 0: nu = 2 h Ub / Reb
    Real nu(Real h) const { return (nu_override >= 0 ? nu_override : (2.0 * h * Ub) / Reb); }
    Real dt_init{1e-3};
    Real dt_max{1e-2};
    Real cfl{0.5};
    Real cvisc{0.5};
    bool adapt{true};
    Real t_end{200.0};
    Real F0{0.0};
    int nforce{1};
    Real lin_drag{0.0};
    std::string progress_path{};
    bool resume{false};
    Real t0{0.0};
    std::string init{"load"};          // laminar | rand | ts | mix | load | diffusion | diffusion2d | mms
    Real amp{0.5};
    Real alpha{1.2};
    int my{1};
    Real phase{0.0};
    Real rand_amp{0.0};
    unsigned long long seed{123456789ULL};
    std::string load_path{""};
    bool load_use_psi{false};
    std::string snap_fields{"all"};    // "all" | "omega" | "omega_psi"
    int rand_nx{48};
    int rand_mymax{8};
    Real rand_k0{0.0};
    Real rand_sigma{0.6};
    Real rand_amp_abs{0.0};
    bool mms{false};
    Real mms_A0{1e-3};
    Real mms_eps{0.1};
    Real mms_Om{1.0};
    int mms_kx{1};
    bool closure_diag{false};
};

// Wall-normal metrics (src/grid.cu:7-94): uniform, tanh (beta, 2.5 when beta <= 0) or the table
// of dataset /y of the HDF5 file P.ytable. Throws std::runtime_error on a bad stretch or table.
void build_y_metrics(const Grid& Gin, const Params& P, Grid& Gout);
