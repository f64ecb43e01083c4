// The reference's Poisson solver object (src/poisson.cuh:18-119 of the reference): solve
// (delta_eta_eta,mapped - k^2) psi-hat = -omega-hat for every streamwise wavenumber, with
// Dirichlet psi_bot / psi_top on kx = 0 (the reference's Dirichlet enforcement). Same members a
// driver uses: the constructor, enable_mapped, solve, set_profile / profile_reset / profile_get.
// The work is this library's: a real row transform of Nx/2 complex points (no cuFFT), the
// segmented tridiagonal solve and the inverse transform, on a workspace owned by the object. Each
// object holds an nse2d solver context of its grid.
#pragma once
#include "grid.hpp"

typedef struct CUstream_st* cudaStream_t;

struct Poisson2D_Z2Z {
    int Nx, Ny;
    bool profile{false};
    float acc_fft_ms{0.0f};
    float acc_tridiag_ms{0.0f};
    bool mapped{false};
    const Real* d_a_node{nullptr};
    const Real* d_a_edge{nullptr};
    Real inv_deta2{0.0};

    // uniform-grid solver (the reference's fallback coefficients from the physical dy)
    explicit Poisson2D_Z2Z(const Grid& G, cudaStream_t s = 0);
    ~Poisson2D_Z2Z();
    Poisson2D_Z2Z(const Poisson2D_Z2Z&) = delete;
    Poisson2D_Z2Z& operator=(const Poisson2D_Z2Z&) = delete;
    inline void set_profile(bool on) { profile = on; }
    inline void profile_reset() { acc_fft_ms = 0.0f; acc_tridiag_ms = 0.0f; }
    inline void profile_get(float& fft_ms, float& tridiag_ms) { fft_ms = acc_fft_ms; tridiag_ms = acc_tridiag_ms; }
    // the mapped operator from device a_node [Ny] and a_edge [Ny-1] (copied at this call)
    void enable_mapped(const Real* a_node, const Real* a_edge, Real inv_deta, cudaStream_t s = 0);
    // psi from omega (device [Ny][Nx], 16-byte aligned); dy is unused, as in the reference
    void solve(const Real* d_omega, Real* d_psi, Real dy, Real psi_bot, Real psi_top, cudaStream_t s = 0);

  private:
    struct Impl;
    Impl* impl_{nullptr};
    double Lx_{0}, h_{1};
};
