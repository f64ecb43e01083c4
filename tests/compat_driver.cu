// TEST INFRASTRUCTURE: a driver written against the reference's C++ API as this library exports
// it (include/nse2d/grid.hpp, ops.hpp, diag.hpp, poisson.hpp), in the shape of the reference's
// time loop (src/main.cu:197-213 and 434-541): metrics from build_y_metrics, the initial solve
// and Thom closure, then per step the adaptive dt from launch_max_uv_from_psi_mapped and three
// stages of J, Laplacian, rhs, combine, Poisson2D_Z2Z::solve and the wall closure. Compiled and run
// by tests/test_compat_gpu.py, linked with libnse2d_b200.so only.
//
//   compat_driver <omega_in.bin> <out.bin> Nx Ny Lx beta Reb F0 nforce drag nsteps
// omega_in.bin: Ny*Nx float64; out.bin: omega, psi (Ny*Nx float64 each), then t and the sums of
// the diagnostic launchers (K, Omega, |grad omega|^2, epsilon, P_in, P_Omega) of the final state.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "nse2d/diag.hpp"
#include "nse2d/grid.hpp"
#include "nse2d/ops.hpp"
#include "nse2d/poisson.hpp"

#define CK(e)                                                                                  \
    do {                                                                                       \
        cudaError_t r__ = (e);                                                                 \
        if (r__ != cudaSuccess) { std::fprintf(stderr, "%s: %s\n", #e, cudaGetErrorString(r__)); std::exit(1); } \
    } while (0)

static Real* dev(const std::vector<Real>& h) {
    Real* d = nullptr;
    CK(cudaMalloc(&d, h.size() * sizeof(Real)));
    CK(cudaMemcpy(d, h.data(), h.size() * sizeof(Real), cudaMemcpyHostToDevice));
    return d;
}

int main(int argc, char** argv) {
    if (argc != 12) { std::fprintf(stderr, "usage: see the header\n"); return 2; }
    Grid G;
    G.Nx = std::atoi(argv[3]); G.Ny = std::atoi(argv[4]); G.Lx = std::atof(argv[5]); G.h = 1.0;
    Params P;
    P.stretch = "tanh"; P.beta = std::atof(argv[6]); P.Ub = 1.0; P.Reb = std::atof(argv[7]);
    P.F0 = std::atof(argv[8]); P.nforce = std::atoi(argv[9]); P.lin_drag = std::atof(argv[10]);
    P.adapt = true; P.cfl = 0.5; P.dt_max = 1e-2;
    const int nsteps = std::atoi(argv[11]);
    Grid Gm;
    build_y_metrics(G, P, Gm);
    G = Gm;
    const int Nx = G.Nx, Ny = G.Ny;
    const size_t N = (size_t)Nx * Ny;
    const Real nu = P.nu(G.h), dx = G.dx(), dy = G.dy(), inv_dx = 1.0 / dx, inv_dx2 = inv_dx * inv_dx;
    const Real deta = 2.0 / (Real)(Ny - 1), inv_deta = 1.0 / deta, inv_deta2 = inv_deta * inv_deta;
    Real dy_min = std::fabs(G.dy_edge[0]);
    for (int j = 1; j < Ny - 1; ++j) dy_min = std::fmin(dy_min, std::fabs(G.dy_edge[j]));
    const Real inv_dymin2 = 1.0 / (dy_min * dy_min);

    std::vector<Real> w0(N);
    FILE* f = std::fopen(argv[1], "rb");
    if (!f || std::fread(w0.data(), sizeof(Real), N, f) != N) { std::fprintf(stderr, "bad input\n"); return 1; }
    std::fclose(f);
    Real *a_node = dev(G.a_node), *a_edge = dev(G.a_edge), *y = dev(G.y), *dy_edge = dev(G.dy_edge);
    Real* w_node = dev(G.w_node);
    Real* w = dev(w0);
    Real *w1, *w2, *psi, *rhs, *J, *lap, *sc;
    for (Real** p : {&w1, &w2, &psi, &rhs, &J, &lap}) CK(cudaMalloc(p, N * sizeof(Real)));
    CK(cudaMalloc(&sc, 16 * sizeof(Real)));
    cudaStream_t s = 0;
    Poisson2D_Z2Z poisson(G, s);
    poisson.enable_mapped(a_node, a_edge, inv_deta, s);
    const Real psi_bot = 0.0, psi_top = 2.0 * G.h * P.Ub;
    poisson.solve(w, psi, dy, psi_bot, psi_top, s);
    launch_thom_wall_vorticity_mapped(w, psi, Nx, Ny, dy_edge, psi_bot, psi_top, s);

    Real t = 0.0, dt = P.dt_init;
    auto stage = [&](const Real* win) {
        launch_arakawa_J_mapped(psi, win, J, Nx, Ny, inv_dx, inv_deta, a_node, s);
        launch_laplacian_fd_mapped(win, lap, Nx, Ny, inv_dx2, inv_deta2, a_node, a_edge, s);
        launch_rhs_mapped(J, lap, win, rhs, Nx, Ny, nu, P.F0, P.nforce, G.h, P.lin_drag, y, s);
    };
    for (int n = 0; n < nsteps; ++n) {
        launch_max_uv_from_psi_mapped(psi, Nx, Ny, inv_dx, inv_deta, a_node, sc, sc + 1, sc + 2, s);
        Real m[3];
        CK(cudaMemcpy(m, sc, 3 * sizeof(Real), cudaMemcpyDeviceToHost));
        const Real dt_x = (m[0] > 0 ? P.cfl * (dx / m[0]) : 1e30), dt_y = (m[2] > 0 ? P.cfl * (deta / m[2]) : 1e30);
        const Real dt_vis = (nu > 0) ? P.cvisc * 0.5 / (nu * (inv_dx2 + inv_dymin2)) : 1e30;
        dt = std::fmin(P.dt_max, std::fmin(std::fmin(dt_x, dt_y), dt_vis));
        stage(w);
        launch_axpy(w1, w, rhs, dt, N, s);
        poisson.solve(w1, psi, dy, psi_bot, psi_top, s);
        launch_thom_wall_vorticity_mapped(w1, psi, Nx, Ny, dy_edge, psi_bot, psi_top, s);
        stage(w1);
        launch_ssprk2(w2, w, w1, rhs, dt, N, s);
        poisson.solve(w2, psi, dy, psi_bot, psi_top, s);
        launch_thom_wall_vorticity_mapped(w2, psi, Nx, Ny, dy_edge, psi_bot, psi_top, s);
        stage(w2);
        launch_ssprk3(w, w, w2, rhs, dt, N, s);
        poisson.solve(w, psi, dy, psi_bot, psi_top, s);
        launch_thom_wall_vorticity_mapped(w, psi, Nx, Ny, dy_edge, psi_bot, psi_top, s);
        t += dt;
    }
    // the diagnostic sums of the final state (the launchers the reference's output block calls)
    launch_kinetic_energy_mapped(psi, Nx, Ny, inv_dx, inv_deta, a_node, w_node, sc + 0, s);
    launch_enstrophy_diss_mapped(w, Nx, Ny, inv_dx, inv_deta, a_node, w_node, sc + 1, sc + 2, s);
    launch_energy_dissipation_mapped(psi, w, Nx, Ny, inv_dx, inv_deta, a_node, a_edge, w_node, sc + 3, s);
    launch_power_input_mapped(psi, Nx, Ny, inv_deta, G.h, P.F0, P.nforce, a_node, y, w_node, sc + 4, s);
    launch_enstrophy_input_mapped_full(w, Nx, Ny, G.h, P.F0, P.nforce, y, w_node, sc + 5, s);
    CK(cudaDeviceSynchronize());
    std::vector<Real> ho(N), hp(N), sums(6);
    CK(cudaMemcpy(ho.data(), w, N * sizeof(Real), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(hp.data(), psi, N * sizeof(Real), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(sums.data(), sc, 6 * sizeof(Real), cudaMemcpyDeviceToHost));
    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 1;
    std::fwrite(ho.data(), sizeof(Real), N, o);
    std::fwrite(hp.data(), sizeof(Real), N, o);
    std::fwrite(&t, sizeof(Real), 1, o);
    std::fwrite(sums.data(), sizeof(Real), 6, o);
    std::fclose(o);
    return 0;
}
