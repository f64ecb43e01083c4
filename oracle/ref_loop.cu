// TEST INFRASTRUCTURE (not part of the product): the reference's own SSPRK(3,3) time loop,
// driven through the reference's own launchers, for field parity on the same seeded inputs.
//
// Compiled by oracle/ref.mk together with the reference's sources (its headers on the include
// path, built with -DNSE2D_BUILD_AS_LIB so that src/main.cu contributes no main()) into
// oracle/_ref/libnse2d_refloop.so. Nothing of the reference is copied here: this file calls
//   build_y_metrics                     src/grid.cu:7-94
//   Poisson2D_Z2Z (ctor, enable_mapped, solve)   src/poisson.cuh:18-119
//   launch_thom_wall_vorticity_mapped   src/ops.cu:270-276
//   launch_arakawa_J_mapped, launch_laplacian_fd_mapped, launch_rhs_mapped,
//   launch_mms_add_forcing, launch_axpy / launch_ssprk2 / launch_ssprk3   src/ops.cu
//   launch_max_uv_from_psi_mapped       src/diag.cu:821-866
// in the order of the reference's driver: the initial solve and closure (src/main.cu:197-213),
// then per step the adaptive dt (src/main.cu:439-464, three blocking copies of the maxima) and
// the three stages (src/main.cu:482-541). Output scheduling (dt trimming, snapping) is not
// driven: the harness has no output times. The walls are no-slip (the library is built without
// FREE_SLIP_WALLS).
//
// C ABI for ctypes (oracle/ref_loop.py): refloop_create / _set_omega / _step / _get / _destroy.
#include "common.cuh"
#include "diag.cuh"
#include "grid.cuh"
#include "ops.cuh"
#include "poisson.cuh"

namespace {

struct RefLoop {
    Grid G;
    Params P;
    size_t N = 0;
    double dx = 0, inv_dx = 0, inv_dx2 = 0, dy = 0, deta = 0, inv_deta = 0, inv_deta2 = 0;
    double nu = 0, inv_dymin2 = 0, psi_bot = 0, psi_top = 0;
    double t = 0, dt = 0;
    long long step = 0;
    Real *w = nullptr, *w1 = nullptr, *w2 = nullptr, *psi = nullptr, *rhs = nullptr, *J = nullptr, *lap = nullptr;
    Real *a_node = nullptr, *a_edge = nullptr, *y_node = nullptr, *dy_edge = nullptr;
    Real *umax = nullptr, *vmax = nullptr, *vmaxm = nullptr;
    Poisson2D_Z2Z* poisson = nullptr;
    cudaStream_t s = 0;
};

template <typename T> void upload(Real** d, const std::vector<T>& h) {
    CUDA_CHECK(cudaMalloc(d, h.size() * sizeof(Real)));
    CUDA_CHECK(cudaMemcpy(*d, h.data(), h.size() * sizeof(Real), cudaMemcpyHostToDevice));
}

// omega^(s+1) = combine(...), then psi from it and the Thom wall rows: the tail of every stage
void solve_and_close(RefLoop* r, Real* w_stage) {
    r->poisson->solve(w_stage, r->psi, r->dy, r->psi_bot, r->psi_top, r->s);
    launch_thom_wall_vorticity_mapped(w_stage, r->psi, r->G.Nx, r->G.Ny, r->dy_edge, r->psi_bot, r->psi_top, r->s);
}

// J, the mapped Laplacian and the rhs of state (psi, w_in) at time tm, with the MMS forcing
void stage_rhs(RefLoop* r, const Real* w_in, double tm) {
    const Grid& G = r->G;
    const Params& P = r->P;
    launch_arakawa_J_mapped(r->psi, w_in, r->J, G.Nx, G.Ny, r->inv_dx, r->inv_deta, r->a_node, r->s);
    launch_laplacian_fd_mapped(w_in, r->lap, G.Nx, G.Ny, r->inv_dx2, r->inv_deta2, r->a_node, r->a_edge, r->s);
    launch_rhs_mapped(r->J, r->lap, w_in, r->rhs, G.Nx, G.Ny, r->nu, P.F0, P.nforce, G.h, P.lin_drag, r->y_node, r->s);
    if (P.mms)
        launch_mms_add_forcing(r->rhs, G.Nx, G.Ny, G.Lx, G.h, tm, r->nu, P.lin_drag, P.mms_A0, P.mms_eps, P.mms_Om,
                               P.mms_kx, r->y_node, r->s);
}

}  // namespace

extern "C" {

// Grid and physics as the reference's Grid/Params fields (src/common.cuh:42-114); stretch 0
// uniform, 1 tanh. dt_init is the fixed dt when adapt == 0, as --no-adapt --dt in the reference.
void* refloop_create(int Nx, int Ny, double Lx, double h, int stretch, double beta, double Ub, double Reb,
                     double nu_override, double F0, int nforce, double lin_drag, int adapt, double cfl, double cvisc,
                     double dt_max, double dt_init, int mms, double mms_A0, double mms_eps, double mms_Om,
                     int mms_kx) {
    RefLoop* r = new RefLoop();
    Grid Gin;
    Gin.Nx = Nx; Gin.Ny = Ny; Gin.Lx = Lx; Gin.h = h;
    Params& P = r->P;
    P.stretch = stretch ? "tanh" : "none";
    P.beta = beta; P.Ub = Ub; P.Reb = Reb; P.nu_override = nu_override;
    P.F0 = F0; P.nforce = nforce; P.lin_drag = lin_drag; P.adapt = adapt != 0;
    P.cfl = cfl; P.cvisc = cvisc; P.dt_max = dt_max; P.dt_init = dt_init;
    P.mms = mms != 0; P.mms_A0 = mms_A0; P.mms_eps = mms_eps; P.mms_Om = mms_Om; P.mms_kx = mms_kx;
    build_y_metrics(Gin, P, r->G);
    const Grid& G = r->G;
    r->N = (size_t)Nx * Ny;
    r->dx = G.dx(); r->dy = G.dy();
    r->inv_dx = 1.0 / r->dx; r->inv_dx2 = r->inv_dx * r->inv_dx;
    r->deta = 2.0 / (Real)(Ny - 1); r->inv_deta = 1.0 / r->deta; r->inv_deta2 = r->inv_deta * r->inv_deta;
    r->nu = P.nu(G.h);
    double dy_min = std::fabs(G.dy_edge[0]);
    for (int j = 1; j < Ny - 1; ++j) dy_min = std::min(dy_min, std::fabs(G.dy_edge[j]));
    r->inv_dymin2 = 1.0 / (dy_min * dy_min);
    r->psi_bot = 0.0; r->psi_top = 2.0 * G.h * P.Ub;
    upload(&r->a_node, G.a_node);
    upload(&r->a_edge, G.a_edge);
    upload(&r->y_node, G.y);
    upload(&r->dy_edge, G.dy_edge);
    for (Real** f : {&r->w, &r->w1, &r->w2, &r->psi, &r->rhs, &r->J, &r->lap}) CUDA_CHECK(cudaMalloc(f, r->N * sizeof(Real)));
    for (Real** f : {&r->umax, &r->vmax, &r->vmaxm}) CUDA_CHECK(cudaMalloc(f, sizeof(Real)));
    r->poisson = new Poisson2D_Z2Z(G, r->s);
    r->poisson->enable_mapped(r->a_node, r->a_edge, r->inv_deta, r->s);
    CUDA_CHECK(cudaDeviceSynchronize());
    return r;
}

// omega from a host array, then the initial solve and wall closure; t = 0, dt = dt_init
void refloop_set_omega(void* h, const double* host_w) {
    RefLoop* r = static_cast<RefLoop*>(h);
    CUDA_CHECK(cudaMemcpy(r->w, host_w, r->N * sizeof(Real), cudaMemcpyHostToDevice));
    solve_and_close(r, r->w);
    CUDA_CHECK(cudaDeviceSynchronize());
    r->t = 0.0; r->dt = r->P.dt_init; r->step = 0;
}

// nsteps steps of the reference's loop body
void refloop_step(void* h, int nsteps) {
    RefLoop* r = static_cast<RefLoop*>(h);
    const Grid& G = r->G;
    const Params& P = r->P;
    for (int n = 0; n < nsteps; ++n) {
        if (P.adapt) {
            launch_max_uv_from_psi_mapped(r->psi, G.Nx, G.Ny, r->inv_dx, r->inv_deta, r->a_node, r->umax, r->vmax,
                                          r->vmaxm, r->s);
            Real um, vm, vmm;
            CUDA_CHECK(cudaMemcpy(&um, r->umax, sizeof(Real), cudaMemcpyDeviceToHost));
            CUDA_CHECK(cudaMemcpy(&vm, r->vmax, sizeof(Real), cudaMemcpyDeviceToHost));
            CUDA_CHECK(cudaMemcpy(&vmm, r->vmaxm, sizeof(Real), cudaMemcpyDeviceToHost));
            const Real dt_x = (um > 0 ? P.cfl * (r->dx / um) : 1e30);
            const Real dt_y = (vmm > 0 ? P.cfl * (r->deta / vmm) : 1e30);
            const Real dt_vis = (r->nu > 0) ? P.cvisc * 0.5 / (r->nu * (r->inv_dx2 + r->inv_dymin2)) : 1e30;
            r->dt = fmin(P.dt_max, fmin(fmin(dt_x, dt_y), dt_vis));
        }
        const double t = r->t, dt = r->dt;
        stage_rhs(r, r->w, t);
        launch_axpy(r->w1, r->w, r->rhs, dt, r->N, r->s);
        solve_and_close(r, r->w1);
        stage_rhs(r, r->w1, t + dt);
        launch_ssprk2(r->w2, r->w, r->w1, r->rhs, dt, r->N, r->s);
        solve_and_close(r, r->w2);
        stage_rhs(r, r->w2, t + 0.5 * dt);
        launch_ssprk3(r->w, r->w, r->w2, r->rhs, dt, r->N, r->s);
        solve_and_close(r, r->w);
        r->t = t + dt;
        r->step += 1;
    }
    CUDA_CHECK(cudaDeviceSynchronize());
}

// omega, psi (host arrays, either may be NULL), t, dt and the step count
void refloop_get(void* h, double* host_w, double* host_psi, double* t, double* dt, long long* step) {
    RefLoop* r = static_cast<RefLoop*>(h);
    if (host_w) CUDA_CHECK(cudaMemcpy(host_w, r->w, r->N * sizeof(Real), cudaMemcpyDeviceToHost));
    if (host_psi) CUDA_CHECK(cudaMemcpy(host_psi, r->psi, r->N * sizeof(Real), cudaMemcpyDeviceToHost));
    if (t) *t = r->t;
    if (dt) *dt = r->dt;
    if (step) *step = r->step;
}

void refloop_destroy(void* h) {
    RefLoop* r = static_cast<RefLoop*>(h);
    if (!r) return;
    delete r->poisson;
    for (Real* f : {r->w, r->w1, r->w2, r->psi, r->rhs, r->J, r->lap, r->a_node, r->a_edge, r->y_node, r->dy_edge,
                    r->umax, r->vmax, r->vmaxm})
        cudaFree(f);
    delete r;
}

}  // extern "C"
