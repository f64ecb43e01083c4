// Standalone operators: the reference's C-linkage test API (src/test_api.cu:8-92) and the
// operators behind it (src/ops.cu), plus J/rhs at a state for the diagnostics.
// Written for this project. These are not on the time-step path (which uses the fused
// kernels of step_kernels.cuh); they serve the drop-in ABI, the diagnostics and tests.
#include <cstdio>
#include <cstdlib>

#include "nse2d_internal.h"
#include "step_kernels.cuh"
#include "../../include/nse2d.h"

namespace nse2d {

static bool g_abort_on_error = true;
static bool g_free_slip = false;

// Reference semantics of CUDA_CHECK (src/common.cuh:116-117): print and abort.
static void after_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return;
    set_error("%s: %s", what, cudaGetErrorString(e));
    if (g_abort_on_error) {
        std::fprintf(stderr, "CUDA error in %s: %s\n", what, cudaGetErrorString(e));
        std::abort();
    }
}

void compat_check_launch(const char* what) { after_launch(what); }
bool compat_free_slip() { return g_free_slip; }

static dim3 grid2d(int Nx, int Ny, dim3 tb) { return dim3((Nx + tb.x - 1) / tb.x, (Ny + tb.y - 1) / tb.y); }

// u, v with clamped j+-1 at the walls: src/ops.cu:47-63
__global__ void k_uv(const double* __restrict__ psi, double* __restrict__ u, double* __restrict__ v, int Nx, int Ny,
                     double inv_dx, double inv_deta, const double* __restrict__ a_node) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= Nx || iy >= Ny) return;
    const int xm = wrapi(ix - 1, Nx), xp = wrapi(ix + 1, Nx);
    const int ym = (iy == 0 ? 0 : iy - 1), yp = (iy == Ny - 1 ? Ny - 1 : iy + 1);
    const double dpsideta = (psi[(size_t)yp * Nx + ix] - psi[(size_t)ym * Nx + ix]) * 0.5 * inv_deta;
    const double dpsidx = (psi[(size_t)iy * Nx + xp] - psi[(size_t)iy * Nx + xm]) * 0.5 * inv_dx;
    u[(size_t)iy * Nx + ix] = a_node[iy] * dpsideta;
    v[(size_t)iy * Nx + ix] = -dpsidx;
}

// omega from psi on interior rows: src/ops.cu:72-93
__global__ void k_omega_from_psi(double* __restrict__ w, const double* __restrict__ psi, int Nx, int Ny,
                                 double inv_dx2, double inv_deta2, const double* __restrict__ a_node,
                                 const double* __restrict__ a_edge) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= Nx || iy >= Ny || iy == 0 || iy == Ny - 1) return;
    const int xm = wrapi(ix - 1, Nx), xp = wrapi(ix + 1, Nx);
    const size_t c = (size_t)iy * Nx + ix;
    const double lapx = psi[(size_t)iy * Nx + xp] - 2.0 * psi[c] + psi[(size_t)iy * Nx + xm];
    const double lapy = a_node[iy] * (a_edge[iy] * (psi[c + Nx] - psi[c]) - a_edge[iy - 1] * (psi[c] - psi[c - Nx]));
    w[c] = -(inv_dx2 * lapx + inv_deta2 * lapy);
}

// Arakawa J1, J2, J3 at an interior point: src/ops.cu:305-322
__device__ __forceinline__ void arakawa3(const double* __restrict__ psi, const double* __restrict__ omg, int Nx,
                                         int iy, int ix, double inv_dx, double inv_deta, double a,
                                         double& J1, double& J2, double& J3) {
    const int xm = wrapi(ix - 1, Nx), xp = wrapi(ix + 1, Nx), ym = iy - 1, yp = iy + 1;
    const size_t cxp = (size_t)iy * Nx + xp, cxm = (size_t)iy * Nx + xm;
    const size_t cyp = (size_t)yp * Nx + ix, cym = (size_t)ym * Nx + ix;
    const size_t ip_jp = (size_t)yp * Nx + xp, ip_jm = (size_t)ym * Nx + xp;
    const size_t im_jp = (size_t)yp * Nx + xm, im_jm = (size_t)ym * Nx + xm;
    const double inv4dxde = 0.25 * inv_dx * inv_deta;
    J1 = ((psi[cxp] - psi[cxm]) * (a * (omg[cyp] - omg[cym])) - (a * (psi[cyp] - psi[cym])) * (omg[cxp] - omg[cxm])) * inv4dxde;
    J2 = (psi[cxp] * (a * (omg[ip_jp] - omg[ip_jm])) - psi[cxm] * (a * (omg[im_jp] - omg[im_jm]))
          - a * (psi[cyp] * (omg[ip_jp] - omg[im_jp]) - psi[cym] * (omg[ip_jm] - omg[im_jm]))) * inv4dxde;
    J3 = (-omg[cxp] * (a * (psi[ip_jp] - psi[ip_jm])) + omg[cxm] * (a * (psi[im_jp] - psi[im_jm]))
          + a * (omg[cyp] * (psi[ip_jp] - psi[im_jp]) - omg[cym] * (psi[ip_jm] - psi[im_jm]))) * inv4dxde;
}

__global__ void k_arakawa(const double* __restrict__ psi, const double* __restrict__ omg, double* __restrict__ J,
                          int Nx, int Ny, double inv_dx, double inv_deta, const double* __restrict__ a_node) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= Nx || iy >= Ny) return;
    const size_t c = (size_t)iy * Nx + ix;
    if (iy == 0 || iy == Ny - 1) { J[c] = 0.0; return; }
    double J1, J2, J3;
    arakawa3(psi, omg, Nx, iy, ix, inv_dx, inv_deta, a_node[iy], J1, J2, J3);
    J[c] = -((J1 + J2 + J3) * (1.0 / 3.0));
}

// split outputs, any may be NULL: src/ops.cu:415-467
__global__ void k_arakawa_split(const double* __restrict__ psi, const double* __restrict__ omg, double* J1o,
                                double* J2o, double* J3o, double* Jadv, int Nx, int Ny, double inv_dx,
                                double inv_deta, const double* __restrict__ a_node) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= Nx || iy >= Ny) return;
    const size_t c = (size_t)iy * Nx + ix;
    if (iy == 0 || iy == Ny - 1) {
        if (J1o) J1o[c] = 0.0;
        if (J2o) J2o[c] = 0.0;
        if (J3o) J3o[c] = 0.0;
        if (Jadv) Jadv[c] = 0.0;
        return;
    }
    double J1, J2, J3;
    arakawa3(psi, omg, Nx, iy, ix, inv_dx, inv_deta, a_node[iy], J1, J2, J3);
    if (J1o) J1o[c] = J1;
    if (J2o) J2o[c] = J2;
    if (J3o) J3o[c] = J3;
    if (Jadv) Jadv[c] = -((J1 + J2 + J3) * (1.0 / 3.0));
}

// advective reference from (u, v): src/ops.cu:339-371
__global__ void k_adv_from_uv(const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ omg,
                              double* __restrict__ Jadv, int Nx, int Ny, double inv_dx, double inv_deta,
                              const double* __restrict__ a_node) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= Nx || iy >= Ny) return;
    const size_t c = (size_t)iy * Nx + ix;
    if (iy == 0 || iy == Ny - 1) { Jadv[c] = 0.0; return; }
    const int xm = wrapi(ix - 1, Nx), xp = wrapi(ix + 1, Nx);
    const double inv2dx = 0.5 * inv_dx, inv2de = 0.5 * inv_deta, a = a_node[iy];
    const double dx_omg = (omg[(size_t)iy * Nx + xp] - omg[(size_t)iy * Nx + xm]) * inv2dx;
    const double dy_omg = a * (omg[c + Nx] - omg[c - Nx]) * inv2de;
    Jadv[c] = u[c] * dx_omg + v[c] * dy_omg;
}

// conservative flux form: src/ops.cu:372-409
__global__ void k_adv_flux(const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ omg,
                           double* __restrict__ Jadv, int Nx, int Ny, double inv_dx, double inv_deta,
                           const double* __restrict__ a_node) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= Nx || iy >= Ny) return;
    const size_t c = (size_t)iy * Nx + ix;
    if (iy == 0 || iy == Ny - 1) { Jadv[c] = 0.0; return; }
    const int xm = wrapi(ix - 1, Nx), xp = wrapi(ix + 1, Nx);
    const size_t cxm = (size_t)iy * Nx + xm, cxp = (size_t)iy * Nx + xp, cym = c - Nx, cyp = c + Nx;
    const double u_ip = (u[cxp] + u[c]) * 0.5, u_im = (u[c] + u[cxm]) * 0.5;
    const double w_ip = (omg[cxp] + omg[c]) * 0.5, w_im = (omg[c] + omg[cxm]) * 0.5;
    const double dFdx = (u_ip * w_ip - u_im * w_im) * inv_dx;
    const double v_jp = (v[cyp] + v[c]) * 0.5, v_jm = (v[c] + v[cym]) * 0.5;
    const double w_jp = (omg[cyp] + omg[c]) * 0.5, w_jm = (omg[c] + omg[cym]) * 0.5;
    const double dFdy = a_node[iy] * ((v_jp * w_jp - v_jm * w_jm) * (0.5 * inv_deta * 2.0));
    Jadv[c] = dFdx + dFdy;
}

// J and rhs at one state (for the diagnostics, src/main.cu:345-362 and :595-599), the same
// arithmetic as the fused stage kernel.
__global__ void k_rhs_state(StageParams p, double* __restrict__ Jout, double* __restrict__ rhs_out, double tm) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= p.Nx || iy >= p.Ny) return;
    double mA = 0.0, mAp = 0.0;
    if (p.mms) {
        mA = p.mms_A0 * (1.0 + p.mms_eps * sin(p.mms_Om * tm));
        mAp = p.mms_A0 * (p.mms_eps * p.mms_Om * cos(p.mms_Om * tm));
    }
    const size_t c = (size_t)iy * p.Nx + ix;
    const double wc = p.w_in[c];
    rhs_out[c] = point_rhs(p, iy, ix, p.rt.frow[iy], wc, mA, mAp);
    if (Jout) {
        if (iy == 0 || iy == p.Ny - 1) {
            Jout[c] = 0.0;
        } else {
            double J1, J2, J3;
            arakawa3(p.psi, p.w_in, p.Nx, iy, ix, p.inv_dx, p.inv_deta, p.rt.a_node[iy], J1, J2, J3);
            Jout[c] = -((J1 + J2 + J3) * (1.0 / 3.0));
        }
    }
}

int rhs_at_state(Context* c, const double* w, const double* psi, double* J, double* rhs, double tm, cudaStream_t s) {
    StageParams p{};
    p.psi = psi; p.w_in = w; p.rt = c->rt;
    p.Nx = c->Nx; p.Ny = c->Ny; p.mms = c->cfg.mms;
    p.inv_dx = c->inv_dx; p.inv_deta = c->inv_deta; p.inv_dx2 = c->inv_dx2; p.inv_deta2 = c->inv_deta2;
    p.nu = c->nu; p.lin_drag = c->cfg.lin_drag;
    p.mms_A0 = c->cfg.mms_A0; p.mms_eps = c->cfg.mms_eps; p.mms_Om = c->cfg.mms_Om;
    p.mms_k = 2.0 * kPiD * (double)c->cfg.mms_kx / c->cfg.Lx; p.mms_c = kPiD / (2.0 * c->cfg.h);
    const dim3 tb(128, 2);
    k_rhs_state<<<grid2d(c->Nx, c->Ny, tb), tb, 0, s>>>(p, J, rhs, tm);
    NSE_CUDA_TRY(cudaGetLastError());
    return 0;
}

int uv_from_psi(Context* c, const double* psi, double* u, double* v, cudaStream_t s) {
    const dim3 tb(128, 2);
    k_uv<<<grid2d(c->Nx, c->Ny, tb), tb, 0, s>>>(psi, u, v, c->Nx, c->Ny, c->inv_dx, c->inv_deta, c->rt.a_node);
    NSE_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace nse2d

using namespace nse2d;

extern "C" {

void nse2d_set_abort_on_error(int on) { g_abort_on_error = (on != 0); }
void nse2d_testapi_set_free_slip(int on) { g_free_slip = (on != 0); }

void testapi_uv_from_psi_mapped(const double* d_psi, double* d_u, double* d_v, int Nx, int Ny, double inv_dx,
                                double inv_deta, const double* d_a_node, cudaStream_t s) {
    const dim3 tb(32, 8);
    k_uv<<<grid2d(Nx, Ny, tb), tb, 0, s>>>(d_psi, d_u, d_v, Nx, Ny, inv_dx, inv_deta, d_a_node);
    after_launch("testapi_uv_from_psi_mapped");
}

void testapi_omega_from_psi_interior_mapped(double* d_w, const double* d_psi, int Nx, int Ny, double inv_dx2,
                                            double inv_deta2, const double* d_a_node, const double* d_a_edge,
                                            cudaStream_t s) {
    const dim3 tb(32, 8);
    k_omega_from_psi<<<grid2d(Nx, Ny, tb), tb, 0, s>>>(d_w, d_psi, Nx, Ny, inv_dx2, inv_deta2, d_a_node, d_a_edge);
    after_launch("testapi_omega_from_psi_interior_mapped");
}

void testapi_thom_wall_vorticity_mapped(double* d_w, const double* d_psi, int Nx, int Ny, const double* d_dy_edge,
                                        double psi_bot, double psi_top, cudaStream_t s) {
    ThomParams p{};
    p.w = d_w; p.psi = d_psi; p.dy_edge = d_dy_edge;
    p.Nx = Nx; p.Ny = Ny; p.free_slip = g_free_slip ? 1 : 0;
    p.psi_bot = psi_bot; p.psi_top = psi_top;
    k_thom<<<(Nx + 255) / 256, 256, 0, s>>>(p);
    after_launch("testapi_thom_wall_vorticity_mapped");
}

void testapi_arakawa_J_mapped(const double* d_psi, const double* d_w, double* d_J, int Nx, int Ny, double inv_dx,
                              double inv_deta, const double* d_a_node, cudaStream_t s) {
    const dim3 tb(32, 8);
    k_arakawa<<<grid2d(Nx, Ny, tb), tb, 0, s>>>(d_psi, d_w, d_J, Nx, Ny, inv_dx, inv_deta, d_a_node);
    after_launch("testapi_arakawa_J_mapped");
}

void testapi_compute_adv_from_uv_mapped(const double* d_u, const double* d_v, const double* d_omg, double* d_Jref,
                                        int Nx, int Ny, double inv_dx, double inv_deta, const double* d_a_node,
                                        cudaStream_t s) {
    const dim3 tb(32, 4);
    k_adv_from_uv<<<grid2d(Nx, Ny, tb), tb, 0, s>>>(d_u, d_v, d_omg, d_Jref, Nx, Ny, inv_dx, inv_deta, d_a_node);
    after_launch("testapi_compute_adv_from_uv_mapped");
}

void testapi_compute_adv_flux_mapped(const double* d_u, const double* d_v, const double* d_omg, double* d_Jref,
                                     int Nx, int Ny, double inv_dx, double inv_deta, const double* d_a_node,
                                     cudaStream_t s) {
    const dim3 tb(32, 4);
    k_adv_flux<<<grid2d(Nx, Ny, tb), tb, 0, s>>>(d_u, d_v, d_omg, d_Jref, Nx, Ny, inv_dx, inv_deta, d_a_node);
    after_launch("testapi_compute_adv_flux_mapped");
}

void testapi_arakawa_J_mapped_split(const double* d_psi, const double* d_omg, double* d_J1, double* d_J2,
                                    double* d_J3, double* d_Jadv, int Nx, int Ny, double inv_dx, double inv_deta,
                                    const double* d_a_node, cudaStream_t s) {
    const dim3 tb(32, 4);
    k_arakawa_split<<<grid2d(Nx, Ny, tb), tb, 0, s>>>(d_psi, d_omg, d_J1, d_J2, d_J3, d_Jadv, Nx, Ny, inv_dx,
                                                      inv_deta, d_a_node);
    after_launch("testapi_arakawa_J_mapped_split");
}

}  // extern "C"
