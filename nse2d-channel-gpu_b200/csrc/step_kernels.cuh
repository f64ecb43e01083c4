// Device kernels of one SSPRK(3,3) step (FP64). Written for this project.
//
// Per stage s (reference loop src/main.cu:482-538):
//   k_stage_tma   2-D tiles: omega^(s+1) = RK combine of omega^(s) + dt rhs(psi, omega^(s)),
//                 rhs = -J_arakawa + nu lap + f(y) - r omega (+ MMS forcing). psi and omega
//                 tiles with a one-cell halo arrive in shared memory by TMA (k_stage, with
//                 plain loads, below 128 columns).
//   k_fft_fwd     forward real FFT of every interior row of omega^(s+1) -> omega-hat [Ny][Hp].
//   k_thomas_cluster  y-direction tridiagonal solve of every kx column, in place
//                 (omega-hat -> psi-hat). One thread-block cluster owns 8 kx columns and
//                 splits the Ny-2 rows among its CTAs; each thread sweeps a segment of rows and
//                 the segments are joined through their affine carries (smem + DSMEM). Very
//                 tall grids use the two-pass form (k_thomas_maps, k_thomas_apply).
//   k_ifft_thom   inverse real FFT of every row -> psi [Ny][Nx], then the Thom wall vorticity
//                 of omega^(s+1) by the CTAs that own rows 1-2 and Ny-3..Ny-2.
// Per step: k_maxuv_dt (max|u|,|v|,|v|a -> adaptive dt on the device) before stage 1; the
// last CTA of the stage-3 k_ifft_thom advances the time.
#pragma once
#include <cuda.h>
#include <cooperative_groups.h>
#include <cstdint>

#include "common.cuh"
#include "fft_rows.cuh"

namespace nse2d {

constexpr double kPiD = 3.141592653589793;   // the double nearest pi (CUDART_PI)

__device__ __forceinline__ int wrapi(int i, int Nx) { return i < 0 ? i + Nx : (i >= Nx ? i - Nx : i); }

struct StageParams {
    const double* psi;       // [Ny][Nx]
    const double* w_in;      // omega^(s), stencil input
    const double* w_n;       // omega^n (stages 2, 3); may alias w_out in stage 3
    double* w_out;           // omega^(s+1)
    double* rhs_out;         // optional: store rhs (the stage-3 rhs read by the diagnostics)
    const double* closure;   // optional: learned subgrid term tau [Ny][Nx], rhs -= tau on interior rows
    RowTables rt;
    Ctl* ctl;
    int Nx, Ny, stage, mms;
    double inv_dx, inv_deta, inv_dx2, inv_deta2, nu, lin_drag;
    double mms_A0, mms_eps, mms_Om, mms_k, mms_c;
    // dt_from_max (stage 1): dt from the maxima the previous step's inverse transform left in
    // ctl->mx_next (adaptive_dt); CTA 0 writes it and those maxima to the control block
    int dt_from_max;
    double cfl, cvisc, dx, deta, inv_dymin2, dt_max;
};

// Mapped Arakawa Jacobian (src/ops.cu:305-325) and Laplacian (src/ops.cu:488-498) from the
// 3x3 neighbourhood: p[r][c], o[r][c] with r = 0,1,2 for rows j-1, j, j+1 and c for x-1, x, x+1.
__device__ __forceinline__ void stencil_J_lap(const double p[3][3], const double o[3][3], double a, double ap,
                                              double am, double inv_dx, double inv_deta, double inv_dx2,
                                              double inv_deta2, double& J, double& lap) {
    const double inv4dxde = 0.25 * inv_dx * inv_deta;
    const double psi_xp = p[1][2], psi_xm = p[1][0], psi_yp = p[2][1], psi_ym = p[0][1];
    const double psi_pp = p[2][2], psi_pm = p[0][2], psi_mp = p[2][0], psi_mm = p[0][0];
    const double om_xp = o[1][2], om_xm = o[1][0], om_yp = o[2][1], om_ym = o[0][1];
    const double om_pp = o[2][2], om_pm = o[0][2], om_mp = o[2][0], om_mm = o[0][0];
    const double wc = o[1][1];
    const double J1 = ((psi_xp - psi_xm) * (a * (om_yp - om_ym)) - (a * (psi_yp - psi_ym)) * (om_xp - om_xm)) * inv4dxde;
    const double J2 = (psi_xp * (a * (om_pp - om_pm)) - psi_xm * (a * (om_mp - om_mm))
                       - a * (psi_yp * (om_pp - om_mp) - psi_ym * (om_pm - om_mm))) * inv4dxde;
    const double J3 = (-om_xp * (a * (psi_pp - psi_pm)) + om_xm * (a * (psi_mp - psi_mm))
                       + a * (om_yp * (psi_pp - psi_mp) - om_ym * (psi_pm - psi_mm))) * inv4dxde;
    J = -((J1 + J2 + J3) * (1.0 / 3.0));
    const double dxx = (om_xp - 2 * wc + om_xm) * inv_dx2;
    const double dyy = a * (ap * (om_yp - wc) - am * (wc - om_ym)) * inv_deta2;
    lap = dxx + dyy;
}

// MMS forcing at one point (src/ops.cu:587-624), with per-row and per-column tables.
__device__ __forceinline__ double mms_term(const StageParams& p, int j, int i, double mA, double mAp) {
    const double k = p.mms_k, c = p.mms_c, c2 = c * c, c3 = c2 * c;
    const double g = p.rt.mms_g[j], gpp = p.rt.mms_gpp[j], sin2 = p.rt.mms_sin2[j];
    const double sk = p.rt.mms_sk[i], s2k = p.rt.mms_s2k[i];
    const double term_lin = mAp * g + (p.nu * mA) * ((k * k) * g - gpp) + (p.lin_drag * mA) * g;
    const double term_adv = -(mA * mA) * k * c3 * s2k * sin2;
    return sk * term_lin + term_adv;
}

// rhs at one point from global memory (used outside the step: diagnostics, J/rhs at a state)
__device__ __forceinline__ double point_rhs(const StageParams& p, int j, int i, double fj, double wc,
                                            double mA, double mAp, double* Jout = nullptr) {
    const int Nx = p.Nx;
    double J = 0.0, lap = 0.0;
    if (j != 0 && j != p.Ny - 1) {
        double ps[3][3], om[3][3];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const size_t id = (size_t)(j - 1 + r) * Nx + wrapi(i - 1 + c, Nx);
                ps[r][c] = p.psi[id];
                om[r][c] = p.w_in[id];
            }
        stencil_J_lap(ps, om, p.rt.a_node[j], p.rt.a_edge[j], p.rt.a_edge[j - 1], p.inv_dx, p.inv_deta, p.inv_dx2,
                      p.inv_deta2, J, lap);
    }
    if (Jout) *Jout = J;
    double rhs = -J + p.nu * lap + fj - p.lin_drag * wc;
    if (p.mms) rhs += mms_term(p, j, i, mA, mAp);
    return rhs;
}

// The larger of a and b for a >= 0 that is not NaN: a compare and a select. A NaN b is skipped
// (as fmax skips it), and an accumulator that starts at 0 never becomes NaN.
__device__ __forceinline__ double nn_max(double a, double b) { return b > a ? b : a; }

// Programmatic dependent launch: a step kernel launched with the programmatic-serialisation
// attribute may be launched while the kernel before it in the stream is still finishing (its
// CTAs trigger the next launch as they exit). Every step kernel begins with pdl_begin: it waits
// until the grids it depends on have completed and their writes are visible (a no-op for a kernel
// launched without the attribute). Nothing is read or written before the wait. An explicit trigger
// right after the wait, which lets the next kernel's CTAs become resident early, measured slower.
__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
}
__device__ __forceinline__ double warp_max_nn(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nn_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double time_tol_d(double t) { return 64.0 * 2.220446049250313e-16 * fmax(1.0, fabs(t)); }

// The adaptive dt of the reference (src/main.cu:439-480) from max |u| and max |v| a: CFL limits in
// x and eta, the viscous limit, dt_max, and the trim to the next output time. Every caller (the
// max reduction's last CTA, the stage kernel when the maxima come from the previous step's
// inverse transform) evaluates this one function, so dt has the same bits either way.
__device__ __forceinline__ double adaptive_dt(double umax, double vmaxm, double t, double t_next, double cfl,
                                             double dx, double deta, double cvisc, double nu, double inv_dx2,
                                             double inv_dymin2, double dt_max) {
    const double dt_x = (umax > 0 ? cfl * (dx / umax) : 1e30);
    const double dt_y = (vmaxm > 0 ? cfl * (deta / vmaxm) : 1e30);
    const double dt_adv = fmin(dt_x, dt_y);
    const double dt_vis = (nu > 0) ? cvisc * 0.5 / (nu * (inv_dx2 + inv_dymin2)) : 1e30;
    double dt = fmin(dt_max, fmin(dt_adv, dt_vis));
    if (t_next < 1e299) {
        const double rem = t_next - t;
        const double tol = fmax(time_tol_d(t_next), 1e-6 * dt);
        if (rem > tol && rem < 0.5 * dt) dt = rem;
    }
    return dt;
}

// ---- stage kernels: 2-D tiles of ST_TX x ST_TY points, halo of psi and omega^(s) in shared memory ----
// 256 threads = 64 columns x 4 row groups; a thread sweeps 8 consecutive rows of one column
// with a sliding 3-row window of psi and omega in registers (6 shared loads per point).
constexpr int ST_TX = 64, ST_TY = 32, ST_RPT = 8, ST_W = ST_TX + 2, ST_H = ST_TY + 2;

// Stage constants of one launch: dt, and the MMS amplitude at the stage time (main.cu:487-528).
struct StageTime {
    double dt, mA, mAp;
};
__device__ __forceinline__ StageTime stage_time(const StageParams& p) {
    StageTime st;
    if (p.dt_from_max && p.stage == 1) {
        Ctl* c = p.ctl;
        const double um = c->mx_next[0], vm = c->mx_next[1], vmm = c->mx_next[2];
        st.dt = adaptive_dt(um, vmm, c->t, c->next_out, p.cfl, p.dx, p.deta, p.cvisc, p.nu, p.inv_dx2, p.inv_dymin2,
                            p.dt_max);
        if (blockIdx.x == 0 && threadIdx.x == 0) {   // for the later kernels and the host; no CTA of this one reads them
            c->dt = st.dt;
            c->umax = um; c->vmax = vm; c->vmaxm = vmm;
        }
    } else {
        st.dt = p.ctl->dt;
    }
    const double t = p.ctl->t;
    const double ts = (p.stage == 1) ? t : (p.stage == 2 ? t + st.dt : t + 0.5 * st.dt);
    st.mA = 0.0;
    st.mAp = 0.0;
    if (p.mms) {
        st.mA = p.mms_A0 * (1.0 + p.mms_eps * sin(p.mms_Om * ts));
        st.mAp = p.mms_A0 * (p.mms_eps * p.mms_Om * cos(p.mms_Om * ts));
    }
    return st;
}

// The points of one tile from its halo in shared memory: sp/so[r * ld + c] holds row y0 - 1 + r,
// column x0 - 1 - coff + c.
//
// The arithmetic is the reference's rhs = -J + nu lap + f - r omega (src/ops.cu:532) with the
// Arakawa Jacobian (src/ops.cu:305-325) and the mapped Laplacian (src/ops.cu:488-498), regrouped
// for fewer FP64 operations: every term of J1 + J2 + J3 carries the factor a_j / (4 dx deta), so
//   J = -c_j S,  c_j = a_j / (12 dx deta),
//   S = Dx psi_j Dy om_i - Dy psi_i Dx om_j
//     + psi_{i+1,j} Dy om_{i+1} - psi_{i-1,j} Dy om_{i-1} - psi_{i,j+1} Dx om_{j+1} + psi_{i,j-1} Dx om_{j-1}
//     - om_{i+1,j} Dy psi_{i+1} + om_{i-1,j} Dy psi_{i-1} + om_{i,j+1} Dx psi_{j+1} - om_{i,j-1} Dx psi_{j-1},
// with Dx f_j = f_{i+1,j} - f_{i-1,j} and Dy f_i = f_{i,j+1} - f_{i,j-1}, the very differences the
// reference forms; the x differences of rows j-1 and j are carried down the sliding window.
// nu lap = nu/dx^2 (om_{i+1} + om_{i-1} - 2 om) + A+_j (om_{j+1} - om) - A-_j (om - om_{j-1}),
// A+-_j = nu a_j a_{j+-1/2} / deta^2 from the row tables. The regrouping moves the result by a few
// ulps of its terms; the stage parity bounds hold with margin.
__device__ __forceinline__ double stage_rhs_interior(double rhs, double wc, double p_xm, double p_xp, double p_ym,
                                                    double p_yp, double dyp_m, double dyp_c, double dyp_p,
                                                    const double (&dxp)[3], double o_xm, double o_xp, double o_ym,
                                                    double o_yp, double dyo_m, double dyo_c, double dyo_p,
                                                    const double (&dxo)[3], double nu_dx2, double ap, double am,
                                                    double cj) {
    double s1 = dxp[1] * dyo_c;
    s1 = fma(-dyp_c, dxo[1], s1);
    s1 = fma(p_xp, dyo_p, s1);
    s1 = fma(-p_xm, dyo_m, s1);
    s1 = fma(-p_yp, dxo[2], s1);
    s1 = fma(p_ym, dxo[0], s1);
    double s2 = -o_xp * dyp_p;
    s2 = fma(o_xm, dyp_m, s2);
    s2 = fma(o_yp, dxp[2], s2);
    s2 = fma(-o_ym, dxp[0], s2);
    const double lapx = fma(-2.0, wc, o_xp + o_xm);
    rhs = fma(nu_dx2, lapx, rhs);
    rhs = fma(ap, o_yp - wc, rhs);
    rhs = fma(-am, wc - o_ym, rhs);
    return fma(cj, s1 + s2, rhs);                                                         // -J = c_j S
}

__device__ __forceinline__ void stage_tile(const StageParams& p, const StageTime& st, const double* sp,
                                           const double* so, int ld, int coff, int x0, int y0,
                                           const double* swn = nullptr) {
    const int Nx = p.Nx, Ny = p.Ny;
    const int lx = threadIdx.x & (ST_TX - 1), g = threadIdx.x / ST_TX;
    const int i = x0 + lx;
    if (i >= Nx) return;
    const int ly0 = g * ST_RPT;                         // first local row (tile row ly0 <-> smem row ly0 + 1)
    const int cb = lx + coff;
    const double nu_dx2 = p.nu * p.inv_dx2;
    double ps[3][3], om[3][3], dxp[3], dxo[3];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c) { ps[r + 1][c] = sp[(ly0 + r) * ld + cb + c]; om[r + 1][c] = so[(ly0 + r) * ld + cb + c]; }
        dxp[r + 1] = ps[r + 1][2] - ps[r + 1][0];
        dxo[r + 1] = om[r + 1][2] - om[r + 1][0];
    }
#pragma unroll
    for (int q = 0; q < ST_RPT; ++q) {
        const int ly = ly0 + q, j = y0 + ly;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            ps[0][c] = ps[1][c]; ps[1][c] = ps[2][c]; ps[2][c] = sp[(ly + 2) * ld + cb + c];
            om[0][c] = om[1][c]; om[1][c] = om[2][c]; om[2][c] = so[(ly + 2) * ld + cb + c];
        }
        dxp[0] = dxp[1]; dxp[1] = dxp[2]; dxp[2] = ps[2][2] - ps[2][0];
        dxo[0] = dxo[1]; dxo[1] = dxo[2]; dxo[2] = om[2][2] - om[2][0];
        if (j >= Ny) break;
        const double wc = om[1][1];
        double rhs = fma(-p.lin_drag, wc, __ldg(&p.rt.frow[j]));                        // f - r omega
        if (j != 0 && j != Ny - 1) {
            const double dyo_m = om[2][0] - om[0][0], dyo_c = om[2][1] - om[0][1], dyo_p = om[2][2] - om[0][2];
            const double dyp_m = ps[2][0] - ps[0][0], dyp_c = ps[2][1] - ps[0][1], dyp_p = ps[2][2] - ps[0][2];
            const double ap = __ldg(&p.rt.st_ap[j]), am = __ldg(&p.rt.st_am[j]), cj = __ldg(&p.rt.st_cj[j]);
            rhs = stage_rhs_interior(rhs, wc, ps[1][0], ps[1][2], ps[0][1], ps[2][1], dyp_m, dyp_c, dyp_p, dxp,
                                     om[1][0], om[1][2], om[0][1], om[2][1], dyo_m, dyo_c, dyo_p, dxo,
                                     nu_dx2, ap, am, cj);
        }
        if (p.mms) rhs += mms_term(p, j, i, st.mA, st.mAp);
        const size_t id = (size_t)j * Nx + i;
        if (p.closure && j != 0 && j != Ny - 1) rhs -= __ldg(&p.closure[id]);
        if (p.rhs_out) p.rhs_out[id] = rhs;
        double wnew;
        const double dt = st.dt;
        if (p.stage == 1) {
            wnew = wc + dt * rhs;                                                          // ops.cu:646
        } else {
            const double wn = swn ? swn[ly * ST_TX + lx] : p.w_n[id];
            if (p.stage == 2) wnew = 0.75 * wn + 0.25 * (wc + dt * rhs);                   // ops.cu:650
            else wnew = (1.0 / 3.0) * wn + (2.0 / 3.0) * (wc + dt * rhs);                 // ops.cu:654
        }
        p.w_out[id] = wnew;
    }
}

// One CTA per tile, halo loaded with plain loads (used when Nx < 2 ST_TX).
static __global__ void __launch_bounds__(256) k_stage(StageParams p) {
    __shared__ double sp[ST_H][ST_W + 1];
    __shared__ double so[ST_H][ST_W + 1];
    pdl_begin();
    const int Nx = p.Nx, Ny = p.Ny;
    const int x0 = blockIdx.x * ST_TX, y0 = blockIdx.y * ST_TY;
    // all halo loads of a thread are issued before any of them is stored (fixed trip count)
    constexpr int NLD = (ST_H * ST_W + 255) / 256;
    {
        double vp[NLD], vo[NLD];
#pragma unroll
        for (int u = 0; u < NLD; ++u) {
            const int idx = threadIdx.x + 256 * u;
            const int r = idx / ST_W, c = idx - r * ST_W;
            const int gy = y0 - 1 + r;
            int gx = x0 - 1 + c;
            // x0 + ST_TX <= Nx when Nx >= ST_TX (Nx a power of two), so gx lies in [-1, Nx]
            gx = (Nx >= ST_TX) ? (gx < 0 ? gx + Nx : (gx >= Nx ? gx - Nx : gx)) : ((gx % Nx) + Nx) % Nx;
            vp[u] = 0.0;
            vo[u] = 0.0;
            if (idx < ST_H * ST_W && gy >= 0 && gy < Ny) {
                const size_t id = (size_t)gy * Nx + gx;
                vp[u] = __ldg(&p.psi[id]);
                vo[u] = __ldg(&p.w_in[id]);
            }
        }
#pragma unroll
        for (int u = 0; u < NLD; ++u) {
            const int idx = threadIdx.x + 256 * u;
            if (idx < ST_H * ST_W) {
                const int r = idx / ST_W, c = idx - r * ST_W;
                sp[r][c] = vp[u];
                so[r][c] = vo[u];
            }
        }
    }
    __syncthreads();
    stage_tile(p, stage_time(p), &sp[0][0], &so[0][0], ST_W + 1, 0, x0, y0);
}

// ---- k_stage_tma: persistent, with the halos moved by the tensor memory accelerator ----
// A CTA walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ...; the halo of the next tile is
// in flight (cp.async.bulk.tensor into the other of two buffers) while the current one is
// computed, together with the tile of omega^n in stages 2 and 3 (a third box, 64 x 32). The
// halo box starts at column x0 - 2 so that its x coordinate is a multiple of 16 bytes
// (68 columns x 34 rows, FP64); rows outside [0, Ny) and columns outside [0, Nx) arrive as
// zeros, and the periodic columns -1 and Nx of the first and last tile column are patched
// with plain loads once the box has landed. A wait that does not complete within
// kTmaWaitLimit polls sets bit 1 of the control block's error flags and ends the CTA (the next
// tile's copy is issued only after that wait, so no other copy is in flight).
constexpr int SB_W = ST_TX + 4, SB_H = ST_TY + 2;
constexpr int SB_FIELD = ((SB_H * SB_W * 8 + 127) / 128) * 128;     // bytes per field, 128-byte aligned
constexpr int SB_WN = ST_TX * ST_TY * 8;                          // omega^n tile (128-byte multiple)
constexpr int SB_BUF = 2 * SB_FIELD + SB_WN;                       // psi + omega halos, omega^n tile
constexpr unsigned SB_TX_BYTES = 2u * SB_H * SB_W * 8;             // bytes the two halo boxes deliver
constexpr unsigned kTmaWaitLimit = 1u << 22;
__host__ __device__ constexpr size_t stage_tma_smem_bytes() { return 2 * (size_t)SB_BUF + 128; }   // + alignment slack

struct StageMaps {
    CUtensorMap psi, w;      // halo boxes (SB_W x SB_H)
    CUtensorMap wn;          // omega^n tile box (ST_TX x ST_TY), stages 2 and 3
};

__device__ __forceinline__ unsigned smem_u32(const void* ptr) { return (unsigned)__cvta_generic_to_shared(ptr); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
    for (unsigned it = 0; it < kTmaWaitLimit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
        ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar)) : "memory");
}

// The points of one tile from the TMA box (row stride SB_W; box column b holds x = x0 - 2 + b),
// two adjacent columns per thread: warp g takes tile rows 4g .. 4g + 3, lane l the columns
// x0 + 2l and x0 + 2l + 1. A row of the window (columns x - 1 .. x + 2) is three 16-byte shared
// loads, the two points share their y differences, and the results leave as 16-byte stores.
// srow[q][r] holds the row tables frow, st_ap, st_am, st_cj (q = 0..3) of tile row r.
// The arithmetic of every point is stage_tile's (stage_rhs_interior), so both give the same bits.
constexpr int ST2_RPT = 4;
static_assert(8 * ST2_RPT == ST_TY && 64 == ST_TX, "pair layout: 8 warps x 4 rows, 32 lanes x 2 columns");

__device__ __forceinline__ void stage_tile2(const StageParams& p, const StageTime& st, const double* sp,
                                            const double* so, const double* swn, int x0, int y0,
                                            const double (*srow)[ST_TY]) {
    const int Nx = p.Nx, Ny = p.Ny;
    const int lp = threadIdx.x & 31, g = threadIdx.x >> 5;
    const int i0 = x0 + 2 * lp;
    const int ly0 = g * ST2_RPT;                        // tile row ly <-> box row ly + 1
    const double nu_dx2 = p.nu * p.inv_dx2;
    double P[3][4], O[3][4];                            // rows j-1, j, j+1 x columns i0-1 .. i0+2
    double dxpA[3], dxpB[3], dxoA[3], dxoB[3];          // x differences of the two points' rows
    auto ld_row = [&](const double* f, int r, double (&v)[4]) {
        const double2* q = reinterpret_cast<const double2*>(f + r * SB_W + 2 * lp);
        const double2 a = q[0], b = q[1], c = q[2];
        v[0] = a.y; v[1] = b.x; v[2] = b.y; v[3] = c.x;
    };
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        ld_row(sp, ly0 + r, P[r + 1]);
        ld_row(so, ly0 + r, O[r + 1]);
        dxpA[r + 1] = P[r + 1][2] - P[r + 1][0]; dxpB[r + 1] = P[r + 1][3] - P[r + 1][1];
        dxoA[r + 1] = O[r + 1][2] - O[r + 1][0]; dxoB[r + 1] = O[r + 1][3] - O[r + 1][1];
    }
#pragma unroll
    for (int q = 0; q < ST2_RPT; ++q) {
        const int ly = ly0 + q, j = y0 + ly;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            P[0][c] = P[1][c]; P[1][c] = P[2][c];
            O[0][c] = O[1][c]; O[1][c] = O[2][c];
        }
        ld_row(sp, ly + 2, P[2]);
        ld_row(so, ly + 2, O[2]);
        dxpA[0] = dxpA[1]; dxpA[1] = dxpA[2]; dxpA[2] = P[2][2] - P[2][0];
        dxpB[0] = dxpB[1]; dxpB[1] = dxpB[2]; dxpB[2] = P[2][3] - P[2][1];
        dxoA[0] = dxoA[1]; dxoA[1] = dxoA[2]; dxoA[2] = O[2][2] - O[2][0];
        dxoB[0] = dxoB[1]; dxoB[1] = dxoB[2]; dxoB[2] = O[2][3] - O[2][1];
        if (j >= Ny) break;
        const double wa = O[1][1], wb = O[1][2];
        const double fj = srow[0][ly];
        double ra = fma(-p.lin_drag, wa, fj), rb = fma(-p.lin_drag, wb, fj);              // f - r omega
        const bool interior = (j != 0 && j != Ny - 1);
        if (interior) {
            double dyo[4], dyp[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) { dyo[c] = O[2][c] - O[0][c]; dyp[c] = P[2][c] - P[0][c]; }
            const double ap = srow[1][ly], am = srow[2][ly], cj = srow[3][ly];
            ra = stage_rhs_interior(ra, wa, P[1][0], P[1][2], P[0][1], P[2][1], dyp[0], dyp[1], dyp[2], dxpA,
                                    O[1][0], O[1][2], O[0][1], O[2][1], dyo[0], dyo[1], dyo[2], dxoA, nu_dx2, ap, am, cj);
            rb = stage_rhs_interior(rb, wb, P[1][1], P[1][3], P[0][2], P[2][2], dyp[1], dyp[2], dyp[3], dxpB,
                                    O[1][1], O[1][3], O[0][2], O[2][2], dyo[1], dyo[2], dyo[3], dxoB, nu_dx2, ap, am, cj);
        }
        if (p.mms) {
            ra += mms_term(p, j, i0, st.mA, st.mAp);
            rb += mms_term(p, j, i0 + 1, st.mA, st.mAp);
        }
        const size_t id = (size_t)j * Nx + i0;
        if (p.closure && interior) {
            const double2 tau = __ldg(reinterpret_cast<const double2*>(p.closure + id));
            ra -= tau.x;
            rb -= tau.y;
        }
        if (p.rhs_out) *reinterpret_cast<double2*>(p.rhs_out + id) = make_double2(ra, rb);
        double na, nb;
        const double dt = st.dt;
        if (p.stage == 1) {
            na = wa + dt * ra;                                                              // ops.cu:646
            nb = wb + dt * rb;
        } else {
            const double2 wn = *reinterpret_cast<const double2*>(swn + ly * ST_TX + 2 * lp);
            if (p.stage == 2) {
                na = 0.75 * wn.x + 0.25 * (wa + dt * ra);                                   // ops.cu:650
                nb = 0.75 * wn.y + 0.25 * (wb + dt * rb);
            } else {
                na = (1.0 / 3.0) * wn.x + (2.0 / 3.0) * (wa + dt * ra);                    // ops.cu:654
                nb = (1.0 / 3.0) * wn.y + (2.0 / 3.0) * (wb + dt * rb);
            }
        }
        *reinterpret_cast<double2*>(p.w_out + id) = make_double2(na, nb);
    }
}

static __global__ void __launch_bounds__(256, 2) k_stage_tma(const __grid_constant__ StageMaps maps, StageParams p) {
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    pdl_begin();
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ double srow[2][4][ST_TY];                // per buffer: the row tables of its tile
    // the boxes land at 128-byte aligned shared addresses
    unsigned char* smem_raw = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);
    const int Nx = p.Nx, Ny = p.Ny;
    const int tiles_x = Nx / ST_TX, ntiles = tiles_x * ((Ny + ST_TY - 1) / ST_TY);
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        fence_proxy_async_smem();
    }
    __syncthreads();
    auto issue = [&](int tile, int b) {
        const int tx = tile % tiles_x, ty = tile / tiles_x;
        unsigned char* dst = smem_raw + b * SB_BUF;
        mbar_expect_tx(&bars[b], SB_TX_BYTES + (p.stage > 1 ? (unsigned)SB_WN : 0u));
        tma_load_2d(dst, &maps.psi, tx * ST_TX - 2, ty * ST_TY - 1, &bars[b]);
        tma_load_2d(dst + SB_FIELD, &maps.w, tx * ST_TX - 2, ty * ST_TY - 1, &bars[b]);
        if (p.stage > 1) tma_load_2d(dst + 2 * SB_FIELD, &maps.wn, tx * ST_TX, ty * ST_TY, &bars[b]);
    };
    const StageTime st = stage_time(p);
    int k = 0;
    if (threadIdx.x == 0 && (int)blockIdx.x < ntiles) issue(blockIdx.x, 0);
    // One barrier per tile: it finds this tile's box landed, orders the table values staged
    // before it, and tells thread 0 that every thread is done with the other buffer (the
    // previous tile, whose reads each thread fenced against the async proxy), so that the next
    // tile's box may be issued into it.
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++k) {
        const int b = k & 1;
        const int next = tile + gridDim.x;
        const int tx = tile % tiles_x, ty = tile / tiles_x;
        const int x0 = tx * ST_TX, y0 = ty * ST_TY;
        if (threadIdx.x < 4 * ST_TY) {                   // the tile rows' table values (read by stage_tile2)
            const int q = threadIdx.x / ST_TY, r = threadIdx.x % ST_TY, jr = min(y0 + r, Ny - 1);
            const double* tab = q == 0 ? p.rt.frow : (q == 1 ? p.rt.st_ap : (q == 2 ? p.rt.st_am : p.rt.st_cj));
            srow[b][q][r] = __ldg(&tab[jr]);
        }
        const bool ok = __syncthreads_and(mbar_wait_bounded(&bars[b], (k >> 1) & 1));
        if (!ok) {                                       // nothing else is in flight
            if (threadIdx.x == 0) atomicOr(const_cast<int*>(&p.ctl->nonfinite), 2);
            return;
        }
        if (threadIdx.x == 0 && next < ntiles) issue(next, b ^ 1);
        double* sp = reinterpret_cast<double*>(smem_raw + b * SB_BUF);
        double* so = reinterpret_cast<double*>(smem_raw + b * SB_BUF + SB_FIELD);
        if (tx == 0 || tx == tiles_x - 1) {
            // periodic halo columns: box column 1 is x = -1, box column ST_TX + 2 is x = Nx
            for (int r = threadIdx.x; r < SB_H; r += blockDim.x) {
                const int gy = y0 - 1 + r;
                if (gy < 0 || gy >= Ny) continue;
                if (tx == 0) {
                    sp[r * SB_W + 1] = __ldg(&p.psi[(size_t)gy * Nx + Nx - 1]);
                    so[r * SB_W + 1] = __ldg(&p.w_in[(size_t)gy * Nx + Nx - 1]);
                }
                if (tx == tiles_x - 1) {
                    sp[r * SB_W + ST_TX + 2] = __ldg(&p.psi[(size_t)gy * Nx]);
                    so[r * SB_W + ST_TX + 2] = __ldg(&p.w_in[(size_t)gy * Nx]);
                }
            }
            __syncthreads();                             // tx is the same for the whole CTA
        }
        stage_tile2(p, st, sp, so, reinterpret_cast<const double*>(smem_raw + b * SB_BUF + 2 * SB_FIELD), x0, y0,
                    srow[b]);
        fence_proxy_async_smem();                        // reads of buffer b before its next TMA write
    }
}

// t += dt, step++, and the snap to the scheduled output times (src/main.cu:541-551): the
// tolerance is re-evaluated after the first snap, as the reference does.
__device__ __forceinline__ void advance_time(Ctl* ctl) {
    const double dt = ctl->dt;
    double t = ctl->t + dt;
    const double ns = ctl->next_snap, nd = ctl->next_diag;
    if (ns < 1e299 && fabs(t - ns) <= fmax(time_tol_d(t), 1e-6 * fmax(1e-300, fabs(dt)))) t = ns;
    if (nd < 1e299 && fabs(t - nd) <= fmax(time_tol_d(t), 1e-6 * fmax(1e-300, fabs(dt)))) t = nd;
    ctl->t = t;
    ctl->step += 1;
    if (ctl->run) {
        // the host's output and loop tests of src/main.cu:434,553-566,695 after this step
        // (with the wider snapshot tolerance, so that no due output is missed)
        const double tol = fmax(time_tol_d(t), 1e-6 * fmax(1e-300, fabs(dt)));
        int r = 0;
        if (fmin(ns, nd) < 1e299 && t + tol >= fmin(ns, nd)) r |= 1;
        if (ctl->stats_every > 0 && (ctl->step % ctl->stats_every) == 0) r |= 2;
        if (!(t < ctl->t_end - 0.5 * dt)) r |= 4;
        if (ctl->nonfinite & 2) r |= 8;     // a bounded wait gave up
        // the first NaN or Inf a reduction meets halts the run once, so that the host sees it; the
        // run may then go on, as the reference's loop does with non-finite fields
        if ((ctl->nonfinite & 1) && !ctl->nonfinite_halted) {
            r |= 8;
            ctl->nonfinite_halted = 1;
        }
        if (r) {
            ctl->halt = 1;
            ctl->halt_reason = r;
        }
    }
}

// ---- row FFT kernels ----
struct FftParams {
    const double* src;       // forward: real rows [Ny][Nx]
    cpx<double>* hat;        // [Ny][Hp]
    double* psi;             // inverse output [Ny][Nx]
    const cpx<double>* tw;   // per-pass twiddles of the radix-16 plan (p16_twiddle_table)
    const cpx<double>* wN;   // M + 1 twiddles e^{-2 pi i k/Nx} of the split/merge step
    int Nx, Ny, Hp;
    int row0, nrows;         // forward: transform rows row0 .. row0 + nrows - 1
    // inverse only: Thom closure (src/ops.cu:102-158) and the closure_diag wall bookkeeping
    double* w;               // omega^(s+1): wall rows rewritten
    const double* dy_edge;
    const double* w_node;
    Ctl* ctl;
    int free_slip, closure, stage, do_thom, advance;
    double psi_bot, psi_top, invA_full;
    // fuse_max (the stage-3 launch of an adaptive step): max |u|, |v|, |v| a of the psi written,
    // for the next step's dt; bcount [grid + 1] arrival counters of the band boundaries
    int fuse_max;
    const double* a_node;
    unsigned int* bcount;
    double inv_dx, inv_deta;
};


__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Row FFT kernels: one CTA of IP_NT threads transforms one row at a time in ONE shared buffer
// (in-place decimation-in-time passes, fft_rows.cuh), so that 5 CTAs fit on an SM and the
// load latency of one row is hidden behind the passes of the others.
// 16-byte read-only load that does not allocate in L1 (rows read once, so that they do not
// evict the twiddle tables the passes read from L1)
__device__ __forceinline__ double2 ld_na(const double2* p) {
    double2 v;
    asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ float2 ld_na(const float2* p) {
    float2 v;
    asm("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
    return v;
}

constexpr int IP_NT = 128;
__host__ __device__ constexpr size_t fft_smem_bytes(int M) { return (size_t)ip_size(M) * 16; }

// The last pass of the forward transform at M = 16 IP_NT (= 2048) fused with the split step.
// The last pass (radix 8, LP = 256) has butterflies mm = 0..255 holding Z_{mm + 256 r}; thread t
// takes mm = t and its mirror 256 - t (thread 0: 0 and 128), so that every pair (Z_k, Z_{M-k})
// of the split is in one thread's registers:
//   t >= 1: k = t + 256 r with Z_{M-k} = B[7 - r], and k = 256 - t + 256 r with Z_{M-k} = A[7 - r];
//   t = 0:  k = 256 r with Z_{M-k} = A[(8 - r) & 7] (r = 0 is the X_0 / X_M pair, and k = 1024
//           pairs with itself), and k = 128 + 256 r with Z_{M-k} = B[7 - r];  r = 0..3.
// X_k and X_{M-k} leave from registers; the split twiddles W_2M^k come from W_2M^t and the
// e^{-i pi j/16} constants. The buffer is only read here.
template <typename T, int M, typename D2>
__device__ __forceinline__ void fwd_last_pass_split(const cpx<T>* buf, const cpx<T>* tw, const cpx<T>* wN,
                                                    D2* dst) {
    static_assert(M == 16 * IP_NT && p16_plan<M>::P == 3 && p16_plan<M>::R(2) == 8 && p16_plan<M>::LP(2) == 256,
                  "the fused split is written for M = 2048 (passes 16, 16, 8)");
    const int t = threadIdx.x;
    cpx<T> A[8], B[8];
    p16_bfly<T, M, 2, false>(buf, tw, t, A);
    p16_bfly<T, M, 2, false>(buf, tw, t == 0 ? 128 : 256 - t, B);
    // X_k = s/2 + (W^k/2)(-i d), X_{M-k} = conj(s)/2 + (-conj(W^k)/2)(i conj d) with
    // s = Z_k + conj Z_{M-k}, d = Z_k - conj Z_{M-k}; wk is W^k / 2
    auto split = [&](int k, const cpx<T>& a, const cpx<T>& b, const cpx<T>& wk) {
        const cpx<T> sm = {(T)0.5 * (a.x + b.x), (T)0.5 * (a.y - b.y)};
        const cpx<T> df = {a.x - b.x, a.y + b.y};
        const cpx<T> X = cadd(sm, cmul(wk, mul_mi(df)));
        dst[k] = D2{X.x, X.y};
        if (k < M / 2) {
            const cpx<T> wm = {-wk.x, wk.y};
            const cpx<T> Y = cadd(cpx<T>{sm.x, -sm.y}, cmul(wm, cpx<T>{df.y, df.x}));
            dst[M - k] = D2{Y.x, Y.y};
        }
    };
    const cpx<T> w1 = ldtw(wN, t);
    const cpx<T> wh = {(T)0.5 * w1.x, (T)0.5 * w1.y};                 // W^t / 2 (exact halving)
    const cpx<T> whc = {wh.x, -wh.y};                                   // conj(W^t) / 2
    const cpx<T> half = {(T)0.5, (T)0};
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const cpx<T> bA = (t == 0) ? A[(8 - r) & 7] : B[7 - r];
        split(t + 256 * r, A[r], bA, r == 0 ? wh : cmul(wh, w32<T>(2 * r)));
        const cpx<T> wB = (t == 0) ? cmul(half, w32<T>(1 + 2 * r)) : cmul(whc, w32<T>(2 + 2 * r));
        split((t == 0 ? 128 : 256 - t) + 256 * r, B[r], (t == 0) ? B[7 - r] : A[7 - r], wB);
    }
    if (t == 0) split(M / 2, A[4], A[4], cmul(half, w32<T>(8)));
}

// Forward real FFT of rows row0 .. row0 + nrows - 1: rows 1..Ny-2 in the Poisson solve (the
// reference's pack + cuFFT forward, src/poisson.cuh:93-96), all rows for the 1-D spectra:
// a row is read as M complex points z_n = x_2n + i x_2n+1, scattered by cp.async into the
// digit-reversed layout; after the passes the split step writes X_k, k = 0..M:
//   E_k = (Z_k + conj Z_{M-k}) / 2,  O_k = -i (Z_k - conj Z_{M-k}) / 2,  X_k = E_k + W_{2M}^k O_k.
template <int M>
static __global__ void __launch_bounds__(IP_NT, 5) k_fft_fwd(FftParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_begin();
    cpx<double>* buf = reinterpret_cast<cpx<double>*>(smem_raw);
    const int je = p.row0 + p.nrows;
    constexpr int R0 = p16_plan<M>::R(0), NB0 = M / R0;
    for (int j = p.row0 + blockIdx.x; j < je; j += gridDim.x) {      // rows strided over one wave of CTAs
        const double2* row = reinterpret_cast<const double2*>(p.src + (size_t)j * p.Nx);
        // pass 0 from global: thread t transforms the points t + NB0 r (a coalesced column)
#pragma unroll 1
        for (int b0 = 0; b0 < NB0; b0 += IP_NT) {
            const int t = b0 + (int)threadIdx.x;
            if (NB0 % IP_NT != 0 && t >= NB0) break;
            cpx<double> v[R0];
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const double2 z = ld_na(row + t + NB0 * r);
                v[r] = {z.x, z.y};
            }
            dftR<double, R0, false>(v);
            const int p0 = dit16_pos<M>(t);
#pragma unroll
            for (int q = 0; q < R0; ++q) buf[ip_idx<M>(p0 + q)] = v[q];
        }
        __syncthreads();
        double2* dst = reinterpret_cast<double2*>(p.hat + (size_t)j * p.Hp);
        if constexpr (M == 16 * IP_NT) {
            p16_pass<double, M, 1, false, IP_NT>(buf, p.tw);
            __syncthreads();
            fwd_last_pass_split<double, M>(buf, p.tw, p.wN, dst);
        } else {
            p16_passes_from<double, M, 1, false, IP_NT>(buf, p.tw);
            // X_k and X_{M-k} from one pair: with s = Z_k + conj Z_{M-k}, d = Z_k - conj Z_{M-k},
            //   X_k = s/2 + W^k (-i d)/2,   X_{M-k} = conj(s)/2 + W^{M-k} (i conj d)/2
            // (k = 0 pairs Z_0 with itself and gives X_0 and X_M; k = M/2 is its own pair).
            // wk is W^k / 2: the halving of d moves into the twiddle (exact, the same bits)
            auto split = [&](int k, const cpx<double>& wk) {
                const int kb = (k == 0 ? 0 : M - k);
                const cpx<double> a = buf[ip_idx<M>(k)];
                const cpx<double> b = buf[ip_idx<M>(kb)];
                const cpx<double> sm = {0.5 * (a.x + b.x), 0.5 * (a.y - b.y)};     // s/2
                const cpx<double> df = {a.x - b.x, a.y + b.y};                     // d
                const cpx<double> X = cadd(sm, cmul(wk, mul_mi(df)));
                dst[k] = make_double2(X.x, X.y);
                if (k < M / 2) {
                    const int m = M - k;                                           // m = M when k = 0
                    const cpx<double> wm = {-wk.x, wk.y};                          // W^{M-k} = -conj(W^k)
                    const cpx<double> Y = cadd(cpx<double>{sm.x, -sm.y}, cmul(wm, cpx<double>{df.y, df.x}));
                    dst[m] = make_double2(Y.x, Y.y);
                }
            };
#pragma unroll 2
            for (int k = threadIdx.x; k <= M / 2; k += IP_NT) {
                const cpx<double> w1 = ldtw(p.wN, k);
                split(k, cpx<double>{0.5 * w1.x, 0.5 * w1.y});
            }
        }
        __syncthreads();                                 // the buffer read before the next row's pass 0
    }
}

// Thom wall vorticity of one wall (src/ops.cu:114-151) from the psi rows this CTA just wrote,
// with the closure_diag enstrophy jump of the wall row (src/main.cu:271-298). One CTA writes the
// whole wall row while the other CTAs of the launch finish their bands, so its loads (psi rows
// from L2, the old wall row) are issued CH columns per thread at a time, all before any store:
// a loop of one column per iteration would wait for L2 once per column and hold the whole launch
// up by tens of microseconds at Nx = 4096. CH is set by the caller's register budget.
template <int NT, int CH>
__device__ __forceinline__ void thom_row(const FftParams& p, bool top) {
    const int Nx = p.Nx, Ny = p.Ny;
    const double d1 = top ? p.dy_edge[Ny - 2] : p.dy_edge[0];
    const double d2 = top ? p.dy_edge[Ny - 3] : p.dy_edge[1];
    const double A = 2.0 * (1.0 / (d1 * d1) + 1.0 / (d1 * d2));
    const double B = (-2.0) * d1 / (d2 * (d1 + d2) * (d1 + d2));
    const double pw = top ? p.psi_top : p.psi_bot;
    const double* r1 = p.psi + (size_t)(top ? Ny - 2 : 1) * Nx;
    const double* r2 = p.psi + (size_t)(top ? Ny - 3 : 2) * Nx;
    double* wr = p.w + (size_t)(top ? Ny - 1 : 0) * Nx;
    const double wq = p.closure ? p.w_node[top ? Ny - 1 : 0] : 0.0;
    double sb = 0.0, sa = 0.0;
    for (int i0 = threadIdx.x; i0 < Nx; i0 += NT * CH) {
        double a1[CH], a2[CH], ov[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const int i = i0 + c * NT;
            if (i < Nx) {
                a1[c] = __ldcg(&r1[i]);
                a2[c] = __ldcg(&r2[i]);
                ov[c] = wr[i];
            }
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const int i = i0 + c * NT;
            if (i < Nx) {
                double nv = 0.0;
                if (!p.free_slip) nv = -(A * (a1[c] - pw) + B * (a2[c] - pw));
                wr[i] = nv;
                sb += wq * ov[c] * ov[c];
                sa += wq * nv * nv;
            }
        }
    }
    if (!p.closure) return;
    __shared__ double rb[NT], ra[NT];
    rb[threadIdx.x] = sb; ra[threadIdx.x] = sa;
    __syncthreads();
    for (int s = NT / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) { rb[threadIdx.x] += rb[threadIdx.x + s]; ra[threadIdx.x] += ra[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(&p.ctl->jwall[p.stage - 1], 0.5 * ra[0] * p.invA_full - 0.5 * rb[0] * p.invA_full);
    __syncthreads();
}

// Contiguous row bands of L rows; the last band also takes a short remainder. With L >= 3
// and Ny >= 5 the first band holds rows 0..2 and the last band rows Ny-3..Ny-1.
__host__ __device__ __forceinline__ void band_of(int b, int nb, int L, int Ny, int& j0, int& j1) {
    j0 = b * L;
    j1 = (b == nb - 1) ? Ny : min(Ny, (b + 1) * L);
}

// Inverse real FFT of every row (the reference's cuFFT inverse + scale, src/poisson.cuh:110-114):
// the merge step forms Z_k = E_k + i O_k, E_k = (X_k + conj X_{M-k}) / 2,
// O_k = (X_k - conj X_{M-k}) W_{2M}^{-k} / 2, straight from HBM into the registers of the first
// (radix-16) pass; the passes give z_n = x_2n + i x_2n+1 (times M). The Thom closure of
// omega^(s+1) is applied by the CTA that writes the second of rows 1-2 (bottom) or
// Ny-3..Ny-2 (top), and, in the stage-3 launch, the last CTA advances the time.
template <int M>
static __global__ void __launch_bounds__(IP_NT, 5) k_ifft_thom(FftParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_begin();
    cpx<double>* buf = reinterpret_cast<cpx<double>*>(smem_raw);
    __shared__ bool thom_now;
    const int Nx = p.Nx, Ny = p.Ny;
    constexpr double scale = 0.5 / (double)M;          // the merge forms 2 Z_n (see below)
    constexpr int R0 = p16_plan<M>::R(0), NB0 = M / R0;
    constexpr bool kPairLanes = (NB0 == IP_NT) && (R0 == 16) && (IP_NT == 128);   // M = 2048
    int j0, j1;
    // an even split of the rows over one wave of CTAs: bands of floor or ceil(Ny / grid) rows,
    // the longer ones spread over the grid, so that every SM gets about the same number of rows
    j0 = (int)(((long long)blockIdx.x * Ny) / gridDim.x);
    j1 = (int)(((long long)(blockIdx.x + 1) * Ny) / gridDim.x);
    for (int j = j0; j < j1; ++j) {                                   // a contiguous band of rows
        double* dst = p.psi + (size_t)j * Nx;
        if (j == 0 || j == Ny - 1) {
            const double v = (j == 0) ? p.psi_bot : p.psi_top;
            for (int i = threadIdx.x; i < Nx; i += IP_NT) dst[i] = v;
            continue;
        }
        // pass 0 from global with the merge: thread t forms 2 Z_n, n = t + NB0 r, from X_n and
        // X_{M-n} (s = X_n + conj X_{M-n}, d = X_n - conj X_{M-n}, 2 Z_n = s + i d conj(W^n)) and
        // transforms them in registers. The factor 2 is exact, it scales every later value by
        // exactly 2, and the output scale 1/(2M) removes it, so the bits are those of Z_n.
        const double2* X = reinterpret_cast<const double2*>(p.hat + (size_t)j * p.Hp);
        if constexpr (kPairLanes) {
            // Butterfly b of a thread: lanes 0..15 of warp w take b = 16 w + l, lanes 16..31 the
            // mirrors 128 - b (lane 16 of warp 0, whose mirror would be b = 0 again, takes b = 64).
            // The mirror point of n = b + 128 r is M - n = (128 - b) + 128 (15 - r), a point of the
            // partner lane (l ^ 16): each thread loads only its own 16 points and gets the mirrors
            // by shuffle. b = 64 is its own mirror (r <-> 15 - r); b = 0 mirrors r to 16 - r, and
            // r = 0 to X_M, which it loads.
            const int w = (int)threadIdx.x >> 5, l = (int)threadIdx.x & 31;
            int b = (l < 16) ? 16 * w + l : 128 - (16 * w + l - 16);
            if (b == 128) b = 64;
            double2 x[16];
#pragma unroll
            for (int r = 0; r < 16; ++r) x[r] = __ldcs(X + b + 128 * r);
            const double2 xM = (b == 0) ? __ldcs(X + M) : make_double2(0.0, 0.0);
            // W_{2M}^n for n = b + 128 r is W_{2M}^b e^{-i pi r/16} (one table load per thread)
            const cpx<double> wt = ldtw(p.wN, b);
            auto merge = [&](const double2& av, const double2& bv, int r) {
                const cpx<double> sm = {av.x + bv.x, av.y - bv.y};
                const cpx<double> df = {av.x - bv.x, av.y + bv.y};
                const cpx<double> wn = (r == 0) ? wt : cmul(wt, w32<double>(r));
                return cadd(sm, mul_pi(cmulc(df, wn)));
            };
            cpx<double> v[16];
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int r2 = 15 - r;
                double2 ma, mb;                          // the mirrors of the points r and 15 - r
                ma.x = __shfl_xor_sync(0xffffffffu, x[r2].x, 16);
                ma.y = __shfl_xor_sync(0xffffffffu, x[r2].y, 16);
                mb.x = __shfl_xor_sync(0xffffffffu, x[r].x, 16);
                mb.y = __shfl_xor_sync(0xffffffffu, x[r].y, 16);
                if (b == 64) { ma = x[r2]; mb = x[r]; }
                if (b == 0) { ma = (r == 0) ? xM : x[16 - r]; mb = x[r + 1]; }
                v[r] = merge(x[r], ma, r);
                v[r2] = merge(x[r2], mb, r2);
            }
            dftR<double, 16, true>(v);
            const int p0 = dit16_pos<M>(b);
#pragma unroll
            for (int q = 0; q < 16; ++q) buf[ip_idx<M>(p0 + q)] = v[q];
        } else {
#pragma unroll 1
        for (int b0 = 0; b0 < NB0; b0 += IP_NT) {
            const int t = b0 + (int)threadIdx.x;
            if (NB0 % IP_NT != 0 && t >= NB0) break;
            cpx<double> v[R0];
            // W_{2M}^n for n = t + NB0 r is W_{2M}^t e^{-i pi r/16} (one table load per thread)
            const cpx<double> wt = ldtw(p.wN, t);
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int n = t + NB0 * r;
                const double2 av = __ldcs(X + n), bv = __ldcs(X + (M - n));
                const cpx<double> sm = {av.x + bv.x, av.y - bv.y};
                const cpx<double> df = {av.x - bv.x, av.y + bv.y};
                const cpx<double> wn = (R0 == 16) ? (r == 0 ? wt : cmul(wt, w32<double>(r))) : ldtw(p.wN, n);
                v[r] = cadd(sm, mul_pi(cmulc(df, wn)));
            }
            dftR<double, R0, true>(v);
            const int p0 = dit16_pos<M>(t);
#pragma unroll
            for (int q = 0; q < R0; ++q) buf[ip_idx<M>(p0 + q)] = v[q];
        }
        }
        __syncthreads();
        if constexpr (p16_plan<M>::P >= 2) {
            // the last pass stores z_n = x_2n + i x_2n+1 straight from registers
            p16_passes_to<double, M, 1, true, IP_NT>(buf, p.tw, [&](int n, const cpx<double>& z) {
                reinterpret_cast<double2*>(dst)[n] = make_double2(z.x * scale, z.y * scale);
            });
        } else {
            p16_passes_from<double, M, 1, true, IP_NT>(buf, p.tw);
            for (int n = threadIdx.x; n < M; n += IP_NT) {
                const cpx<double> z = buf[ip_idx<M>(n)];
                reinterpret_cast<double2*>(dst)[n] = make_double2(z.x * scale, z.y * scale);
            }
        }
        __syncthreads();
        if (p.do_thom) {
            // rows 1, 2 close the bottom wall and rows Ny-3, Ny-2 the top one: the CTA that
            // writes the second row of a wall applies its Thom closure (an arrival count per
            // wall, reset by that CTA)
            const bool bot = (j == 1 || j == 2), top = (j == Ny - 3 || j == Ny - 2);
            if (bot || top) {
                __threadfence();                             // this row before the arrival count
                __syncthreads();
                for (int wall = 0; wall < 2; ++wall) {
                    if (!(wall == 0 ? bot : top)) continue;
                    if (threadIdx.x == 0) thom_now = (atomicAdd(&p.ctl->thom_done[wall], 1u) == 1u);
                    __syncthreads();
                    if (thom_now) {
                        __threadfence();
                        thom_row<IP_NT, 2>(p, wall == 1);
                        if (threadIdx.x == 0) p.ctl->thom_done[wall] = 0;
                    }
                    __syncthreads();
                }
            }
        }
    }
    if (p.advance) {
        // the last CTA to finish advances the time: t += dt and the output snap
        __shared__ bool last;
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            last = (atomicAdd(&p.ctl->ifft_done, 1u) == gridDim.x - 1);
        }
        __syncthreads();
        if (last && threadIdx.x == 0) {
            p.ctl->ifft_done = 0;
            advance_time(p.ctl);
        }
    }
}

// The inverse transform at M = 2048 with the spectral rows prefetched: a bulk copy
// (cp.async.bulk, completion on an mbarrier) brings row j+1's X_0..X_M into a shared staging
// buffer while row j is transformed, so pass 0 reads X_n and X_{M-n} from shared memory instead
// of waiting on global loads. Thread t takes the pass-0 butterfly t (points t + 128 r) with the
// same merge and DFT as k_ifft_thom; compiled in another kernel, where the compiler may fuse other
// multiply-adds, it gives psi to round-off (not the same bits).
// The staging buffer is read in pass 0 only; after the barrier that ends pass 0, thread 0 issues
// the next row's copy into it. Three CTAs of 66 KB per SM. Every wait is bounded: a wait that
// runs out sets bit 1 of the non-finite flag, no further copy is issued, and the CTA waits once
// more (bounded) for the copy in flight before it exits.
template <int M> struct IfftPf {
    static constexpr size_t stage_off = ((size_t)ip_size(M) * 16 + 127) / 128 * 128;
    static constexpr unsigned row_bytes = (unsigned)(M + 1) * 16u;
    static constexpr size_t bar_off = (stage_off + row_bytes + 15) / 16 * 16;
    static constexpr size_t smem = bar_off + 16;
};
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

// The max reductions take 60-column strips per warp: lanes 1..30 own two columns each, lanes 0
// and 31 hold the outer neighbours (k_maxuv_dt, maxuv_rows).
constexpr int MX_WCOLS = 60, MX_COLS = 8 * MX_WCOLS;

// max |u|, |v|, |v| a and the non-finite probe of the interior rows ja..jb of psi, by the warps of a
// CTA over 60-column strips, with the per-point arithmetic of k_maxuv_dt (the same maxima for the
// same psi). A strip's rows ja-1..jb+1 (at most MX_RB + 2 at a time) and two strips per warp are
// loaded before any is reduced, so up to 2 (MX_RB + 2) 16-byte loads per lane are in flight: the
// rows were written earlier in the same launch and come from L2, where the reduction is bound by
// latency. Nx even, psi 16-byte aligned; all threads of the CTA call it with the same ja, jb.
constexpr int MX_RB = 8;
__device__ __forceinline__ void maxuv_rows(const double* __restrict__ psi, const double* __restrict__ a_node, int Nx,
                                           int ja, int jb, double cx, double cy,
                                           double& um, double& vm, double& vmm, double& probe) {
    const int lane = (int)threadIdx.x & 31, warp = (int)threadIdx.x >> 5, nw = (int)blockDim.x >> 5;
    for (int j = ja; j <= jb; j += MX_RB) {
        const int n = min(MX_RB, jb - j + 1);          // rows j..j+n-1, loads of rows j-1..j+n
        const double* r0 = psi + (size_t)(j - 1) * Nx;
        for (int base = warp * MX_WCOLS; base < Nx; base += 2 * nw * MX_WCOLS) {
            double2 w[2][MX_RB + 2];
            int ca[2];
            bool own[2];
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const int c = base + s * nw * MX_WCOLS + 2 * (lane - 1);
                own[s] = lane >= 1 && lane <= 30 && c < Nx;
                ca[s] = ((c % Nx) + Nx) % Nx;
            }
            const bool second = base + nw * MX_WCOLS < Nx;   // warp-uniform
#pragma unroll
            for (int r = 0; r < MX_RB + 2; ++r)
                if (r < n + 2) {
                    w[0][r] = __ldcg(reinterpret_cast<const double2*>(r0 + (size_t)r * Nx + ca[0]));
                    if (second) w[1][r] = __ldcg(reinterpret_cast<const double2*>(r0 + (size_t)r * Nx + ca[1]));
                }
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                if (s == 1 && !second) break;
#pragma unroll
                for (int r = 1; r <= MX_RB; ++r) {
                    if (r > n) break;
                    const double2 wm = w[s][r - 1], wc = w[s][r], wp = w[s][r + 1];
                    const double xl = __shfl_up_sync(0xffffffffu, wc.y, 1);      // column c - 1
                    const double xr = __shfl_down_sync(0xffffffffu, wc.x, 1);    // column c + 2
                    if (own[s]) {
                        const double a = __ldg(&a_node[j + r - 1]);
                        const double e0 = wp.x - wm.x, e1 = wp.y - wm.y;
                        const double f0 = wc.y - xl, f1 = xr - wc.x;
                        probe += (e0 + f0) + (e1 + f1);
                        const double dym = nn_max(fabs(e0), fabs(e1)), dxm = nn_max(fabs(f0), fabs(f1));
                        const double av = dxm * cx;
                        um = nn_max(um, a * (dym * cy));
                        vm = nn_max(vm, av);
                        vmm = nn_max(vmm, av * a);
                    }
                }
            }
        }
    }
}

// The max reduction of the rows of an inverse-transform launch whose bands hold two or more rows,
// after the CTA has stored its band [j0, j1). The two rows next to a band boundary (jb - 1, jb)
// are reduced by the second of the two CTAs to arrive at that boundary's counter, which then
// finds both bands stored (the Thom closure's arrival pattern, with no waiting); the CTA's rows
// j0 < j < j1 - 1 have their neighbours in its own band. So a CTA reduces one contiguous range of
// rows: from j0 - 1 (it arrived second at its lower boundary) or j0 + 1, to j1 (second at its
// upper boundary) or j1 - 2. The CTA maxima go to the control block by atomic maxima on their bit
// patterns; NaN or Inf sets bit 0 of the non-finite flag. All threads call it.
__device__ __forceinline__ void band_maxuv(const FftParams& p, int j0, int j1) {
    __shared__ int bnd[2];
    __shared__ double red[3][IP_NT / 32];
    const int Ny = p.Ny;
    double um = 0.0, vm = 0.0, vmm = 0.0, probe = 0.0;
    __threadfence();                                   // this CTA's rows before its boundary arrivals
    __syncthreads();
    if (threadIdx.x == 0) {
        bnd[0] = (blockIdx.x > 0) && (atomicAdd(&p.bcount[blockIdx.x], 1u) == 1u);
        bnd[1] = (blockIdx.x + 1 < gridDim.x) && (atomicAdd(&p.bcount[blockIdx.x + 1], 1u) == 1u);
        if (bnd[0] || bnd[1]) __threadfence();         // the neighbour band's rows after its arrival
    }
    __syncthreads();
    const int ja = max(bnd[0] ? j0 - 1 : j0 + 1, 1);
    const int jb = min(bnd[1] ? j1 : j1 - 2, Ny - 2);
    if (ja <= jb) maxuv_rows(p.psi, p.a_node, p.Nx, ja, jb, 0.5 * p.inv_dx, 0.5 * p.inv_deta, um, vm, vmm, probe);
    const int lane = (int)threadIdx.x & 31, warp = (int)threadIdx.x >> 5;
    um = warp_max_nn(um); vm = warp_max_nn(vm); vmm = warp_max_nn(vmm);
    if (lane == 0) { red[0][warp] = um; red[1][warp] = vm; red[2][warp] = vmm; }
    const int anynf = __syncthreads_or(!(probe - probe == 0.0) || !(um <= 1e300) || !(vm <= 1e300));
    if (threadIdx.x == 0) {
        for (int k = 0; k < 2; ++k)
            if (bnd[k]) p.bcount[blockIdx.x + k] = 0;  // the second arrival resets the counter
        double m[3] = {0.0, 0.0, 0.0};
        for (int w = 0; w < IP_NT / 32; ++w)
            for (int q = 0; q < 3; ++q) m[q] = nn_max(m[q], red[q][w]);
        unsigned long long* acc = p.ctl->mx_acc;
        for (int q = 0; q < 3; ++q) atomicMax(&acc[q], (unsigned long long)__double_as_longlong(m[q]));
        if (anynf) atomicOr(&p.ctl->nonfinite, 1);
    }
    __syncthreads();
}

// The forward transform at M = 2048 with its real rows prefetched the same way: a bulk copy brings
// row j + grid's Nx reals into a shared staging buffer while row j is transformed; pass 0 reads
// z_n = x_2n + i x_2n+1 from shared memory. The arithmetic is k_fft_fwd's, in the same order.
template <int M> struct FftPf {
    static constexpr size_t stage_off = ((size_t)ip_size(M) * 16 + 127) / 128 * 128;
    static constexpr unsigned row_bytes = (unsigned)M * 16u;
    static constexpr size_t bar_off = stage_off + row_bytes;
    static constexpr size_t smem = bar_off + 16;
};

template <int M>
static __global__ void __launch_bounds__(IP_NT, 3) k_fft_fwd_pf(FftParams p) {
    static_assert(M / 16 == IP_NT && p16_plan<M>::R(0) == 16 && M == 16 * IP_NT, "one pass-0 butterfly per thread");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_begin();
    cpx<double>* buf = reinterpret_cast<cpx<double>*>(smem_raw);
    const double2* stage = reinterpret_cast<const double2*>(smem_raw + FftPf<M>::stage_off);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + FftPf<M>::bar_off);
    const int je = p.row0 + p.nrows;
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        fence_proxy_async_smem();
    }
    __syncthreads();
    auto issue = [&](int j) {
        mbar_expect_tx(bar, FftPf<M>::row_bytes);
        bulk_load(const_cast<double2*>(stage), p.src + (size_t)j * p.Nx, FftPf<M>::row_bytes, bar);
    };
    const int jfirst = p.row0 + blockIdx.x;
    if (threadIdx.x == 0 && jfirst < je) issue(jfirst);
    unsigned parity = 0;
    bool live = true;
    for (int j = jfirst; j < je; j += gridDim.x) {
        if (live) {
            live = __syncthreads_and(mbar_wait_bounded(bar, parity));
            if (live) parity ^= 1u;
            else if (threadIdx.x == 0) atomicOr(&p.ctl->nonfinite, 2);
        }
        {
            const int t = (int)threadIdx.x;
            cpx<double> v[16];
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                const double2 z = stage[t + IP_NT * r];
                v[r] = {z.x, z.y};
            }
            dftR<double, 16, false>(v);
            const int p0 = dit16_pos<M>(t);
#pragma unroll
            for (int q = 0; q < 16; ++q) buf[ip_idx<M>(p0 + q)] = v[q];
        }
        __syncthreads();                               // pass 0 done: the staging buffer is free
        if (threadIdx.x == 0 && live && j + (int)gridDim.x < je) {
            fence_proxy_async_smem();
            issue(j + (int)gridDim.x);
        }
        p16_pass<double, M, 1, false, IP_NT>(buf, p.tw);
        __syncthreads();
        fwd_last_pass_split<double, M>(buf, p.tw, p.wN, reinterpret_cast<double2*>(p.hat + (size_t)j * p.Hp));
        __syncthreads();                               // the buffer read before the next row's pass 0
    }
    if (!live && threadIdx.x == 0) mbar_wait_bounded(bar, parity);   // the copy still in flight
}

template <int M>
static __global__ void __launch_bounds__(IP_NT, 3) k_ifft_thom_pf(FftParams p) {
    static_assert(M / 16 == IP_NT && p16_plan<M>::R(0) == 16 && p16_plan<M>::P >= 2, "one pass-0 butterfly per thread");
    extern __shared__ __align__(16) unsigned char smem_raw[];   // offsets: stage at 128 B, barrier at 16 B multiples
    pdl_begin();
    cpx<double>* buf = reinterpret_cast<cpx<double>*>(smem_raw);
    const double2* stage = reinterpret_cast<const double2*>(smem_raw + IfftPf<M>::stage_off);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + IfftPf<M>::bar_off);
    __shared__ bool thom_now;
    const int Nx = p.Nx, Ny = p.Ny;
    constexpr double scale = 0.5 / (double)M;          // the merge forms 2 Z_n
    const int j0 = (int)(((long long)blockIdx.x * Ny) / gridDim.x);
    const int j1 = (int)(((long long)(blockIdx.x + 1) * Ny) / gridDim.x);
    const int jlo = max(j0, 1), jhi = min(j1, Ny - 1);   // the band's interior rows [jlo, jhi)
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        fence_proxy_async_smem();
    }
    __syncthreads();
    auto issue = [&](int j) {
        mbar_expect_tx(bar, IfftPf<M>::row_bytes);
        bulk_load(const_cast<double2*>(stage), p.hat + (size_t)j * p.Hp, IfftPf<M>::row_bytes, bar);
    };
    if (threadIdx.x == 0 && jlo < jhi) issue(jlo);
    unsigned parity = 0;
    bool live = true;                                  // no wait has run out
    for (int j = j0; j < j1; ++j) {
        double* dst = p.psi + (size_t)j * Nx;
        if (j == 0 || j == Ny - 1) {
            const double v = (j == 0) ? p.psi_bot : p.psi_top;
            for (int i = threadIdx.x; i < Nx; i += IP_NT) dst[i] = v;
            continue;
        }
        if (live) {
            live = __syncthreads_and(mbar_wait_bounded(bar, parity));
            if (live) parity ^= 1u;                    // else the copy of phase `parity` is still in flight
            else if (threadIdx.x == 0) atomicOr(&p.ctl->nonfinite, 2);
        }
        {
            // pass 0: 2 Z_n = s + i d conj(W^n) from X_n, X_{M-n} (n = b + 128 r), as k_ifft_thom
            const int b = (int)threadIdx.x;
            const cpx<double> wt = ldtw(p.wN, b);
            cpx<double> v[16];
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                const int n = b + IP_NT * r;
                const double2 av = stage[n], bv = stage[M - n];
                const cpx<double> sm = {av.x + bv.x, av.y - bv.y};
                const cpx<double> df = {av.x - bv.x, av.y + bv.y};
                const cpx<double> wn = (r == 0) ? wt : cmul(wt, w32<double>(r));
                v[r] = cadd(sm, mul_pi(cmulc(df, wn)));
            }
            dftR<double, 16, true>(v);
            const int p0 = dit16_pos<M>(b);
#pragma unroll
            for (int q = 0; q < 16; ++q) buf[ip_idx<M>(p0 + q)] = v[q];
        }
        __syncthreads();                               // pass 0 done: the staging buffer is free
        if (threadIdx.x == 0 && live && j + 1 < jhi) {
            fence_proxy_async_smem();                  // the reads of the staging buffer before its next write
            issue(j + 1);
        }
        p16_passes_to<double, M, 1, true, IP_NT>(buf, p.tw, [&](int n, const cpx<double>& z) {
            reinterpret_cast<double2*>(dst)[n] = make_double2(z.x * scale, z.y * scale);
        });
        __syncthreads();
        if (p.do_thom) {
            const bool bot = (j == 1 || j == 2), top = (j == Ny - 3 || j == Ny - 2);
            if (bot || top) {
                __threadfence();
                __syncthreads();
                for (int wall = 0; wall < 2; ++wall) {
                    if (!(wall == 0 ? bot : top)) continue;
                    if (threadIdx.x == 0) thom_now = (atomicAdd(&p.ctl->thom_done[wall], 1u) == 1u);
                    __syncthreads();
                    if (thom_now) {
                        __threadfence();
                        thom_row<IP_NT, 8>(p, wall == 1);
                        if (threadIdx.x == 0) p.ctl->thom_done[wall] = 0;
                    }
                    __syncthreads();
                }
            }
        }
    }
    if (!live && threadIdx.x == 0) mbar_wait_bounded(bar, parity);   // the copy still in flight
    if (p.fuse_max) band_maxuv(p, j0, j1);
    if (p.advance) {
        __shared__ bool last;
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            last = (atomicAdd(&p.ctl->ifft_done, 1u) == gridDim.x - 1);
        }
        __syncthreads();
        if (last && threadIdx.x == 0) {
            __threadfence();
            Ctl* ctl = p.ctl;
            ctl->ifft_done = 0;
            if (p.fuse_max)                            // the maxima of psi^(n+1), for the next step's dt
                for (int q = 0; q < 3; ++q)
                    ctl->mx_next[q] = __longlong_as_double((long long)atomicExch(&ctl->mx_acc[q], 0ull));
            advance_time(ctl);
        }
    }
}

struct ThomasParams {
    cpx<double>* hat;        // [Ny][Hp], in place: omega-hat in, psi-hat out
    cpx<float>* hat32;       // the same in FP32 (the FP32-bulk step; the arithmetic stays FP64)
    const double* cp;        // [Ni][Hp]
    const double* asub;      // [Ny]
    const double* inv_csup;  // [Ny]
    const double* csup;      // [Ny]
    double* tconst;          // [nseg][3][Hp]: P, V, Q of every segment (data independent)
    double* tmaps;           // [nseg][2][2 Hp]: D, U of every segment and real column
    double* tblk;            // [groups][nsb][5][32]: block aggregates P, D, B0, B1, Q
    double* tbcarry;         // [groups][nsb][2][32]: carries c (from below) and X (from above) of every block
    unsigned int* tcount;    // [groups]: arrival counters of the map pass
    int Nx, Ny, Hp, H, Ni, nseg, nsb;
    double psi_bot, psi_top;
    Ctl* ctl;                // error flags (bounded TMA waits of the cluster solve)
};

// Spectral values of the solve: FP64 storage, or FP32 storage widened on load and rounded on
// store (F32), with FP64 arithmetic either way.
template <bool F32> struct SpecT { using T = double; using T2 = double2; };
template <> struct SpecT<true> { using T = float; using T2 = float2; };
__device__ __forceinline__ double2 spec_wide(const double2& v) { return v; }
__device__ __forceinline__ double2 spec_wide(const float2& v) { return make_double2((double)v.x, (double)v.y); }
template <bool F32> __device__ __forceinline__ typename SpecT<F32>::T2 spec_narrow(double x, double y) {
    if constexpr (F32) return make_float2((float)x, (float)y);
    else return make_double2(x, y);
}

// Thomas sweeps of the reference (src/poisson.cu:70-133), split into segments of TS_ROWS rows.
//
// Forward elimination dp_j = (r_j - a_j dp_{j-1}) / (b_j - a_j cp_{j-1}) is written
// dp_j = alpha_j r_j + beta_j dp_{j-1} with alpha_j = cp_j / c_j, beta_j = -a_j alpha_j, and the
// back substitution is x_j = dp_j - cp_j x_{j+1}. Both are affine in the value entering a
// segment, so a segment of rows a..b with incoming carries c (dp_{a-1}) and X (x_{b+1}) gives
//   dp_b = D + P c,   x_a = U + V c + Q X,
// where D, U come from running the segment with zero carries, P = prod beta, Q = prod (-cp) and
// V = the back substitution of the partial products of beta (P, V, Q do not depend on the data
// and are tabulated once). A block of TS_NW consecutive segments composes in the same way:
//   dp_last = D_blk + P_blk c_blk,   x_first = B0 + B1 c_blk + Q_blk X_blk.
// One warp owns one segment of one 16-column group (32 real columns, re/im interleaved as in
// HBM); one CTA owns a block. The map pass (k_thomas_maps) writes D, U of every segment and the
// block aggregates; the last CTA of a column group to finish folds that group's block
// aggregates into the carries of every block. The apply pass (k_thomas_apply) resolves the
// carries of the block's segments from the block carries and reruns each segment from them.
constexpr int TS_ROWS = 16;  // rows per segment
constexpr int TS_NW = 8;     // warps (segments) per CTA

// Right-hand side of interior row j (0-based interior index r = j - 1): -omega-hat, with the
// k = 0 Dirichlet wall terms of src/poisson.cu:91-95,109-114 on the real part.
__device__ __forceinline__ double thomas_rhs(const ThomasParams& p, double w, int j, bool kx0re) {
    double v = -w;
    if (kx0re) {
        if (j == 1) v -= p.asub[1] * p.psi_bot * (double)p.Nx;
        if (j == p.Ny - 2) v -= p.csup[p.Ny - 2] * p.psi_top * (double)p.Nx;
    }
    return v;
}

// One-time table of P, V, Q per (segment, kx), one thread per (segment, kx).
static __global__ void k_thomas_consts(ThomasParams p) {
    const int kx = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (kx >= p.Hp) return;
    const int r0 = s * TS_ROWS, n = min(TS_ROWS, p.Ni - r0);
    double Pc[TS_ROWS], cpr[TS_ROWS];
    double P = 1.0;
    for (int t = 0; t < n; ++t) {
        const int j = r0 + t + 1;
        cpr[t] = p.cp[(size_t)(r0 + t) * p.Hp + kx];
        const double alpha = cpr[t] * p.inv_csup[j];
        P = (-p.asub[j] * alpha) * P;
        Pc[t] = P;
    }
    double V = 0.0, Q = 1.0;
    for (int t = n - 1; t >= 0; --t) {
        V = Pc[t] - cpr[t] * V;
        Q = -cpr[t] * Q;
    }
    double* o = p.tconst + (size_t)s * 3 * p.Hp;
    o[kx] = P;
    o[p.Hp + kx] = V;
    o[2 * p.Hp + kx] = Q;
}

// Shared memory of the map and apply passes: per warp, its segment's values [TS_ROWS][32]
// (16 kx, re/im interleaved as in HBM) and cp [TS_ROWS][16]; per CTA, asub and 1/csup of its rows.
__host__ __device__ constexpr size_t thomas_smem_bytes() {
    return sizeof(double) * ((size_t)TS_NW * TS_ROWS * 32 + (size_t)TS_NW * TS_ROWS * 16 + 2 * (size_t)TS_NW * TS_ROWS);
}

struct ThomasTile {
    double* v;               // [TS_ROWS][32] of this warp
    double* cp;              // [TS_ROWS][16] of this warp
    const double* sa;        // asub of the warp's rows
    const double* sic;       // 1/csup of the warp's rows
};

__device__ __forceinline__ ThomasTile thomas_tile(unsigned char* smem_raw, int warp) {
    double* base = reinterpret_cast<double*>(smem_raw);
    ThomasTile tl;
    tl.v = base + (size_t)warp * TS_ROWS * 32;
    tl.cp = base + (size_t)TS_NW * TS_ROWS * 32 + (size_t)warp * TS_ROWS * 16;
    double* rows = base + (size_t)TS_NW * TS_ROWS * 48;
    tl.sa = rows + warp * TS_ROWS;
    tl.sic = rows + TS_NW * TS_ROWS + warp * TS_ROWS;
    return tl;
}

// asub and 1/csup of one warp's rows (8-byte cp.async), and the warp's tile by 16-byte
// cp.async copies (the padding columns kx >= H of omega-hat and of cp hold zeros, so every chunk of a
// valid row is a valid address); rows past the end are left unread and never used.
__device__ __forceinline__ void thomas_stage_warp_rows(const ThomasParams& p, unsigned char* smem_raw, int s) {
    double* rows = reinterpret_cast<double*>(smem_raw) + (size_t)TS_NW * TS_ROWS * 48;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int t = lane; t < 2 * TS_ROWS; t += 32) {
        const int tt = t % TS_ROWS, j = s * TS_ROWS + tt + 1;
        if (j <= p.Ni) {
            if (t < TS_ROWS) cp_async8(&rows[warp * TS_ROWS + tt], &p.asub[j]);
            else cp_async8(&rows[TS_NW * TS_ROWS + warp * TS_ROWS + tt], &p.inv_csup[j]);
        }
    }
}

template <bool F32>
__device__ __forceinline__ void thomas_issue_loads(const ThomasParams& p, int r0, int n, int g, const ThomasTile& tl) {
    const size_t rowstride = (size_t)p.Hp * 2;
    const int lane = threadIdx.x & 31;
    if constexpr (F32) {
        // FP32 spectra: plain 16-byte loads of four values, widened into the FP64 tile
        const float* hatf = reinterpret_cast<const float*>(p.hat32);
#pragma unroll
        for (int i = 0; i < TS_ROWS / 4; ++i) {         // 8 chunks of 16 bytes per row
            const int ch = lane + 32 * i, row = ch >> 3, part = ch & 7;
            if (row < n) {
                const float4 v = __ldcg(reinterpret_cast<const float4*>(
                    &hatf[(size_t)(r0 + row + 1) * rowstride + (size_t)g * 32 + part * 4]));
                double* d = &tl.v[row * 32 + part * 4];
                d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
            }
        }
    } else {
        const double* hatd = reinterpret_cast<const double*>(p.hat);
#pragma unroll
        for (int i = 0; i < TS_ROWS / 2; ++i) {         // 16 chunks of 16 bytes per row
            const int ch = lane + 32 * i, row = ch >> 4, part = ch & 15;
            if (row < n) cp_async16(&tl.v[row * 32 + part * 2], &hatd[(size_t)(r0 + row + 1) * rowstride + (size_t)g * 32 + part * 2]);
        }
    }
#pragma unroll
    for (int i = 0; i < TS_ROWS / 4; ++i) {             // 8 chunks per row
        const int ch = lane + 32 * i, row = ch >> 3, part = ch & 7;
        if (row < n) cp_async16(&tl.cp[row * 16 + part * 2], &p.cp[(size_t)(r0 + row) * p.Hp + (size_t)g * 16 + part * 2]);
    }
}

// Forward elimination over the segment from the carry d, in place in the tile; returns dp at
// the last row.
__device__ __forceinline__ double thomas_forward(const ThomasParams& p, int r0, int n, bool kx0re, double d,
                                                 const ThomasTile& tl) {
    const int lane = threadIdx.x & 31, k16 = lane >> 1;
#pragma unroll 8
    for (int t = 0; t < n; ++t) {
        const double alpha = tl.cp[t * 16 + k16] * tl.sic[t];
        const double beta = -tl.sa[t] * alpha;
        d = alpha * thomas_rhs(p, tl.v[t * 32 + lane], r0 + t + 1, kx0re) + beta * d;
        tl.v[t * 32 + lane] = d;
    }
    return d;
}

// Copies the per-segment maps (P, V, Q from the table, D, U of this solve) of segment s into
// e[5][32] (one warp, cp.async): slots 0 P, 1 D, 2 V, 3 Q, 4 U.
__device__ __forceinline__ void thomas_seg_maps(const ThomasParams& p, int s, int kx, int col, int lane, double* e) {
    const int cols = 2 * p.Hp;
    cp_async8(&e[0 * 32 + lane], &p.tconst[((size_t)s * 3 + 0) * p.Hp + kx]);
    cp_async8(&e[2 * 32 + lane], &p.tconst[((size_t)s * 3 + 1) * p.Hp + kx]);
    cp_async8(&e[3 * 32 + lane], &p.tconst[((size_t)s * 3 + 2) * p.Hp + kx]);
    cp_async8(&e[1 * 32 + lane], &p.tmaps[((size_t)s * 2 + 0) * cols + col]);
    cp_async8(&e[4 * 32 + lane], &p.tmaps[((size_t)s * 2 + 1) * cols + col]);
}

template <bool F32>
static __global__ void __launch_bounds__(TS_NW * 32) k_thomas_maps(ThomasParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_begin();
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = blockIdx.x / p.nsb, sb = blockIdx.x - g * p.nsb;
    const int kx = g * 16 + (lane >> 1), col = g * 32 + lane;
    const bool kx0re = (kx == 0) && ((lane & 1) == 0);
    const int cols = 2 * p.Hp;
    const int s = sb * TS_NW + warp;
    const ThomasTile tl = thomas_tile(smem_raw, warp);
    double* e = tl.v;                                  // [5][32] maps of this warp's segment, after use of the tile
    const int r0 = s * TS_ROWS, n = (s < p.nseg) ? min(TS_ROWS, p.Ni - r0) : 0;
    double Ps = 0.0, Vs = 0.0, Qs = 0.0;
    if (s < p.nseg) {
        thomas_issue_loads<F32>(p, r0, n, g, tl);
        thomas_stage_warp_rows(p, smem_raw, s);
        Ps = __ldg(&p.tconst[((size_t)s * 3 + 0) * p.Hp + kx]);
        Vs = __ldg(&p.tconst[((size_t)s * 3 + 1) * p.Hp + kx]);
        Qs = __ldg(&p.tconst[((size_t)s * 3 + 2) * p.Hp + kx]);
        cp_async_wait_all();
        __syncwarp();
        const double D = thomas_forward(p, r0, n, kx0re, 0.0, tl);
        double U = 0.0;
#pragma unroll 8
        for (int t = n - 1; t >= 0; --t) U = tl.v[t * 32 + lane] - tl.cp[t * 16 + (lane >> 1)] * U;
        p.tmaps[((size_t)s * 2 + 0) * cols + col] = D;
        p.tmaps[((size_t)s * 2 + 1) * cols + col] = U;
        __syncwarp();
        e[0 * 32 + lane] = Ps;
        e[1 * 32 + lane] = D;
        e[2 * 32 + lane] = Vs;
        e[3 * 32 + lane] = Qs;
        e[4 * 32 + lane] = U;
    }
    __syncthreads();
    double* blk = p.tblk + ((size_t)g * p.nsb + sb) * 5 * 32;
    if (warp == 0) {
        // block aggregate: forward carries c_s = c0_s + Pp_s c_blk inside the block, then the
        // backward maps B_s = (U_s + V_s c0_s) + (V_s Pp_s) c_blk composed from the top down
        const int ns = min(TS_NW, p.nseg - sb * TS_NW);
        double c0[TS_NW], Pp[TS_NW];
        double Pa = 1.0, Da = 0.0;
#pragma unroll
        for (int w = 0; w < TS_NW; ++w) {
            if (w < ns) {
                const double* ew = thomas_tile(smem_raw, w).v;
                c0[w] = Da;
                Pp[w] = Pa;
                Da = ew[1 * 32 + lane] + ew[0 * 32 + lane] * Da;
                Pa = ew[0 * 32 + lane] * Pa;
            }
        }
        double B0 = 0.0, B1 = 0.0, Qb = 1.0;
#pragma unroll
        for (int w = TS_NW - 1; w >= 0; --w) {
            if (w < ns) {
                const double* ew = thomas_tile(smem_raw, w).v;
                const double Vs = ew[2 * 32 + lane], Qs = ew[3 * 32 + lane], Us = ew[4 * 32 + lane];
                B0 = (Us + Vs * c0[w]) + Qs * B0;
                B1 = Vs * Pp[w] + Qs * B1;
                Qb = Qs * Qb;
            }
        }
        blk[0 * 32 + lane] = Pa;
        blk[1 * 32 + lane] = Da;
        blk[2 * 32 + lane] = B0;
        blk[3 * 32 + lane] = B1;
        blk[4 * 32 + lane] = Qb;
        __threadfence();                               // the aggregate before the arrival count
    }
    // the last CTA of this column group folds the block aggregates into block carries
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(&p.tcount[g], 1u) == (unsigned)(p.nsb - 1));
    __syncthreads();
    if (!last) return;
    __threadfence();
    double* fb = reinterpret_cast<double*>(smem_raw);  // [nsb][5][32], the tiles are free now
    const double* gblk = p.tblk + (size_t)g * p.nsb * 5 * 32;
    const int nfit = (int)(thomas_smem_bytes() / sizeof(double)) / (5 * 32);
    double* bc = p.tbcarry + (size_t)g * p.nsb * 2 * 32;
    if (p.nsb <= nfit) {
        for (int i = threadIdx.x; i < p.nsb * 5 * 32; i += blockDim.x) fb[i] = __ldcg(&gblk[i]);
        __syncthreads();
        if (warp == 0) {
            double c = 0.0;
            for (int b = 0; b < p.nsb; ++b) {
                bc[(size_t)b * 64 + lane] = c;
                c = fb[b * 160 + 32 + lane] + fb[b * 160 + lane] * c;
            }
            double X = 0.0;
            for (int b = p.nsb - 1; b >= 0; --b) {
                bc[(size_t)b * 64 + 32 + lane] = X;
                const double cb = bc[(size_t)b * 64 + lane];
                X = fb[b * 160 + 64 + lane] + fb[b * 160 + 96 + lane] * cb + fb[b * 160 + 128 + lane] * X;
            }
        }
    } else if (warp == 0) {
        double c = 0.0;
        for (int b = 0; b < p.nsb; ++b) {
            bc[(size_t)b * 64 + lane] = c;
            c = __ldcg(&gblk[b * 160 + 32 + lane]) + __ldcg(&gblk[b * 160 + lane]) * c;
        }
        double X = 0.0;
        for (int b = p.nsb - 1; b >= 0; --b) {
            bc[(size_t)b * 64 + 32 + lane] = X;
            const double cb = bc[(size_t)b * 64 + lane];
            X = __ldcg(&gblk[b * 160 + 64 + lane]) + __ldcg(&gblk[b * 160 + 96 + lane]) * cb +
                __ldcg(&gblk[b * 160 + 128 + lane]) * X;
        }
    }
    if (threadIdx.x == 0) p.tcount[g] = 0;      // ready for the next solve
}

template <bool F32>
static __global__ void __launch_bounds__(TS_NW * 32) k_thomas_apply(ThomasParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_begin();
    __shared__ double segm[TS_NW][5 * 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = blockIdx.x / p.nsb, sb = blockIdx.x - g * p.nsb;
    const int kx = g * 16 + (lane >> 1), col = g * 32 + lane;
    const bool kx0re = (kx == 0) && ((lane & 1) == 0);
    const bool valid = kx < p.H;
    const int s = sb * TS_NW + warp;
    const int ns = min(TS_NW, p.nseg - sb * TS_NW);
    const ThomasTile tl = thomas_tile(smem_raw, warp);
    const int r0 = s * TS_ROWS, n = (s < p.nseg) ? min(TS_ROWS, p.Ni - r0) : 0;
    if (s < p.nseg) {
        thomas_issue_loads<F32>(p, r0, n, g, tl);
        thomas_stage_warp_rows(p, smem_raw, s);
        thomas_seg_maps(p, s, kx, col, lane, segm[warp]);
    }
    const double* bcar = p.tbcarry + ((size_t)g * p.nsb + sb) * 2 * 32;
    const double cblk = __ldcg(&bcar[lane]), Xblk = __ldcg(&bcar[32 + lane]);
    cp_async_wait_all();
    __syncthreads();
    if (s >= p.nseg) return;
    // carries of this warp's segment from the block carries: forward through the lower
    // segments of the block, then backward from the top of the block down to this one
    double cs[TS_NW];
    double c = cblk;
#pragma unroll
    for (int w = 0; w < TS_NW; ++w) {
        cs[w] = c;
        if (w < ns) c = segm[w][32 + lane] + segm[w][lane] * c;
    }
    double x = Xblk;
#pragma unroll
    for (int w = TS_NW - 1; w >= 0; --w)
        if (w > warp && w < ns) x = (segm[w][128 + lane] + segm[w][64 + lane] * cs[w]) + segm[w][96 + lane] * x;
    double cw = cblk;
#pragma unroll
    for (int w = 0; w < TS_NW; ++w)
        if (w == warp) cw = cs[w];
    thomas_forward(p, r0, n, kx0re, cw, tl);
    using ST = typename SpecT<F32>::T;
    ST* hatw = F32 ? reinterpret_cast<ST*>(p.hat32) : reinterpret_cast<ST*>(p.hat);
    const size_t rowstride = (size_t)p.Hp * 2;
#pragma unroll 8
    for (int t = n - 1; t >= 0; --t) {
        x = tl.v[t * 32 + lane] - tl.cp[t * 16 + (lane >> 1)] * x;
        if (valid) hatw[(size_t)(r0 + t + 1) * rowstride + col] = (ST)x;
    }
    // wall rows of psi-hat: Nx psi_bot / Nx psi_top at kx = 0, else 0 (poisson.cu:130-132)
    if (valid) {
        if (s == 0) hatw[col] = (ST)(kx0re ? (double)p.Nx * p.psi_bot : 0.0);
        if (s == p.nseg - 1) hatw[(size_t)(p.Ny - 1) * rowstride + col] = (ST)(kx0re ? (double)p.Nx * p.psi_top : 0.0);
    }
}

// ---- the same solve in one pass: thread-block clusters over 8-kx column groups ----
//
// The two passes above read omega-hat and cp twice and exchange block aggregates through HBM.
// Here a cluster of C CTAs (C <= 8) splits the interior rows into C blocks of R = 32 L rows, one
// per CTA, and walks the 8-kx column groups cid, cid + nclusters, ... (persistent). The tiles of
// a group (omega-hat [R][8] complex, one 128-byte line per row, and cp [R][8]) arrive by TMA in
// one of two shared-memory buffers while the previous group is solved, so the loads overlap the
// sweeps and the exchanges. Thread (q, k) takes segment q (L consecutive rows) of kx = 8 g + k
// into registers (re and im share every coefficient) and writes psi-hat straight back.
// The segments and the CTAs are joined through the affine carries of the two sweeps:
//   forward:  dp_t = dp0_t + (beta_lo ... beta_t) c,          c = dp before the segment;
//   backward: x_t  = x0_t + ((-cp_t) ... (-cp_hi-1)) X,        X = x after the segment.
// A segment's forward map is (D, P): dp_last = D + P c; composing a lower map a with the next
// one b gives (D_b + P_b D_a, P_b P_a). The backward maps (U, Q) compose from the top the same
// way. The four segments of a warp (lanes 8j + k, q = 4w + j) are scanned with shuffles and the
// warps of a CTA through shared memory; per group:
// 1. forward sweep of every segment from c = 0; scans; the CTA's forward map is pushed to every
//    CTA above it; the maps from below are folded into the carry c of every segment;
// 2. carry term; backward sweep from X = 0; scans; the CTA's backward map is pushed to every CTA
//    below; the maps from above are folded into the carry X of every segment;
// 3. carry term; psi-hat out.
// A push is st.async of the map into the receiver's shared memory, which completes bytes on the
// receiver's mbarrier of that direction and group parity; the receiver waits on its own barrier
// (bounded). No cluster-wide barrier is needed inside the loop, and a push carries no ordering
// for the sender's other memory traffic. Two slots by group parity suffice: a sender finishes a
// group only after the maps of the other direction of that group came back from its receivers,
// so it is never two groups ahead of a receiver. One cluster barrier after the mbarriers are
// initialised, and one before the exit, bracket the pushes.
// A wait that does not complete within kTmaWaitLimit polls sets bit 1 of the control block's
// error flags and the CTA goes on (its results are then void); before it exits it waits
// (bounded) for its TMA copies still in flight.
constexpr int TC_KX = 8;                    // kx per cluster
constexpr int TC_NSEG = 32;                 // segments per CTA
constexpr int TC_THREADS = TC_KX * TC_NSEG;
constexpr int TC_NW = TC_THREADS / 32;
constexpr int TC_MAX_CLUSTER = 8;           // portable cluster size
constexpr int TC_MAX_L = 16;                // rows per segment held in registers
constexpr int TC_BOX = 256;                 // rows per TMA box (the box limit)
constexpr unsigned TC_MAP_BYTES = TC_KX * (16 + 8);   // one CTA's map of one direction: 8 x (complex, real)

struct ThomasMaps {
    CUtensorMap hat;         // [Ny][2 Hp] doubles, box 16 x min(R, 256)
    CUtensorMap cp;          // [Ni][Hp] doubles, box 8 x min(R, 256)
};

// bytes of one buffer (omega-hat tile [R][8] complex + cp tile [R][8]) and of the whole
// dynamic shared memory (two buffers, the rows' asub and 1/csup, alignment slack)
// (F32: the omega-hat tile in FP32, 8 bytes per complex value)
__host__ __device__ constexpr size_t tc_hat_bytes(bool f32) { return f32 ? 8 : 16; }
__host__ __device__ constexpr size_t tc_buf_bytes(int R, bool f32 = false) { return (size_t)R * (tc_hat_bytes(f32) + 8) * TC_KX; }
__host__ __device__ constexpr size_t tc_smem_bytes(int R, bool f32 = false) {
    return 2 * tc_buf_bytes(R, f32) + (size_t)R * 16 + 128;
}

__device__ __forceinline__ void cluster_arrive_release() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait_acquire() {
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
__device__ __forceinline__ unsigned cluster_map_u32(unsigned saddr, int rank) {
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(saddr), "r"(rank));
    return r;
}
__device__ __forceinline__ void st_async_v2f64(unsigned raddr, double2 v, unsigned rbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];\n"
                 ::"r"(raddr), "d"(v.x), "d"(v.y), "r"(rbar) : "memory");
}
__device__ __forceinline__ void st_async_f64(unsigned raddr, double v, unsigned rbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f64 [%0], %1, [%2];\n"
                 ::"r"(raddr), "d"(v), "r"(rbar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_cluster_bounded(uint64_t* bar, unsigned parity) {
    for (unsigned it = 0; it < kTmaWaitLimit; ++it)
        if (mbar_try_wait_cluster(bar, parity)) return true;
    return false;
}

// affine map (D, P) of complex D and real P
struct AffMap {
    double2 D;
    double P;
};
// b after a
__device__ __forceinline__ AffMap aff_after(const AffMap& b, const AffMap& a) {
    return AffMap{make_double2(fma(b.P, a.D.x, b.D.x), fma(b.P, a.D.y, b.D.y)), b.P * a.P};
}
__device__ __forceinline__ AffMap aff_shfl_up(const AffMap& m, int off) {
    return AffMap{make_double2(__shfl_up_sync(0xffffffffu, m.D.x, off), __shfl_up_sync(0xffffffffu, m.D.y, off)),
                  __shfl_up_sync(0xffffffffu, m.P, off)};
}
__device__ __forceinline__ AffMap aff_shfl_down(const AffMap& m, int off) {
    return AffMap{make_double2(__shfl_down_sync(0xffffffffu, m.D.x, off), __shfl_down_sync(0xffffffffu, m.D.y, off)),
                  __shfl_down_sync(0xffffffffu, m.P, off)};
}

template <int L, bool F32>
static __global__ void __launch_bounds__(TC_THREADS, (L <= 8 ? 2 : 1)) k_thomas_cluster(const __grid_constant__ ThomasMaps maps, ThomasParams p) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    pdl_begin();
    __shared__ __align__(8) uint64_t bars[2];            // TMA buffers
    __shared__ __align__(8) uint64_t xbar[2][2];         // [direction 0 forward | 1 backward][group parity]
    __shared__ double2 wD[TC_NW][TC_KX];                 // per-warp aggregates of a scan
    __shared__ double wP[TC_NW][TC_KX];
    __shared__ double2 rD[2][2][TC_MAX_CLUSTER][TC_KX];  // maps pushed by the other CTAs [dir][parity][rank][k]
    __shared__ double rP[2][2][TC_MAX_CLUSTER][TC_KX];
    __shared__ double2 cbuf[TC_KX];                      // the folded carry of the other CTAs, per kx
    constexpr int R = TC_NSEG * L;
    constexpr int RB = R < TC_BOX ? R : TC_BOX;
    constexpr int NBOX = R / RB;
    unsigned char* sm = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);
    constexpr size_t HB = tc_hat_bytes(F32), BUF = tc_buf_bytes(R, F32);
    double2* rows = reinterpret_cast<double2*>(sm + 2 * BUF);   // [R] {asub, 1/csup}
    const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const int cid = blockIdx.x / C, ncl = gridDim.x / C;
    const int ngroups = p.Hp / TC_KX;
    const int tid = threadIdx.x, k = tid & (TC_KX - 1), q = tid >> 3, lane = tid & 31, w = tid >> 5, j = q & 3;
    const int r0 = rank * R;
    const int n = max(0, min(R, p.Ni - r0));
    const int lo = q * L;
    const size_t Hp = (size_t)p.Hp;
    auto issue = [&](int grp, int b) {
        unsigned char* dst = sm + (size_t)b * BUF;
        mbar_expect_tx(&bars[b], (unsigned)BUF);
#pragma unroll
        for (int bx = 0; bx < NBOX; ++bx) {
            tma_load_2d(dst + (size_t)bx * RB * HB * TC_KX, &maps.hat, grp * 2 * TC_KX, r0 + 1 + bx * RB, &bars[b]);
            tma_load_2d(dst + (size_t)R * HB * TC_KX + (size_t)bx * RB * 8 * TC_KX, &maps.cp, grp * TC_KX, r0 + bx * RB, &bars[b]);
        }
    };
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        for (int d = 0; d < 2; ++d)
            for (int par = 0; par < 2; ++par) mbar_init(&xbar[d][par], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        fence_proxy_async_smem();
        if (cid < ngroups) issue(cid, 0);
        if (cid + ncl < ngroups) issue(cid + ncl, 1);
    }
    for (int t = tid; t < R; t += TC_THREADS)
        rows[t] = (t < n) ? make_double2(p.asub[r0 + t + 1], p.inv_csup[r0 + t + 1]) : make_double2(0.0, 0.0);
    cluster_arrive_release();                            // every CTA's mbarriers exist before any push
    cluster_wait_acquire();
    const unsigned nbelow = (unsigned)rank, nabove = (unsigned)(C - 1 - rank);
    bool failed = false;
    int pending[2] = {-1, -1};                           // thread 0: parity of a copy whose wait timed out
    int it = 0;
    for (int g = cid; g < ngroups; g += ncl, ++it) {
        const int b = it & 1, par = it & 1;
        const unsigned ph = (unsigned)((it >> 1) & 1);
        if (tid == 0) {                                  // this group's expected pushes (none: the phase ends now)
            mbar_expect_tx(&xbar[0][par], nbelow * TC_MAP_BYTES);
            mbar_expect_tx(&xbar[1][par], nabove * TC_MAP_BYTES);
        }
        const bool ok = mbar_wait_bounded(&bars[b], ph);
        if (!ok && tid == 0 && pending[b] < 0) pending[b] = (int)ph;
        const int kx = g * TC_KX + k;
        const bool valid = kx < p.H;
        const auto* vt = reinterpret_cast<const typename SpecT<F32>::T2*>(sm + (size_t)b * BUF);
        const double* ct = reinterpret_cast<const double*>(sm + (size_t)b * BUF + (size_t)R * HB * TC_KX);
        double2 x[L];
        double cpv[L];
#pragma unroll
        for (int i = 0; i < L; ++i) {
            x[i] = spec_wide(vt[(lo + i) * TC_KX + k]);
            cpv[i] = ct[(lo + i) * TC_KX + k];
        }
        fence_proxy_async_smem();                        // reads of buffer b before its next TMA write
        if (!__syncthreads_and(ok)) {
            failed = true;
            if (tid == 0) atomicOr(&p.ctl->nonfinite, 2);
        }
        if (tid == 0 && !failed && g + 2 * ncl < ngroups) issue(g + 2 * ncl, b);
        // rhs = -omega-hat, with the k = 0 Dirichlet wall terms of src/poisson.cu:91-95,109-114
        if (kx == 0) {
#pragma unroll
            for (int i = 0; i < L; ++i) {
                const int t = lo + i;
                if (r0 + t == 0 && t < n) x[i].x += p.asub[1] * p.psi_bot * (double)p.Nx;
                if (r0 + t == p.Ni - 1 && t < n) x[i].x += p.csup[p.Ny - 2] * p.psi_top * (double)p.Nx;
            }
        }
        // 1. forward sweep from c = 0
        AffMap m{make_double2(0.0, 0.0), 1.0};
#pragma unroll
        for (int i = 0; i < L; ++i) {
            if (lo + i < n) {
                const double2 rc = rows[lo + i];
                const double alpha = cpv[i] * rc.y;
                const double beta = -rc.x * alpha;
                m.D.x = fma(beta, m.D.x, -alpha * x[i].x);
                m.D.y = fma(beta, m.D.y, -alpha * x[i].y);
                x[i] = m.D;
                m.P = beta * m.P;
            }
        }
        // scans: the warp's segments, then the warps below
        AffMap s = m;
#pragma unroll
        for (int off = 8; off <= 16; off *= 2) {
            const AffMap o = aff_shfl_up(s, off);
            if (lane >= off) s = aff_after(s, o);
        }
        AffMap ex = aff_shfl_up(s, 8);
        if (j == 0) ex = AffMap{make_double2(0.0, 0.0), 1.0};
        if (j == 3) { wD[w][k] = s.D; wP[w][k] = s.P; }
        __syncthreads();
        AffMap A{make_double2(0.0, 0.0), 1.0};
#pragma unroll
        for (int v = 0; v < TC_NW - 1; ++v)
            if (v < w) A = aff_after(AffMap{wD[v][k], wP[v][k]}, A);
        const AffMap E = aff_after(ex, A);               // c = E.D + E.P c_blk
        if (q == TC_NSEG - 1) {                          // push this CTA's forward map to the CTAs above
            const AffMap full = aff_after(s, A);
            const unsigned la = smem_u32(&rD[0][par][rank][k]), lp = smem_u32(&rP[0][par][rank][k]);
            const unsigned lb = smem_u32(&xbar[0][par]);
            for (int d = rank + 1; d < C; ++d) {
                const unsigned rb = cluster_map_u32(lb, d);
                st_async_v2f64(cluster_map_u32(la, d), full.D, rb);
                st_async_f64(cluster_map_u32(lp, d), full.P, rb);
            }
        }
        // the CTAs below: warps 0-1, lane (kx kk, rank r), fold ranks 0 .. rank-1 (dp before the
        // first interior row is 0)
        if (w < 2) {
            const bool got = (nbelow == 0) || mbar_wait_cluster_bounded(&xbar[0][par], ph);
            if (!got) atomicOr(&p.ctl->nonfinite, 2);
            const int r = lane & 7, kk = (lane >> 3) + 4 * w;
            AffMap a{make_double2(0.0, 0.0), 1.0};
            if (r < rank) a = AffMap{rD[0][par][r][kk], rP[0][par][r][kk]};
#pragma unroll
            for (int off = 1; off < 8; off *= 2) {
                const AffMap o = aff_shfl_up(a, off);
                if (r >= off) a = aff_after(a, o);
            }
            if (r == rank - 1) cbuf[kk] = a.D;
            if (rank == 0 && r == 0) cbuf[kk] = make_double2(0.0, 0.0);
        }
        __syncthreads();
        const double2 cb = cbuf[k];
        const double2 c = make_double2(fma(E.P, cb.x, E.D.x), fma(E.P, cb.y, E.D.y));
        // 2. carry term, backward sweep from X = 0: (U, Q)
        {
            double Pc = 1.0;
#pragma unroll
            for (int i = 0; i < L; ++i) {
                if (lo + i < n) {
                    const double2 rc = rows[lo + i];
                    Pc = (-rc.x * (cpv[i] * rc.y)) * Pc;
                    x[i].x = fma(Pc, c.x, x[i].x);
                    x[i].y = fma(Pc, c.y, x[i].y);
                }
            }
        }
        m = AffMap{make_double2(0.0, 0.0), 1.0};
#pragma unroll
        for (int i = L - 1; i >= 0; --i) {
            if (lo + i < n) {
                m.D.x = fma(-cpv[i], m.D.x, x[i].x);
                m.D.y = fma(-cpv[i], m.D.y, x[i].y);
                x[i] = m.D;
                m.P = -cpv[i] * m.P;
            }
        }
        // scans from the top
        s = m;
#pragma unroll
        for (int off = 8; off <= 16; off *= 2) {
            const AffMap o = aff_shfl_down(s, off);
            if (lane + off < 32) s = aff_after(s, o);
        }
        ex = aff_shfl_down(s, 8);
        if (j == 3) ex = AffMap{make_double2(0.0, 0.0), 1.0};
        if (j == 0) { wD[w][k] = s.D; wP[w][k] = s.P; }  // the forward reads of wD ended at the last barrier
        __syncthreads();
        A = AffMap{make_double2(0.0, 0.0), 1.0};
#pragma unroll
        for (int v = TC_NW - 1; v > 0; --v)
            if (v > w) A = aff_after(AffMap{wD[v][k], wP[v][k]}, A);
        const AffMap E2 = aff_after(ex, A);              // X = E2.D + E2.P X_blk
        if (q == 0) {                                    // push this CTA's backward map to the CTAs below
            const AffMap full = aff_after(s, A);
            const unsigned la = smem_u32(&rD[1][par][rank][k]), lp = smem_u32(&rP[1][par][rank][k]);
            const unsigned lb = smem_u32(&xbar[1][par]);
            for (int d = 0; d < rank; ++d) {
                const unsigned rb = cluster_map_u32(lb, d);
                st_async_v2f64(cluster_map_u32(la, d), full.D, rb);
                st_async_f64(cluster_map_u32(lp, d), full.P, rb);
            }
        }
        // the CTAs above: fold ranks C-1 .. rank+1 from the top (x after the last interior row is
        // 0); every thread read cb before the barrier after the backward scan
        if (w < 2) {
            const bool got = (nabove == 0) || mbar_wait_cluster_bounded(&xbar[1][par], ph);
            if (!got) atomicOr(&p.ctl->nonfinite, 2);
            const int r = lane & 7, kk = (lane >> 3) + 4 * w;
            AffMap a{make_double2(0.0, 0.0), 1.0};
            if (r > rank && r < C) a = AffMap{rD[1][par][r][kk], rP[1][par][r][kk]};
#pragma unroll
            for (int off = 1; off < 8; off *= 2) {
                const AffMap o = aff_shfl_down(a, off);
                if (r + off < 8) a = aff_after(a, o);
            }
            if (r == rank + 1) cbuf[kk] = a.D;
            if (rank == C - 1 && r == 0) cbuf[kk] = make_double2(0.0, 0.0);
        }
        __syncthreads();
        const double2 Xb = cbuf[k];
        const double2 X = make_double2(fma(E2.P, Xb.x, E2.D.x), fma(E2.P, Xb.y, E2.D.y));
        // 3. carry term; psi-hat out
        using ST2 = typename SpecT<F32>::T2;
        ST2* hatw = F32 ? reinterpret_cast<ST2*>(p.hat32) : reinterpret_cast<ST2*>(p.hat);
        double Qc = 1.0;
#pragma unroll
        for (int i = L - 1; i >= 0; --i) {
            const int t = lo + i;
            if (t < n) {
                Qc = -cpv[i] * Qc;
                if (valid) hatw[(size_t)(r0 + t + 1) * Hp + kx] = spec_narrow<F32>(fma(Qc, X.x, x[i].x), fma(Qc, X.y, x[i].y));
            }
        }
        // wall rows of psi-hat: Nx psi_bot / Nx psi_top at kx = 0, else 0 (poisson.cu:130-132)
        if (valid && q == 0) {
            if (rank == 0) hatw[kx] = spec_narrow<F32>(kx == 0 ? (double)p.Nx * p.psi_bot : 0.0, 0.0);
            if (rank == C - 1) hatw[(size_t)(p.Ny - 1) * Hp + kx] = spec_narrow<F32>(kx == 0 ? (double)p.Nx * p.psi_top : 0.0, 0.0);
        }
    }
    if (tid == 0) {                                      // copies still in flight after a timeout
        for (int b = 0; b < 2; ++b)
            if (pending[b] >= 0) mbar_wait_bounded(&bars[b], (unsigned)pending[b]);
    }
    cluster_arrive_release();                            // every push of the cluster has been issued
    cluster_wait_acquire();
}

// Thom wall vorticity alone (the reference's launcher, src/ops.cu:102-158,270-276).
struct ThomParams {
    double* w;
    const double* psi;
    const double* dy_edge;
    int Nx, Ny, free_slip;
    double psi_bot, psi_top;
};

static __global__ void __launch_bounds__(256) k_thom(ThomParams p) {
    const int Nx = p.Nx, Ny = p.Ny;
    const double b1 = p.dy_edge[0], b2 = p.dy_edge[1];
    const double Ab = 2.0 * (1.0 / (b1 * b1) + 1.0 / (b1 * b2));
    const double Bb = (-2.0) * b1 / (b2 * (b1 + b2) * (b1 + b2));
    const double t1 = p.dy_edge[Ny - 2], t2 = p.dy_edge[Ny - 3];
    const double At = 2.0 * (1.0 / (t1 * t1) + 1.0 / (t1 * t2));
    const double Bt = (-2.0) * t1 / (t2 * (t1 + t2) * (t1 + t2));
    double* wt = p.w + (size_t)(Ny - 1) * Nx;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Nx; i += gridDim.x * blockDim.x) {
        if (p.free_slip) { p.w[i] = 0.0; wt[i] = 0.0; continue; }
        const double d1 = p.psi[(size_t)1 * Nx + i] - p.psi_bot, d2 = p.psi[(size_t)2 * Nx + i] - p.psi_bot;
        p.w[i] = -(Ab * d1 + Bb * d2);
        const double e1 = p.psi[(size_t)(Ny - 2) * Nx + i] - p.psi_top, e2 = p.psi[(size_t)(Ny - 3) * Nx + i] - p.psi_top;
        wt[i] = -(At * e1 + Bt * e2);
    }
}

// max |u|, |v|, |v| a over the interior (src/diag.cu:702-816) and, in the last block, the
// adaptive time step with output trimming (src/main.cu:439-480).
struct MaxParams {
    const double* psi;
    const double* a_node;
    Ctl* ctl;
    int Nx, Ny, adapt, set_dt;
    int next_only;                    // write the maxima only as the next step's (mx_next)
    int nstrips, nbands, band_rows;   // work items of k_maxuv_dt (maxuv_plan)
    double inv_dx, inv_deta, cfl, cvisc, dx, deta, nu, inv_dx2, inv_dymin2, dt_max;
};


// The block maxima of one reduction CTA (warp shuffles, then the warp maxima in shared memory),
// combined across CTAs by atomic maxima in the control block; the last CTA (a last-block
// counter) reads and resets them and computes dt from the reference's formula with the output
// trimming (src/main.cu:439-480). All threads call it.
__device__ __forceinline__ void maxuv_finish(const MaxParams& p, double um, double vm, double vmm, int nonfinite) {
    __shared__ double s[3][32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    um = warp_max_nn(um); vm = warp_max_nn(vm); vmm = warp_max_nn(vmm);
    if (lane == 0) { s[0][warp] = um; s[1][warp] = vm; s[2][warp] = vmm; }
    const int anynf = __syncthreads_or(nonfinite);
    if (warp == 0) {
        um = lane < nw ? s[0][lane] : 0.0;
        vm = lane < nw ? s[1][lane] : 0.0;
        vmm = lane < nw ? s[2][lane] : 0.0;
        um = warp_max_nn(um); vm = warp_max_nn(vm); vmm = warp_max_nn(vmm);
        if (lane == 0) {
            // non-negative doubles order as their bit patterns: atomic maxima on the patterns
            unsigned long long* acc = p.ctl->mx_acc;
            atomicMax(&acc[0], (unsigned long long)__double_as_longlong(um));
            atomicMax(&acc[1], (unsigned long long)__double_as_longlong(vm));
            atomicMax(&acc[2], (unsigned long long)__double_as_longlong(vmm));
            if (anynf) atomicOr(&p.ctl->nonfinite, 1);
            __threadfence();
            const unsigned int done = atomicAdd(&p.ctl->blocks_done, 1u);
            last = (done == gridDim.x - 1);
        }
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    Ctl* ctl = p.ctl;
    um = __longlong_as_double((long long)atomicExch(&ctl->mx_acc[0], 0ull));     // read and reset
    vm = __longlong_as_double((long long)atomicExch(&ctl->mx_acc[1], 0ull));
    vmm = __longlong_as_double((long long)atomicExch(&ctl->mx_acc[2], 0ull));
    ctl->blocks_done = 0;
    ctl->mx_next[0] = um; ctl->mx_next[1] = vm; ctl->mx_next[2] = vmm;
    if (p.next_only) return;
    ctl->umax = um; ctl->vmax = vm; ctl->vmaxm = vmm;
    if (!p.set_dt || !p.adapt) return;
    ctl->dt = adaptive_dt(um, vmm, ctl->t, ctl->next_out, p.cfl, p.dx, p.deta, p.cvisc, p.nu, p.inv_dx2, p.inv_dymin2,
                          p.dt_max);
}

// max |u|, |v|, |v| a over the interior (src/diag.cu:702-866).
//
// Work items are (column strip, row band) pairs: a band is p.band_rows consecutive interior rows
// and a strip MX_COLS columns, 60 per warp; CTAs stride over the items (one item per CTA at the
// full grid). Lane l of a warp holds
// the columns base + 2 (l - 1) and base + 2 (l - 1) + 1 (taken modulo Nx), so that lanes 1..30
// own the warp's 60 columns and lanes 0 and 31 hold their outer neighbours: the x neighbours
// of every owned column come from the adjacent lanes by warp shuffle. A thread walks down its
// band with a window of rows j-1, j, j+1 in registers, so that every row of the band is read
// from HBM once (plus one halo row at each end of the band); four rows are loaded at a time,
// the next four while the current ones are reduced, to keep loads in flight.
//
// The maxima of |psi_{j+1} - psi_{j-1}| and |psi_{i+1} - psi_{i-1}| of a thread's points in
// row j are scaled once per row: for positive factors, rounding is monotone, so
// max_i |a (d_i c)| = a (max_i |d_i| c) exactly and the result is the reference's per-point
// maximum to the bit. A running sum of the differences turns NaN or Inf anywhere into a
// non-finite flag.
//
// VEC: one 16-byte load per row (Nx even and psi 16-byte aligned); otherwise two 8-byte loads,
// one row at a time, and any Nx >= 2 works.

template <bool VEC>
static __global__ void __launch_bounds__(256, 3) k_maxuv_dt(MaxParams p) {
    pdl_begin();
    const int Nx = p.Nx, Ny = p.Ny;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double um = 0.0, vm = 0.0, vmm = 0.0, probe = 0.0;
    const double cy = 0.5 * p.inv_deta, cx = 0.5 * p.inv_dx;
    const int nitems = p.nstrips * p.nbands;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int strip = item % p.nstrips, band = item / p.nstrips;
        const int c = strip * MX_COLS + warp * MX_WCOLS + 2 * (lane - 1);
        const bool own = lane >= 1 && lane <= 30 && c < Nx, two = c + 1 < Nx;
        const int ca = ((c % Nx) + Nx) % Nx, cb = ((c + 1) % Nx + Nx) % Nx;     // the columns, modulo Nx
        const int j0 = 1 + band * p.band_rows, j1 = min(Ny - 1, j0 + p.band_rows);
        if constexpr (VEC) {
            // one row of the window: rows wm (j-1), wc (j), wp (j+1) of the columns c, c+1
            auto row = [&](const double2& wm, const double2& wc, const double2& wp, double a) {
                const double xl = __shfl_up_sync(0xffffffffu, wc.y, 1);      // column c - 1
                const double xr = __shfl_down_sync(0xffffffffu, wc.x, 1);    // column c + 2
                if (own) {
                    const double e0 = wp.x - wm.x, e1 = wp.y - wm.y;
                    const double f0 = wc.y - xl, f1 = xr - wc.x;
                    probe += (e0 + f0) + (e1 + f1);
                    const double dym = nn_max(fabs(e0), fabs(e1)), dxm = nn_max(fabs(f0), fabs(f1));
                    const double av = dxm * cx;
                    um = nn_max(um, a * (dym * cy));
                    vm = nn_max(vm, av);
                    vmm = nn_max(vmm, av * a);
                }
            };
            const double* rp = p.psi + (size_t)(j0 - 1) * Nx + ca;     // row j0 - 1 of this lane's columns
            const size_t nx1 = (size_t)Nx;
            double2 wm = __ldg(reinterpret_cast<const double2*>(rp));
            double2 wc = __ldg(reinterpret_cast<const double2*>(rp + nx1));
            rp += 2 * nx1;                                            // row j0 + 1
            int j = j0;
            // four rows per step, the next four in flight while these are reduced
            double2 n0, n1, n2, n3;
            auto load4 = [&](const double* q) {
                n0 = __ldg(reinterpret_cast<const double2*>(q));
                n1 = __ldg(reinterpret_cast<const double2*>(q + nx1));
                n2 = __ldg(reinterpret_cast<const double2*>(q + 2 * nx1));
                n3 = __ldg(reinterpret_cast<const double2*>(q + 3 * nx1));
            };
            if (j + 4 <= j1) load4(rp);
            for (; j + 4 <= j1; j += 4) {
                const double2 c0 = n0, c1 = n1, c2 = n2, c3 = n3;
                const double a0 = __ldg(&p.a_node[j]), a1 = __ldg(&p.a_node[j + 1]);
                const double a2 = __ldg(&p.a_node[j + 2]), a3 = __ldg(&p.a_node[j + 3]);
                rp += 4 * nx1;
                if (j + 8 <= j1) load4(rp);
                row(wm, wc, c0, a0);
                row(wc, c0, c1, a1);
                row(c0, c1, c2, a2);
                row(c1, c2, c3, a3);
                wm = c2; wc = c3;
            }
            for (; j < j1; ++j) {                                     // the last rows of the band
                const double2 c0 = __ldg(reinterpret_cast<const double2*>(rp));
                rp += nx1;
                row(wm, wc, c0, __ldg(&p.a_node[j]));
                wm = wc; wc = c0;
            }
        } else {
            auto ld2 = [&](int row) -> double2 {
                const double* r = p.psi + (size_t)row * Nx;
                return make_double2(__ldg(r + ca), __ldg(r + cb));
            };
            double2 w0 = ld2(j0 - 1), w1 = ld2(j0);                   // rows j-1 and j
            for (int j = j0; j < j1; ++j) {
                const double2 wp = ld2(j + 1);
                const double xl = __shfl_up_sync(0xffffffffu, w1.y, 1);     // column c - 1
                const double xr = __shfl_down_sync(0xffffffffu, w1.x, 1);   // column c + 2
                if (own) {
                    // column c: psi_{c+1} - psi_{c-1}; column c+1 (when it exists): psi_{c+2} - psi_{c}
                    const double e0 = wp.x - w0.x, f0 = w1.y - xl;
                    double dym = fabs(e0), dxm = fabs(f0), sum = e0 + f0;
                    if (two) {
                        const double e1 = wp.y - w0.y, f1 = xr - w1.x;
                        dym = nn_max(dym, fabs(e1));
                        dxm = nn_max(dxm, fabs(f1));
                        sum += e1 + f1;
                    }
                    probe += sum;
                    const double a = __ldg(&p.a_node[j]);
                    const double av = dxm * cx;
                    um = nn_max(um, a * (dym * cy));
                    vm = nn_max(vm, av);
                    vmm = nn_max(vmm, av * a);
                }
                w0 = w1; w1 = wp;
            }
        }
    }
    const int nonfinite = !(probe - probe == 0.0) || !(um <= 1e300) || !(vm <= 1e300);
    maxuv_finish(p, um, vm, vmm, nonfinite);
}

// Strips of `cols` columns, bands and grid of the max reduction for a target of `ctas` resident
// CTAs, at most `max_grid` CTAs (the partial slots); the CTAs stride over the items.
inline void maxuv_plan(MaxParams& p, int ctas, int max_grid, int& grid, int cols = MX_COLS) {
    const int Ni = p.Ny - 2;
    p.nstrips = (p.Nx + cols - 1) / cols;
    int nb = ctas / p.nstrips;                       // at most one item per resident CTA
    nb = nb < 1 ? 1 : (nb > Ni ? Ni : nb);
    p.band_rows = (Ni + nb - 1) / nb;
    p.nbands = (Ni + p.band_rows - 1) / p.band_rows;
    const long long items = (long long)p.nstrips * p.nbands;
    long long g = items < ctas ? items : ctas;
    if (g > max_grid) g = max_grid;
    grid = g < 1 ? 1 : (int)g;
}

}  // namespace nse2d
