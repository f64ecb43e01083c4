// Device kernels of one SSPRK(3,3) step (FP64). Written for this project.
//
// Per stage s (reference loop src/main.cu:482-538):
//   k_stage_fft   rows: omega^(s+1) = RK combine of omega^(s) + dt rhs(psi, omega^(s)) with
//                 rhs = -J_arakawa + nu lap + f(y) - r omega (+ MMS forcing), written to HBM,
//                 and the forward real FFT of every interior row -> omega-hat [Ny][Hp].
//   k_thomas      y-direction tridiagonal solve of every kx column, in place
//                 (omega-hat -> psi-hat). One thread-block cluster owns 16 kx columns and
//                 splits the Ny-2 rows among its CTAs; each warp sweeps a 32-row segment and
//                 the segments are joined through their affine carries (smem + DSMEM).
//   k_ifft        inverse real FFT of every row -> psi [Ny][Nx].
//   k_thom        Thom wall vorticity on the two wall rows of omega^(s+1).
// Per step: k_maxuv_dt (max|u|,|v|,|v|a -> adaptive dt on the device) before stage 1 and
// k_advance_time after stage 3.
#pragma once
#include <cooperative_groups.h>
#include "common.cuh"

namespace nse2d {

constexpr double kPiD = 3.141592653589793;   // the double nearest pi (CUDART_PI)

__device__ __forceinline__ int wrapi(int i, int Nx) { return i < 0 ? i + Nx : (i >= Nx ? i - Nx : i); }

struct StageParams {
    const double* psi;       // [Ny][Nx]
    const double* w_in;      // omega^(s), stencil input
    const double* w_n;       // omega^n (stages 2, 3); may alias w_out in stage 3
    double* w_out;           // omega^(s+1)
    double* rhs_out;         // optional: store rhs (the stage-3 rhs read by the diagnostics)
    cpx<double>* hat;        // [Ny][Hp]
    const cpx<double>* tw;
    const cpx<double>* wN;
    RowTables rt;
    const Ctl* ctl;
    int Nx, Ny, M, Hp, stage, mms, rows_per_cta;
    double inv_dx, inv_deta, inv_dx2, inv_deta2, nu, lin_drag, Lx, h;
    double mms_A0, mms_eps, mms_Om, mms_k, mms_c;
};

// rhs at one point; follows src/ops.cu:283-326 (Arakawa), :471-499 (Laplacian),
// :515-534 (rhs) and :559-626 (MMS) with the same grouping of terms.
__device__ __forceinline__ double point_rhs(const StageParams& p, int j, int i, double fj, double wc,
                                            double mA, double mAp) {
    const int Nx = p.Nx;
    double J = 0.0, lap = 0.0;
    if (j != 0 && j != p.Ny - 1) {
        const int xm = wrapi(i - 1, Nx), xp = wrapi(i + 1, Nx);
        const double* __restrict__ ps = p.psi;
        const double* __restrict__ om = p.w_in;
        const size_t r0 = (size_t)j * Nx, rm = r0 - Nx, rp = r0 + Nx;
        const double a = __ldg(&p.rt.a_node[j]);
        const double inv4dxde = 0.25 * p.inv_dx * p.inv_deta;
        const double psi_xp = __ldg(&ps[r0 + xp]), psi_xm = __ldg(&ps[r0 + xm]);
        const double psi_yp = __ldg(&ps[rp + i]), psi_ym = __ldg(&ps[rm + i]);
        const double psi_pp = __ldg(&ps[rp + xp]), psi_pm = __ldg(&ps[rm + xp]);
        const double psi_mp = __ldg(&ps[rp + xm]), psi_mm = __ldg(&ps[rm + xm]);
        const double om_xp = __ldg(&om[r0 + xp]), om_xm = __ldg(&om[r0 + xm]);
        const double om_yp = __ldg(&om[rp + i]), om_ym = __ldg(&om[rm + i]);
        const double om_pp = __ldg(&om[rp + xp]), om_pm = __ldg(&om[rm + xp]);
        const double om_mp = __ldg(&om[rp + xm]), om_mm = __ldg(&om[rm + xm]);
        const double J1 = ((psi_xp - psi_xm) * (a * (om_yp - om_ym))
                           - (a * (psi_yp - psi_ym)) * (om_xp - om_xm)) * inv4dxde;
        const double J2 = (psi_xp * (a * (om_pp - om_pm))
                           - psi_xm * (a * (om_mp - om_mm))
                           - a * (psi_yp * (om_pp - om_mp)
                                  - psi_ym * (om_pm - om_mm))) * inv4dxde;
        const double J3 = (-om_xp * (a * (psi_pp - psi_pm))
                           + om_xm * (a * (psi_mp - psi_mm))
                           + a * (om_yp * (psi_pp - psi_mp)
                                  - om_ym * (psi_pm - psi_mm))) * inv4dxde;
        J = -((J1 + J2 + J3) * (1.0 / 3.0));
        const double dxx = (om_xp - 2 * wc + om_xm) * p.inv_dx2;
        const double ap = __ldg(&p.rt.a_edge[j]), am = __ldg(&p.rt.a_edge[j - 1]);
        const double dyy = a * (ap * (om_yp - wc) - am * (wc - om_ym)) * p.inv_deta2;
        lap = dxx + dyy;
    }
    double rhs = -J + p.nu * lap + fj - p.lin_drag * wc;
    if (p.mms) {
        const double k = p.mms_k, c = p.mms_c, c2 = c * c, c3 = c2 * c;
        const double g = __ldg(&p.rt.mms_g[j]), gpp = __ldg(&p.rt.mms_gpp[j]), sin2 = __ldg(&p.rt.mms_sin2[j]);
        const double sk = __ldg(&p.rt.mms_sk[i]), s2k = __ldg(&p.rt.mms_s2k[i]);
        const double term_lin = mAp * g + (p.nu * mA) * ((k * k) * g - gpp) + (p.lin_drag * mA) * g;
        const double term_adv = -(mA * mA) * k * c3 * s2k * sin2;
        rhs += sk * term_lin + term_adv;
    }
    return rhs;
}

// One stockham pass over the row buffer by the whole CTA.
template <bool INV>
__device__ __forceinline__ void cta_fft(cpx<double>*& in, cpx<double>*& out, int M, const cpx<double>* tw) {
    int rad[24];
    const int np = fft_schedule(M, rad);
    int Ns = 1;
    for (int ps = 0; ps < np; ++ps) {
        const int R = rad[ps];
        const int nb = M / R;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            if (R == 8) stockham_butterfly<double, 8, INV>(b, M, Ns, in, out, tw);
            else if (R == 4) stockham_butterfly<double, 4, INV>(b, M, Ns, in, out, tw);
            else stockham_butterfly<double, 2, INV>(b, M, Ns, in, out, tw);
        }
        __syncthreads();
        Ns *= R;
        cpx<double>* t = in; in = out; out = t;
    }
}

static __global__ void __launch_bounds__(256) k_stage_fft(StageParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int M = p.M, Nx = p.Nx;
    cpx<double>* bufA = reinterpret_cast<cpx<double>*>(smem_raw);
    cpx<double>* bufB = bufA + padded_size(M);
    const double dt = p.ctl->dt;
    const double t = p.ctl->t;
    // stage times: t, t + dt, t + dt/2 (src/main.cu:487-528)
    const double ts = (p.stage == 1) ? t : (p.stage == 2 ? t + dt : t + 0.5 * dt);
    double mA = 0.0, mAp = 0.0;
    if (p.mms) {
        mA = p.mms_A0 * (1.0 + p.mms_eps * sin(p.mms_Om * ts));
        mAp = p.mms_A0 * (p.mms_eps * p.mms_Om * cos(p.mms_Om * ts));
    }
    const int j0 = blockIdx.x * p.rows_per_cta;
    const int j1 = min(p.Ny, j0 + p.rows_per_cta);
    for (int j = j0; j < j1; ++j) {
        const double fj = __ldg(&p.rt.frow[j]);
        const bool interior = (j != 0 && j != p.Ny - 1);
        const size_t row = (size_t)j * Nx;
        if (p.stage == 0 && !interior) continue;   // plain transform: interior rows only
        for (int i = threadIdx.x; i < Nx; i += blockDim.x) {
            const double wc = __ldg(&p.w_in[row + i]);
            if (p.stage == 0) {
                reinterpret_cast<double*>(&bufA[pad_idx(i >> 1)])[i & 1] = wc;
                continue;
            }
            const double rhs = point_rhs(p, j, i, fj, wc, mA, mAp);
            if (p.rhs_out) p.rhs_out[row + i] = rhs;
            double wnew;
            if (p.stage == 1) {
                wnew = wc + dt * rhs;                                        // ops.cu:646
            } else if (p.stage == 2) {
                wnew = 0.75 * p.w_n[row + i] + 0.25 * (wc + dt * rhs);       // ops.cu:650
            } else {
                wnew = (1.0 / 3.0) * p.w_n[row + i] + (2.0 / 3.0) * (wc + dt * rhs);  // ops.cu:654
            }
            p.w_out[row + i] = wnew;
            if (interior) reinterpret_cast<double*>(&bufA[pad_idx(i >> 1)])[i & 1] = wnew;
        }
        if (!interior) continue;   // uniform across the CTA
        __syncthreads();
        cpx<double>* in = bufA;
        cpx<double>* out = bufB;
        cta_fft<false>(in, out, M, p.tw);
        cpx<double>* dst = p.hat + (size_t)j * p.Hp;
        for (int k = threadIdx.x; k <= M; k += blockDim.x) dst[k] = rfft_split(k, M, in, p.wN);
        __syncthreads();
    }
}

struct ThomasParams {
    cpx<double>* hat;        // [Ny][Hp], in place
    const double* cp;        // [Ni][Hp]
    const double* asub;
    const double* inv_csup;
    const double* csup;
    int Nx, Ny, Hp, H, Ni, C, R;
    double psi_bot, psi_top;
};

constexpr int KT_NW = 8;     // warps per CTA

// Affine carries: a segment maps its incoming value c to d + P c.
static __global__ void __launch_bounds__(KT_NW * 32) k_thomas(ThomasParams p) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = (int)cluster.block_rank();
    const int g = blockIdx.x / p.C;                   // kx group of 16 columns
    const int R = p.R;
    double* data = reinterpret_cast<double*>(smem_raw);          // [R][32]
    double* cpv = data + (size_t)R * 32;                         // [R][16]
    double* aggP = cpv + (size_t)R * 16;                         // [NW][32]
    double* aggD = aggP + KT_NW * 32;                            // [NW][32]
    double* ctaF = aggD + KT_NW * 32;                            // [2][32]  (P, d) of this CTA
    double* ctaB = ctaF + 64;                                    // [2][32]  (Q, x) of this CTA
    const int kx = g * 16 + (lane >> 1);
    const int part = lane & 1;
    const bool valid = kx < p.H;
    const int r0 = q * R;                                         // first interior row index (0-based)
    const int r1 = min(p.Ni, r0 + R);
    const int RW = (R + KT_NW - 1) / KT_NW;
    const int wa = min(r1, r0 + warp * RW), wb = min(r1, r0 + (warp + 1) * RW);   // [wa, wb)
    const double* hatd = reinterpret_cast<const double*>(p.hat);
    const size_t rowstride = (size_t)p.Hp * 2;
    // ---- load the warp's rows: rhs = -omega-hat plus the k = 0 wall terms (poisson.cu:91-95,109-114)
    for (int r = wa; r < wb; ++r) {
        const int jrow = r + 1;
        double v = valid ? -hatd[(size_t)jrow * rowstride + (size_t)g * 32 + lane] : 0.0;
        if (kx == 0 && part == 0) {
            if (jrow == 1) v -= p.asub[1] * p.psi_bot * (double)p.Nx;
            if (jrow == p.Ny - 2) v -= p.csup[p.Ny - 2] * p.psi_top * (double)p.Nx;
        }
        data[(size_t)(r - r0) * 32 + lane] = v;
        if (lane < 16) {
            const int kk = g * 16 + lane;
            cpv[(size_t)(r - r0) * 16 + lane] = (kk < p.H) ? p.cp[(size_t)r * p.Hp + kk] : 0.0;
        }
    }
    __syncwarp();
    // ---- phase 1: local forward elimination, dp_j = alpha_j r_j + beta_j dp_{j-1}
    //      alpha_j = 1/den_j = cp_j / csup_j, beta_j = -asub_j alpha_j (poisson.cu:97-119)
    double d = 0.0, P = 1.0;
    for (int r = wa; r < wb; ++r) {
        const int jrow = r + 1;
        const double cpj = cpv[(size_t)(r - r0) * 16 + (lane >> 1)];
        const double alpha = cpj * __ldg(&p.inv_csup[jrow]);
        const double beta = -__ldg(&p.asub[jrow]) * alpha;
        d = alpha * data[(size_t)(r - r0) * 32 + lane] + beta * d;
        P = beta * P;
        data[(size_t)(r - r0) * 32 + lane] = d;
    }
    aggP[warp * 32 + lane] = P;
    aggD[warp * 32 + lane] = d;
    __syncthreads();
    if (warp == 0) {
        double cP = 1.0, cD = 0.0;                    // identity map
        for (int w = 0; w < KT_NW; ++w) {
            const double Pw = aggP[w * 32 + lane], Dw = aggD[w * 32 + lane];
            cD = Dw + Pw * cD;
            cP = Pw * cP;
        }
        ctaF[lane] = cP;
        ctaF[32 + lane] = cD;
    }
    cluster.sync();
    // incoming carry of this CTA: compose the maps of the lower-ranked CTAs
    double c = 0.0;
    for (int qq = 0; qq < q; ++qq) {
        const double* rf = cluster.map_shared_rank(ctaF, qq);
        c = rf[32 + lane] + rf[lane] * c;
    }
    for (int w = 0; w < warp; ++w) c = aggD[w * 32 + lane] + aggP[w * 32 + lane] * c;
    // ---- phase 2: dp_j = dtilde_j + P_j c
    P = 1.0;
    for (int r = wa; r < wb; ++r) {
        const int jrow = r + 1;
        const double cpj = cpv[(size_t)(r - r0) * 16 + (lane >> 1)];
        const double alpha = cpj * __ldg(&p.inv_csup[jrow]);
        const double beta = -__ldg(&p.asub[jrow]) * alpha;
        P = beta * P;
        data[(size_t)(r - r0) * 32 + lane] += P * c;
    }
    // ---- phase 3: local back substitution x_j = dp_j - cp_j x_{j+1} (poisson.cu:121-129)
    double x = 0.0, Q = 1.0;
    for (int r = wb - 1; r >= wa; --r) {
        const double cpj = cpv[(size_t)(r - r0) * 16 + (lane >> 1)];
        x = data[(size_t)(r - r0) * 32 + lane] - cpj * x;
        Q = -cpj * Q;
        data[(size_t)(r - r0) * 32 + lane] = x;
    }
    __syncthreads();                                   // phase-1 aggregates no longer needed
    aggP[warp * 32 + lane] = Q;
    aggD[warp * 32 + lane] = x;
    __syncthreads();
    if (warp == 0) {
        double cQ = 1.0, cX = 0.0;
        for (int w = KT_NW - 1; w >= 0; --w) {
            const double Qw = aggP[w * 32 + lane], Xw = aggD[w * 32 + lane];
            cX = Xw + Qw * cX;
            cQ = Qw * cQ;
        }
        ctaB[lane] = cQ;
        ctaB[32 + lane] = cX;
    }
    cluster.sync();
    double X = 0.0;                                    // x at the row above this CTA
    for (int qq = p.C - 1; qq > q; --qq) {
        const double* rb = cluster.map_shared_rank(ctaB, qq);
        X = rb[32 + lane] + rb[lane] * X;
    }
    for (int w = KT_NW - 1; w > warp; --w) X = aggD[w * 32 + lane] + aggP[w * 32 + lane] * X;
    // ---- phase 4: x_j = xtilde_j + Q_j X, Q_j = prod_{i=j}^{top} (-cp_i); store psi-hat
    double* hatw = reinterpret_cast<double*>(p.hat);
    Q = 1.0;
    for (int r = wb - 1; r >= wa; --r) {
        const double cpj = cpv[(size_t)(r - r0) * 16 + (lane >> 1)];
        Q = -cpj * Q;
        const double xv = data[(size_t)(r - r0) * 32 + lane] + Q * X;
        if (valid) hatw[(size_t)(r + 1) * rowstride + (size_t)g * 32 + lane] = xv;
    }
    // wall rows of psi-hat: Nx psi_bot / Nx psi_top at kx = 0, else 0 (poisson.cu:130-132)
    if (warp == 0 && valid) {
        if (q == 0) hatw[(size_t)g * 32 + lane] = (kx == 0 && part == 0) ? (double)p.Nx * p.psi_bot : 0.0;
        if (q == p.C - 1)
            hatw[(size_t)(p.Ny - 1) * rowstride + (size_t)g * 32 + lane] =
                (kx == 0 && part == 0) ? (double)p.Nx * p.psi_top : 0.0;
    }
    cluster.sync();                                    // keep smem alive for remote readers
}

struct IfftParams {
    const cpx<double>* hat;
    double* psi;
    const cpx<double>* tw;
    const cpx<double>* wN;
    int Nx, Ny, M, Hp, rows_per_cta;
    double psi_bot, psi_top;
};

static __global__ void __launch_bounds__(256) k_ifft(IfftParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int M = p.M, Nx = p.Nx;
    cpx<double>* bufA = reinterpret_cast<cpx<double>*>(smem_raw);
    cpx<double>* bufB = bufA + padded_size(M);
    const int j0 = blockIdx.x * p.rows_per_cta;
    const int j1 = min(p.Ny, j0 + p.rows_per_cta);
    const double scale = 1.0 / (double)M;
    for (int j = j0; j < j1; ++j) {
        double* dst = p.psi + (size_t)j * Nx;
        if (j == 0 || j == p.Ny - 1) {
            const double v = (j == 0) ? p.psi_bot : p.psi_top;
            for (int i = threadIdx.x; i < Nx; i += blockDim.x) dst[i] = v;
            continue;
        }
        const cpx<double>* src = p.hat + (size_t)j * p.Hp;
        for (int k = threadIdx.x; k <= M; k += blockDim.x) bufB[k] = src[k];
        __syncthreads();
        for (int k = threadIdx.x; k < M; k += blockDim.x) bufA[pad_idx(k)] = irfft_merge(k, M, bufB, p.wN);
        __syncthreads();
        cpx<double>* in = bufA;
        cpx<double>* out = bufB;
        cta_fft<true>(in, out, M, p.tw);
        for (int n = threadIdx.x; n < M; n += blockDim.x) {
            const cpx<double> z = in[pad_idx(n)];
            reinterpret_cast<double2*>(dst)[n] = make_double2(z.x * scale, z.y * scale);
        }
        __syncthreads();
    }
}

// Thom wall vorticity (src/ops.cu:102-158); with closure_diag also the wall-row enstrophy
// jump of this stage (src/main.cu:271-298), accumulated into ctl->jwall[stage-1].
struct ThomParams {
    double* w;
    const double* psi;
    const double* dy_edge;
    const double* w_node;
    Ctl* ctl;
    int Nx, Ny, free_slip, closure, stage;
    double psi_bot, psi_top, invA_full;
};

static __global__ void __launch_bounds__(256) k_thom(ThomParams p) {
    const int Nx = p.Nx, Ny = p.Ny;
    double sb = 0.0, sa = 0.0;
    const double wq_b = p.closure ? p.w_node[0] : 0.0, wq_t = p.closure ? p.w_node[Ny - 1] : 0.0;
    const double b1 = p.dy_edge[0], b2 = p.dy_edge[1];
    const double Ab = 2.0 * (1.0 / (b1 * b1) + 1.0 / (b1 * b2));
    const double Bb = (-2.0) * b1 / (b2 * (b1 + b2) * (b1 + b2));
    const double t1 = p.dy_edge[Ny - 2], t2 = p.dy_edge[Ny - 3];
    const double At = 2.0 * (1.0 / (t1 * t1) + 1.0 / (t1 * t2));
    const double Bt = (-2.0) * t1 / (t2 * (t1 + t2) * (t1 + t2));
    double* wt = p.w + (size_t)(Ny - 1) * Nx;
    // one CTA when closure sums are wanted (the reduction below is CTA-local)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Nx; i += gridDim.x * blockDim.x) {
        const double ob = p.w[i], ot = wt[i];
        double nb, nt;
        if (p.free_slip) {
            nb = 0.0; nt = 0.0;
        } else {
            const double d1 = p.psi[(size_t)1 * Nx + i] - p.psi_bot, d2 = p.psi[(size_t)2 * Nx + i] - p.psi_bot;
            nb = -(Ab * d1 + Bb * d2);
            const double e1 = p.psi[(size_t)(Ny - 2) * Nx + i] - p.psi_top, e2 = p.psi[(size_t)(Ny - 3) * Nx + i] - p.psi_top;
            nt = -(At * e1 + Bt * e2);
        }
        p.w[i] = nb;
        wt[i] = nt;
        if (p.closure) {
            sb += wq_b * ob * ob + wq_t * ot * ot;
            sa += wq_b * nb * nb + wq_t * nt * nt;
        }
    }
    if (!p.closure) return;
    __shared__ double rb[256], ra[256];
    rb[threadIdx.x] = sb; ra[threadIdx.x] = sa;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) { rb[threadIdx.x] += rb[threadIdx.x + s]; ra[threadIdx.x] += ra[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        p.ctl->jwall[p.stage - 1] += 0.5 * ra[0] * p.invA_full - 0.5 * rb[0] * p.invA_full;
}

// max |u|, |v|, |v| a over the interior (src/diag.cu:702-816) and, in the last block, the
// adaptive time step with output trimming (src/main.cu:439-480).
struct MaxParams {
    const double* psi;
    const double* a_node;
    double* blocks;          // [gridDim.x][3]
    Ctl* ctl;
    int Nx, Ny, adapt, set_dt;
    double inv_dx, inv_deta, cfl, cvisc, dx, deta, nu, inv_dx2, inv_dymin2, dt_max;
};

__device__ __forceinline__ double time_tol_d(double t) { return 64.0 * 2.220446049250313e-16 * fmax(1.0, fabs(t)); }

static __global__ void __launch_bounds__(256) k_maxuv_dt(MaxParams p) {
    const int Nx = p.Nx, Ny = p.Ny;
    double um = 0.0, vm = 0.0, vmm = 0.0;
    int nonfinite = 0;
    const size_t total = (size_t)Nx * (size_t)(Ny - 2);
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int j = 1 + (int)(q / Nx);
        const int i = (int)(q - (size_t)(j - 1) * Nx);
        const int ip = (i + 1 < Nx) ? i + 1 : 0, im = (i > 0) ? i - 1 : Nx - 1;
        const double dpsideta = (p.psi[(size_t)(j + 1) * Nx + i] - p.psi[(size_t)(j - 1) * Nx + i]) * (0.5 * p.inv_deta);
        const double dpsidx = (p.psi[(size_t)j * Nx + ip] - p.psi[(size_t)j * Nx + im]) * (0.5 * p.inv_dx);
        const double a = __ldg(&p.a_node[j]);
        const double u = a * dpsideta, v = -dpsidx;
        const double au = fabs(u), av = fabs(v), avm = av * a;
        if (!(au <= 1e300) || !(av <= 1e300)) nonfinite = 1;
        um = fmax(um, au); vm = fmax(vm, av); vmm = fmax(vmm, avm);
    }
    __shared__ double s[3][256];
    __shared__ int snf;
    __shared__ bool last;
    if (threadIdx.x == 0) snf = 0;
    s[0][threadIdx.x] = um; s[1][threadIdx.x] = vm; s[2][threadIdx.x] = vmm;
    __syncthreads();
    if (nonfinite) atomicOr(&snf, 1);
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st)
            for (int c = 0; c < 3; ++c) s[c][threadIdx.x] = fmax(s[c][threadIdx.x], s[c][threadIdx.x + st]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int c = 0; c < 3; ++c) p.blocks[blockIdx.x * 3 + c] = s[c][0];
        if (snf) atomicOr(&p.ctl->nonfinite, 1);
        __threadfence();
        const unsigned int done = atomicAdd(&p.ctl->blocks_done, 1u);
        last = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    um = 0.0; vm = 0.0; vmm = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
        um = fmax(um, __ldcg(&p.blocks[b * 3 + 0]));
        vm = fmax(vm, __ldcg(&p.blocks[b * 3 + 1]));
        vmm = fmax(vmm, __ldcg(&p.blocks[b * 3 + 2]));
    }
    s[0][threadIdx.x] = um; s[1][threadIdx.x] = vm; s[2][threadIdx.x] = vmm;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st)
            for (int c = 0; c < 3; ++c) s[c][threadIdx.x] = fmax(s[c][threadIdx.x], s[c][threadIdx.x + st]);
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    Ctl* ctl = p.ctl;
    ctl->blocks_done = 0;
    ctl->umax = s[0][0]; ctl->vmax = s[1][0]; ctl->vmaxm = s[2][0];
    if (!p.set_dt || !p.adapt) return;
    const double umax = s[0][0], vmaxm = s[2][0];
    const double dt_x = (umax > 0 ? p.cfl * (p.dx / umax) : 1e30);
    const double dt_y = (vmaxm > 0 ? p.cfl * (p.deta / vmaxm) : 1e30);
    const double dt_adv = fmin(dt_x, dt_y);
    const double dt_vis = (p.nu > 0) ? p.cvisc * 0.5 / (p.nu * (p.inv_dx2 + p.inv_dymin2)) : 1e30;
    double dt = fmin(p.dt_max, fmin(dt_adv, dt_vis));
    const double t_next = ctl->next_out;
    if (t_next < 1e299) {
        const double rem = t_next - ctl->t;
        const double tol = fmax(time_tol_d(t_next), 1e-6 * dt);
        if (rem > tol && rem < 0.5 * dt) dt = rem;
    }
    ctl->dt = dt;
}

// t += dt, step++, and the snap to the scheduled output times (src/main.cu:541-551): the
// tolerance is re-evaluated after the first snap, as the reference does.
static __global__ void k_advance_time(Ctl* ctl) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double dt = ctl->dt;
    double t = ctl->t + dt;
    const double ns = ctl->next_snap, nd = ctl->next_diag;
    if (ns < 1e299 && fabs(t - ns) <= fmax(time_tol_d(t), 1e-6 * fmax(1e-300, fabs(dt)))) t = ns;
    if (nd < 1e299 && fabs(t - nd) <= fmax(time_tol_d(t), 1e-6 * fmax(1e-300, fabs(dt)))) t = nd;
    ctl->t = t;
    ctl->step += 1;
}

}  // namespace nse2d
