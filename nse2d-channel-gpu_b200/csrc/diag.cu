// Diagnostics reductions for diagnostics.csv (src/diag.cu of the reference, host formulas
// src/main.cu:387-411 and :627-675). Written for this project.
//
// The reference accumulates each sum with one atomicAdd per block (src/diag.cu:27,89,...),
// so its last digits depend on block scheduling. Here every row is reduced by one CTA into
// per-row partials (fixed tree order), and the rows are then summed in row order with a
// compensated (Neumaier) sum: the result is deterministic and at least as accurate.
#include <cstddef>
#include <algorithm>
#include <cmath>
#include <limits>

#include "nse2d_internal.h"
#include "step_kernels.cuh"

namespace nse2d {

enum {
    S_K = 0, S_W2, S_GW2, S_WWY_BOT, S_WWY_TOP, S_WRHS, S_PIN, S_EPS, S_POM, S_MOB, S_MOT,
    S_W2_INT, S_GW2_INT, S_T2_D, S_T2_J, S_T2_W2, S_T2_G2, S_T2_P, S_T2_ETA, S_T2_PHI, S_WALL_WRHS,
    NSUM
};

struct DiagParams {
    const double* psi;
    const double* w;
    const double* rhs;       // may be null
    const double* J;         // may be null
    RowTables rt;
    double* rows;            // [Ny][NSUM]
    int Nx, Ny;
    double inv_dx, inv_deta, h, F0;
    int nforce;
};

__global__ void __launch_bounds__(256) k_diag_rows(DiagParams p) {
    const int Nx = p.Nx, Ny = p.Ny;
    __shared__ double red[NSUM][8];
    const double inv_dx2 = p.inv_dx * p.inv_dx, inv_deta2 = p.inv_deta * p.inv_deta;
    for (int j = blockIdx.x; j < Ny; j += gridDim.x) {
        double s[NSUM];
#pragma unroll
        for (int q = 0; q < NSUM; ++q) s[q] = 0.0;
        const double wq = p.rt.w_node[j], a = p.rt.a_node[j], wt = p.rt.wt_node[j];
        const int ym = (j == 0 ? 0 : j - 1), yp = (j == Ny - 1 ? Ny - 1 : j + 1);
        const double yy = p.rt.y[j];
        const double argF = (double)p.nforce * kPiD * ((yy + p.h) / (2.0 * p.h));
        const double Fx = p.F0 * sin(argF);                                          // diag.cu:359
        const double fom = -p.F0 * ((double)p.nforce * kPiD / (2.0 * p.h)) * cos(argF);  // diag.cu:392-393
        const double* w = p.w;
        const double* psi = p.psi;
        for (int i = threadIdx.x; i < Nx; i += blockDim.x) {
            const int xm = (i == 0 ? Nx - 1 : i - 1), xp = (i == Nx - 1 ? 0 : i + 1);
            const size_t c = (size_t)j * Nx + i;
            const double wc = w[c];
            const bool interior = (j != 0 && j != Ny - 1);
            if (interior) {                                                          // diag.cu:201-223
                const double u = (psi[c + Nx] - psi[c - Nx]) * 0.5 * p.inv_deta * a;
                const double v = -(psi[(size_t)j * Nx + xp] - psi[(size_t)j * Nx + xm]) * 0.5 * p.inv_dx;
                s[S_K] += 0.5 * (u * u + v * v) * wq;
            }
            {                                                                        // diag.cu:43-90
                const double wx = (w[(size_t)j * Nx + xp] - w[(size_t)j * Nx + xm]) * 0.5 * p.inv_dx;
                double weta;
                if (j == 0) weta = (-3.0 * w[i] + 4.0 * w[(size_t)Nx + i] - 1.0 * w[(size_t)2 * Nx + i]) * (0.5 * p.inv_deta);
                else if (j == Ny - 1)
                    weta = (3.0 * w[(size_t)(Ny - 1) * Nx + i] - 4.0 * w[(size_t)(Ny - 2) * Nx + i] + 1.0 * w[(size_t)(Ny - 3) * Nx + i]) * (0.5 * p.inv_deta);
                else weta = (w[c + Nx] - w[c - Nx]) * 0.5 * p.inv_deta;
                const double wy = a * weta;
                s[S_W2] += wq * (wc * wc);
                s[S_GW2] += wq * (wx * wx + wy * wy);
                if (j == 0) { s[S_WWY_BOT] += wc * wy; s[S_MOB] += wc; }             // diag.cu:500-569
                if (j == Ny - 1) { s[S_WWY_TOP] += wc * wy; s[S_MOT] += wc; }
            }
            if (p.rhs) s[S_WRHS] += wq * wc * p.rhs[c];                               // diag.cu:628-671
            {                                                                        // diag.cu:350-367
                const double u = (psi[(size_t)yp * Nx + i] - psi[(size_t)ym * Nx + i]) * 0.5 * p.inv_deta * a;
                s[S_PIN] += u * Fx * wq;
            }
            if (!interior) {                                                         // diag.cu:250-329
                s[S_EPS] += (wc * wc) * wq;
            } else {
                const double ap = p.rt.a_edge[j], am = p.rt.a_edge[j - 1];
                const double pxp = (psi[c + Nx - i + xp] - psi[c + Nx - i + xm]) * (0.5 * p.inv_dx);
                const double pxm = (psi[c - Nx - i + xp] - psi[c - Nx - i + xm]) * (0.5 * p.inv_dx);
                const double ux = a * (pxp - pxm) * (0.5 * p.inv_deta);
                const double vy = -ux;
                const double vx = -(psi[(size_t)j * Nx + xp] - 2.0 * psi[c] + psi[(size_t)j * Nx + xm]) * inv_dx2;
                const double uy = a * (ap * (psi[c + Nx] - psi[c]) - am * (psi[c] - psi[c - Nx])) * inv_deta2;
                s[S_EPS] += (ux * ux + uy * uy + vx * vx + vy * vy) * wq;
            }
            s[S_POM] += wc * fom * wq;                                               // diag.cu:378-409
            if (interior) {                                                          // diag.cu:6-28
                const double wx = (w[(size_t)j * Nx + xp] - w[(size_t)j * Nx + xm]) * 0.5 * p.inv_dx;
                const double wy = a * (w[c + Nx] - w[c - Nx]) * 0.5 * p.inv_deta;
                s[S_W2_INT] += wq * (wc * wc);
                s[S_GW2_INT] += wq * (wx * wx + wy * wy);
                s[S_T2_W2] += wt * (wc * wc);
                s[S_T2_G2] += wt * (wx * wx + wy * wy);
                const double dxw = (w[(size_t)j * Nx + xp] - wc) * p.inv_dx;          // diag.cu:166-190
                s[S_T2_ETA] += wt * dxw * dxw;
            }
            if (p.rhs) s[S_T2_D] += wt * wc * p.rhs[c];
            if (p.J) s[S_T2_J] += wt * wc * p.J[c];
            s[S_T2_P] += wc * fom * wt;
            if (j <= Ny - 2) {
                const double dw = w[c + Nx] - wc;
                s[S_T2_ETA] += p.rt.a_edge[j] * dw * dw * p.inv_deta;
            }
            if (j == 0) s[S_T2_PHI] -= wc * p.rt.a_edge[0] * (w[(size_t)Nx + i] - wc) * p.inv_deta;
            if (j == Ny - 1) s[S_T2_PHI] += wc * p.rt.a_edge[Ny - 2] * (wc - w[(size_t)(Ny - 2) * Nx + i]) * p.inv_deta;
            if (p.rhs && !interior) s[S_WALL_WRHS] += wq * wc * p.rhs[c];           // main.cu:290-296
        }
        // warp tree, then the 8 warps in order
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int q = 0; q < NSUM; ++q) {
            double v = s[q];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) red[q][warp] = v;
        }
        __syncthreads();
        if (threadIdx.x < NSUM) {
            double v = 0.0;
            for (int k = 0; k < 8; ++k) v += red[threadIdx.x][k];
            p.rows[(size_t)j * NSUM + threadIdx.x] = v;
        }
        __syncthreads();
    }
}

// Sum the rows of each quantity in row order, compensated; one warp per quantity.
__global__ void k_diag_final(const double* rows, int Ny, double* out) {
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (q >= NSUM) return;
    double s = 0.0, cmp = 0.0;
    for (int j = lane; j < Ny; j += 32) {
        const double x = rows[(size_t)j * NSUM + q];
        const double t = s + x;
        cmp += (fabs(s) >= fabs(x)) ? (s - t) + x : (x - t) + s;
        s = t;
    }
    __shared__ double part[NSUM][32];
    part[q][lane] = s + cmp;
    __syncwarp();
    if (lane == 0) {
        double S = 0.0, C = 0.0;
        for (int k = 0; k < 32; ++k) {
            const double x = part[q][k];
            const double t = S + x;
            C += (fabs(S) >= fabs(x)) ? (S - t) + x : (x - t) + S;
            S = t;
        }
        out[q] = S + C;
    }
}

int rhs_at_state(Context* c, const double* w, const double* psi, double* J, double* rhs, double tm, cudaStream_t s);

static int diag_sums(Context* c, const double* rhs, const double* J, double* host_out, cudaStream_t s) {
    DiagParams p{};
    p.psi = c->psi; p.w = c->w; p.rhs = rhs; p.J = J; p.rt = c->rt; p.rows = c->red_blocks;
    p.Nx = c->Nx; p.Ny = c->Ny; p.inv_dx = c->inv_dx; p.inv_deta = c->inv_deta; p.h = c->cfg.h;
    p.F0 = c->cfg.F0; p.nforce = c->cfg.nforce;
    if ((size_t)c->Ny * NSUM > c->red_capacity) {
        set_error("diagnostics: reduction buffer too small (%zu < %zu)", c->red_capacity, (size_t)c->Ny * NSUM);
        return -1;
    }
    const int grid = std::min(c->Ny, 8 * c->num_sms);
    k_diag_rows<<<grid, 256, 0, s>>>(p);
    NSE_CUDA_TRY(cudaGetLastError());
    k_diag_final<<<1, 32 * NSUM, 0, s>>>(c->red_blocks, c->Ny, c->red_out);
    NSE_CUDA_TRY(cudaGetLastError());
    NSE_CUDA_TRY(cudaMemcpyAsync(host_out, c->red_out, NSUM * sizeof(double), cudaMemcpyDeviceToHost, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
}

// One diagnostics.csv row (columns umax .. Phi_h), host formulas of src/main.cu:387-411 (t = 0
// row) and :627-688 (output rows). For output rows dOmega_rhs pairs the state with the rhs of
// the last stage-3 evaluation, which the step stores into c->rhs when asked (store_rhs).
int diagnostics_row(Context* c, int t0_row, double* o, cudaStream_t s) {
    const double nan = std::numeric_limits<double>::quiet_NaN();
    if (launch_maxuv(c, c->psi, false, s)) return -1;
    NSE_CUDA_TRY(cudaMemcpyAsync(c->h_ctl, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    const double t = c->h_ctl->t;
    if (t0_row && rhs_at_state(c, c->w, c->psi, nullptr, c->rhs, t, s)) return -1;
    double S[NSUM];
    if (diag_sums(c, c->rhs, nullptr, S, s)) return -1;
    const double nu = c->nu, iA = c->invA_full, h = c->cfg.h, Nx = (double)c->Nx;
    const double mwb = S[S_WWY_BOT] / Nx, mwt = S[S_WWY_TOP] / Nx;
    const double mOb = S[S_MOB] / Nx, mOt = S[S_MOT] / Nx;
    const double tb = -nu * mOb, tt = -nu * mOt;
    const double ut = std::sqrt(0.5 * (std::fabs(tb) + std::fabs(tt)));
    const double Ub = c->cfg.Ub;
    o[0] = c->h_ctl->umax;
    o[1] = c->h_ctl->vmax;
    o[2] = S[S_K] * iA;
    o[3] = 0.5 * S[S_W2] * iA;
    o[4] = S[S_WRHS] * iA;
    o[5] = nu * S[S_GW2] * iA;
    o[6] = (nu > 0.0) ? (nu * (mwt - mwb) / (2.0 * h)) : 0.0;
    o[7] = S[S_PIN] * iA;
    o[8] = nu * S[S_EPS] * iA;
    o[9] = S[S_POM] * iA;
    o[10] = tb;
    o[11] = tt;
    o[12] = (tt - tb) / (2.0 * h) + c->meanFx_A - c->cfg.lin_drag * Ub;
    o[13] = ut;
    o[14] = (Ub != 0.0) ? 2.0 * (0.5 * (std::fabs(tb) + std::fabs(tt))) / (Ub * Ub) : nan;
    o[15] = (nu > 0.0) ? ut * h / nu : 0.0;
    for (int q = 16; q < 29; ++q) o[q] = nan;
    if (!c->closure_diag) return 0;
    if (t0_row) {
        o[16] = o[4]; o[20] = 0.0; o[21] = 0.0; o[22] = 0.0;
        return 0;
    }
    if (rhs_at_state(c, c->w, c->psi, c->J, c->rhs, t, s)) return -1;
    double C[NSUM];
    if (diag_sums(c, c->rhs, c->J, C, s)) return -1;
    const double same = C[S_WRHS] * iA;
    o[16] = same;
    o[17] = same - C[S_WALL_WRHS] * iA;
    o[18] = 0.5 * C[S_W2_INT] * iA;
    o[19] = nu * C[S_GW2_INT] * iA;
    o[20] = c->h_ctl->jwall[0];
    o[21] = c->h_ctl->jwall[1];
    o[22] = c->h_ctl->jwall[2];
    o[23] = 0.5 * C[S_T2_W2] * iA;
    o[24] = C[S_T2_D] * iA;
    o[25] = -C[S_T2_J] * iA;
    o[26] = C[S_T2_P] * iA;
    o[27] = nu * C[S_T2_ETA] * iA;
    o[28] = nu * C[S_T2_PHI] * iA;
    return 0;
}

// ---- time-averaged profiles: row sums of u, v, u^2, v^2, u v (src/diag.cu:468-499) ----
// One CTA per row (grid-stride over rows); u and v as the reference forms them, with the
// neighbouring rows clamped at the walls; a fixed-order reduction, so the sums are
// deterministic.
// ACC: the time-weighted statistics of the run loop (src/main.cu:695-733) on the device: at a step
// that is a multiple of ctl->acc_every, with dtw = t - acc_last_t > 0, out[q][j] += (sum / Nx) dtw,
// the host's accumulation of the same row sums; other steps return at once.
template <bool ACC>
static __global__ void __launch_bounds__(256) k_row_moments(const double* __restrict__ psi, const double* __restrict__ a_node,
                                                           int Nx, int Ny, double inv_dx, double inv_deta,
                                                           double* __restrict__ out, const Ctl* __restrict__ ctl) {
    double dtw = 0.0;
    if constexpr (ACC) {
        if (ctl->acc_every <= 0 || ctl->step % ctl->acc_every != 0) return;
        dtw = ctl->t - ctl->acc_last_t;
        if (!(dtw > 0.0)) return;
    }
    __shared__ double red[5][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int iy = blockIdx.x; iy < Ny; iy += gridDim.x) {
        const int ym = (iy == 0 ? 0 : iy - 1), yp = (iy == Ny - 1 ? Ny - 1 : iy + 1);
        const double a = a_node[iy];
        double lu = 0.0, lv = 0.0, lu2 = 0.0, lv2 = 0.0, luv = 0.0;
        for (int ix = threadIdx.x; ix < Nx; ix += blockDim.x) {
            const int xm = (ix == 0 ? Nx - 1 : ix - 1), xp = (ix == Nx - 1 ? 0 : ix + 1);
            const double u = (psi[(size_t)yp * Nx + ix] - psi[(size_t)ym * Nx + ix]) * 0.5 * inv_deta * a;
            const double v = -(psi[(size_t)iy * Nx + xp] - psi[(size_t)iy * Nx + xm]) * 0.5 * inv_dx;
            lu += u; lv += v; lu2 += u * u; lv2 += v * v; luv += u * v;
        }
        double vals[5] = {lu, lv, lu2, lv2, luv};
#pragma unroll
        for (int q = 0; q < 5; ++q)
            for (int o = 16; o > 0; o >>= 1) vals[q] += __shfl_down_sync(0xffffffffu, vals[q], o);
        if (lane == 0)
            for (int q = 0; q < 5; ++q) red[q][warp] = vals[q];
        __syncthreads();
        if (threadIdx.x < 5) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[threadIdx.x][w];
            // rounded as the host rounds it (no fused multiply-add): the product, then the sum
            if constexpr (ACC)
                out[(size_t)threadIdx.x * Ny + iy] = __dadd_rn(out[(size_t)threadIdx.x * Ny + iy],
                                                               __dmul_rn(t / (double)Nx, dtw));
            else out[(size_t)threadIdx.x * Ny + iy] = t;
        }
        __syncthreads();
    }
}

int row_moments(Context* c, double* out5, cudaStream_t s) {
    if (!c->moments) {
        NSE_CUDA_TRY(cudaMalloc((void**)&c->moments, sizeof(double) * 5 * (size_t)c->Ny));
    }
    const int grid = std::min(c->Ny, 8 * c->num_sms);
    k_row_moments<false><<<grid, 256, 0, s>>>(c->psi, c->rt.a_node, c->Nx, c->Ny, c->inv_dx, c->inv_deta, c->moments,
                                              c->ctl);
    NSE_CUDA_TRY(cudaGetLastError());
    NSE_CUDA_TRY(cudaMemcpyAsync(out5, c->moments, sizeof(double) * 5 * (size_t)c->Ny, cudaMemcpyDeviceToHost, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
}

// after the accumulation of a statistics step: the weight and the time of the last sample
static __global__ void k_stats_commit(Ctl* ctl) {
    if (threadIdx.x != 0 || ctl->acc_every <= 0 || ctl->step % ctl->acc_every != 0) return;
    const double dtw = ctl->t - ctl->acc_last_t;
    if (!(dtw > 0.0)) return;
    ctl->acc_T += dtw;
    ctl->acc_last_t = ctl->t;
}

// The statistics kernels of one step of the run loop (they return at once except at a
// statistics step); the accumulator must exist (stats_device).
int enqueue_stats(Context* c, cudaStream_t s) {
    const int grid = std::min(c->Ny, 8 * c->num_sms);
    k_row_moments<true><<<grid, 256, 0, s>>>(c->psi, c->rt.a_node, c->Nx, c->Ny, c->inv_dx, c->inv_deta, c->stats_acc,
                                             c->ctl);
    NSE_CUDA_TRY(cudaGetLastError());
    k_stats_commit<<<1, 32, 0, s>>>(c->ctl);
    NSE_CUDA_TRY(cudaGetLastError());
    return 0;
}

// Accumulate on the device every `every` steps of the run loop (0: off), from now on: the
// accumulators start at zero and the clock at the current t.
int stats_device(Context* c, int every, cudaStream_t s) {
    if (every < 0) { set_error("nse2d_stats_device: every must be >= 0"); return -1; }
    if (every > 0 && c->prec32) {
        set_error("nse2d_stats_device: statistics on the device need precision 64");
        return -1;
    }
    if (every > 0 && !c->stats_acc) NSE_CUDA_TRY(cudaMalloc((void**)&c->stats_acc, sizeof(double) * 5 * (size_t)c->Ny));
    if (c->stats_acc) NSE_CUDA_TRY(cudaMemsetAsync(c->stats_acc, 0, sizeof(double) * 5 * (size_t)c->Ny, s));
    NSE_CUDA_TRY(cudaMemcpyAsync(c->h_ctl, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    Ctl* h = c->h_ctl;
    h->acc_every = every;
    h->acc_last_t = h->t;
    h->acc_T = 0.0;
    const size_t off = offsetof(Ctl, acc_every), len = offsetof(Ctl, acc_T) + sizeof(double) - off;
    NSE_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<char*>(c->ctl) + off, reinterpret_cast<char*>(h) + off, len,
                                 cudaMemcpyHostToDevice, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    const bool on = every > 0;
    if (on != c->stats_dev) {
        // the run graph holds the statistics kernels only when they are on: capture it again
        if (c->run_exec) { cudaGraphExecDestroy(c->run_exec); c->run_exec = nullptr; }
        c->stats_dev = on;
    }
    return 0;
}

int stats_read(Context* c, double* out5, double* T, cudaStream_t s) {
    NSE_CUDA_TRY(cudaMemcpyAsync(c->h_ctl, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    if (out5) {
        if (c->stats_acc)
            NSE_CUDA_TRY(cudaMemcpyAsync(out5, c->stats_acc, sizeof(double) * 5 * (size_t)c->Ny, cudaMemcpyDeviceToHost, s));
        else
            for (size_t k = 0; k < 5 * (size_t)c->Ny; ++k) out5[k] = 0.0;
    }
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    if (T) *T = c->h_ctl->acc_T;
    return 0;
}

// ---- 1-D energy spectra in x (src/diag.cuh:123-191, src/diag.cu:868-898) ----
// E(k) += w_k / (Nx^2 Ny) sum_j |f-hat_j(k)|^2 for k = 0..Nx/2, w_k = 2 inside the half
// spectrum and 1 at k = 0 and Nx/2, summed over the rows in row order (one thread per k).
static __global__ void k_spectra_reduce(const cpx<double>* __restrict__ hat, int Ny, int Hp, int H, double norm,
                                        double* __restrict__ acc) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= H) return;
    const double wx = (k > 0 && k < H - 1) ? 2.0 : 1.0;
    double sum = 0.0;
    for (int j = 0; j < Ny; ++j) {
        const cpx<double> z = hat[(size_t)j * Hp + k];
        sum += (z.x * z.x + z.y * z.y);
    }
    acc[k] += norm * wx * sum;
}

// One sample of E_u, E_v from device u, v [Ny][Nx] (16-byte aligned): the row transforms of the
// spectral buffer, then the sums over rows of |X_k|^2 (src/diag.cu:868-898).
int spectra_accumulate_uv(Context* c, const double* u, const double* v, cudaStream_t s) {
    if (!c->spec_acc) {
        NSE_CUDA_TRY(cudaMalloc((void**)&c->spec_acc, sizeof(double) * 2 * (size_t)c->Hp));
        NSE_CUDA_TRY(cudaMemsetAsync(c->spec_acc, 0, sizeof(double) * 2 * (size_t)c->Hp, s));
        c->spec_samples = 0;
    }
    const double norm = 1.0 / ((double)c->Nx * (double)c->Nx * (double)c->Ny);
    const int tb = 128, gb = (c->H + tb - 1) / tb;
    for (int q = 0; q < 2; ++q) {
        if (launch_fft_all_rows(c, q == 0 ? u : v, s)) return -1;
        k_spectra_reduce<<<gb, tb, 0, s>>>(c->hat, c->Ny, c->Hp, c->H, norm, c->spec_acc + (size_t)q * c->Hp);
        NSE_CUDA_TRY(cudaGetLastError());
    }
    c->spec_samples += 1;
    return 0;
}

// One spectra sample of the current psi: u and v into the stage buffers (free between steps).
int spectra_accumulate(Context* c, cudaStream_t s) {
    if (uv_from_psi(c, c->psi, c->w1, c->w2, s)) return -1;
    return spectra_accumulate_uv(c, c->w1, c->w2, s);
}

}  // namespace nse2d
