// FP32-bulk variant of the time step, with FP64 islands. Written for this project (no
// counterpart in the reference, which is FP64 throughout).
//
// Why a plain FP32 copy cannot work: the Thom closure multiplies psi next to the wall by
// ~2/dy_1^2 (1e8 on the 4096x2049 tanh grid), and psi there is ~psi_top = 2 h Ub, whose FP32
// rounding (~2e-7) would put O(10) errors into the wall vorticity.
//
// The split: omega = wbar(y) + w' and psi = psibar(y) + psi', with the base profiles wbar, psibar
// FP64 and fixed (the x-means of the initial state; psibar carries the wall values, so psi' is 0
// on both walls and tiny next to them), and the fluctuations w', psi' stored and stepped in FP32.
// Since the base is steady, w' obeys the same Shu-Osher combines with the full rhs.
//   - Stage (k_stage32): the Arakawa sum S of the full fields is S'(psi', w') plus base terms
//     that are FP64 row differences times x-differences of the fluctuations (the x-differences
//     of the base vanish):
//       -2 D psibar Dx w'_j - d+ psibar Dx w'_{j+1} - d- psibar Dx w'_{j-1}
//       +2 D wbar Dx psi'_j + d+ wbar Dx psi'_{j+1} + d- wbar Dx psi'_{j-1},
//     D f = f_{j+1} - f_{j-1}, d+ f = f_{j+1} - f_j, d- f = f_j - f_{j-1}; the base's Laplacian,
//     forcing and drag enter as one FP64 row constant R_j.
//   - Poisson: FP32 row transforms (k_fft_fwd32 / k_ifft_thom32) with the spectral buffer and the
//     whole tridiagonal solve in FP64 (homogeneous Dirichlet for psi', including kx = 0, whose
//     operator is the badly conditioned one).
//   - Thom: w'_wall = [Thom(psibar) - wbar]_wall (FP64 constant) - (A psi'_1 + B psi'_2).
//   - dt: the max reduction over FP32 psi' plus the FP64 base slope.
// The FP64 fields of the context are filled from the split state (export) for diagnostics and
// output.
#pragma once
#include "step_kernels.cuh"

namespace nse2d {

// Row constants of the FP32 stage, [RC32_N][Ny] floats: the regrouped stencil's factors and the
// base-profile terms.
enum { RC_CJ = 0, RC_AP, RC_AM, RC_DPB, RC_DPP, RC_DPM, RC_DWB, RC_DWP, RC_DWM, RC_R, RC32_N };

// ---- state conversion ----
// w, psi (FP64 fields) -> base means wbar, psibar (FP64, fixed-order row reductions) and the
// FP32 fluctuations. One CTA per row.
static __global__ void __launch_bounds__(256) k_split32(const double* __restrict__ w, const double* __restrict__ psi,
                                                       int Nx, int Ny, double* __restrict__ wbar,
                                                       double* __restrict__ psibar, float* __restrict__ wf,
                                                       float* __restrict__ psif) {
    __shared__ double red[2][8];
    __shared__ double mean[2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j = blockIdx.x; j < Ny; j += gridDim.x) {
        const double* rw = w + (size_t)j * Nx;
        const double* rp = psi + (size_t)j * Nx;
        double sw = 0.0, sp = 0.0;
        for (int i = threadIdx.x; i < Nx; i += blockDim.x) { sw += rw[i]; sp += rp[i]; }
        for (int o = 16; o > 0; o >>= 1) {
            sw += __shfl_down_sync(0xffffffffu, sw, o);
            sp += __shfl_down_sync(0xffffffffu, sp, o);
        }
        if (lane == 0) { red[0][warp] = sw; red[1][warp] = sp; }
        __syncthreads();
        if (threadIdx.x < 2) {
            double t = 0.0;
            for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[threadIdx.x][q];
            mean[threadIdx.x] = t / (double)Nx;
        }
        __syncthreads();
        const double mw = mean[0], mp = mean[1];
        if (threadIdx.x == 0) { wbar[j] = mw; psibar[j] = mp; }
        for (int i = threadIdx.x; i < Nx; i += blockDim.x) {
            wf[(size_t)j * Nx + i] = (float)(rw[i] - mw);
            psif[(size_t)j * Nx + i] = (float)(rp[i] - mp);
        }
        __syncthreads();
    }
}

// Full FP64 fields from the split state: dst = base_j + fluct.
static __global__ void k_join32(const double* __restrict__ base, const float* __restrict__ f, double* __restrict__ dst,
                                int Nx, int Ny) {
    const size_t n = (size_t)Nx * Ny;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        dst[k] = base[k / (size_t)Nx] + (double)f[k];
}

static __global__ void k_widen32(const float* __restrict__ f, double* __restrict__ dst, size_t n) {
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        dst[k] = (double)f[k];
}

// Row constants from the base profiles (FP64 arithmetic, stored as floats), one thread per row.
static __global__ void k_rowconst32(RowTables rt, const double* __restrict__ wbar, const double* __restrict__ psibar,
                                    int Ny, double inv4dxde, double nu, double inv_deta2, double lin_drag,
                                    float* __restrict__ rc) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= Ny) return;
    double v[RC32_N] = {0};
    const double f = rt.frow[j];
    if (j >= 1 && j <= Ny - 2) {
        const double an = rt.a_node[j], aep = rt.a_edge[j], aem = rt.a_edge[j - 1];
        v[RC_CJ] = an * (inv4dxde * (1.0 / 3.0));
        v[RC_AP] = nu * (an * aep * inv_deta2);
        v[RC_AM] = nu * (an * aem * inv_deta2);
        v[RC_DPB] = psibar[j + 1] - psibar[j - 1];
        v[RC_DPP] = psibar[j + 1] - psibar[j];
        v[RC_DPM] = psibar[j] - psibar[j - 1];
        v[RC_DWB] = wbar[j + 1] - wbar[j - 1];
        v[RC_DWP] = wbar[j + 1] - wbar[j];
        v[RC_DWM] = wbar[j] - wbar[j - 1];
        const double lapy = an * (aep * (wbar[j + 1] - wbar[j]) - aem * (wbar[j] - wbar[j - 1])) * inv_deta2;
        v[RC_R] = nu * lapy + f - lin_drag * wbar[j];
    } else {
        v[RC_R] = f - lin_drag * wbar[j];
    }
    for (int q = 0; q < RC32_N; ++q) rc[(size_t)q * Ny + j] = (float)v[q];
}

// ---- k_stage32: one CTA per 64 x 32 tile, FP32 halo in shared memory ----
struct Stage32Params {
    const float* psi;        // psi'
    const float* w_in;       // w'^(s)
    const float* w_n;        // w'^n (stages 2, 3)
    float* w_out;            // w'^(s+1)
    float* rhs_out;          // optional: the stage rhs
    const float* rc;         // [RC32_N][Ny]
    const Ctl* ctl;
    int Nx, Ny, stage;
    float nu_dx2, lin_drag;
};

static __global__ void __launch_bounds__(256) k_stage32(Stage32Params p) {
    __shared__ float sp[ST_H][ST_W + 1];
    __shared__ float so[ST_H][ST_W + 1];
    const int Nx = p.Nx, Ny = p.Ny;
    const int x0 = blockIdx.x * ST_TX, y0 = blockIdx.y * ST_TY;
    constexpr int NLD = (ST_H * ST_W + 255) / 256;
    {
        float vp[NLD], vo[NLD];
#pragma unroll
        for (int u = 0; u < NLD; ++u) {
            const int idx = threadIdx.x + 256 * u;
            const int r = idx / ST_W, c = idx - r * ST_W;
            const int gy = y0 - 1 + r;
            int gx = x0 - 1 + c;
            gx = (Nx >= ST_TX) ? (gx < 0 ? gx + Nx : (gx >= Nx ? gx - Nx : gx)) : ((gx % Nx) + Nx) % Nx;
            vp[u] = 0.f;
            vo[u] = 0.f;
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
    const double dtd = p.ctl->dt;
    const float dt = (float)dtd;
    const int lx = threadIdx.x & (ST_TX - 1), g = threadIdx.x / ST_TX;
    const int i = x0 + lx;
    if (i >= Nx) return;
    const int ly0 = g * ST_RPT;
    float ps[3][3], om[3][3], dxp[3], dxo[3];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c) { ps[r + 1][c] = sp[ly0 + r][lx + c]; om[r + 1][c] = so[ly0 + r][lx + c]; }
        dxp[r + 1] = ps[r + 1][2] - ps[r + 1][0];
        dxo[r + 1] = om[r + 1][2] - om[r + 1][0];
    }
    const float* rc = p.rc;
#pragma unroll
    for (int q = 0; q < ST_RPT; ++q) {
        const int ly = ly0 + q, j = y0 + ly;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            ps[0][c] = ps[1][c]; ps[1][c] = ps[2][c]; ps[2][c] = sp[ly + 2][lx + c];
            om[0][c] = om[1][c]; om[1][c] = om[2][c]; om[2][c] = so[ly + 2][lx + c];
        }
        dxp[0] = dxp[1]; dxp[1] = dxp[2]; dxp[2] = ps[2][2] - ps[2][0];
        dxo[0] = dxo[1]; dxo[1] = dxo[2]; dxo[2] = om[2][2] - om[2][0];
        if (j >= Ny) break;
        const float wc = om[1][1];
        float rhs = fmaf(-p.lin_drag, wc, __ldg(&rc[(size_t)RC_R * Ny + j]));
        if (j != 0 && j != Ny - 1) {
            const float dyo_m = om[2][0] - om[0][0], dyo_c = om[2][1] - om[0][1], dyo_p = om[2][2] - om[0][2];
            const float dyp_m = ps[2][0] - ps[0][0], dyp_c = ps[2][1] - ps[0][1], dyp_p = ps[2][2] - ps[0][2];
            float s1 = dxp[1] * dyo_c;
            s1 = fmaf(-dyp_c, dxo[1], s1);
            s1 = fmaf(ps[1][2], dyo_p, s1);
            s1 = fmaf(-ps[1][0], dyo_m, s1);
            s1 = fmaf(-ps[2][1], dxo[2], s1);
            s1 = fmaf(ps[0][1], dxo[0], s1);
            float s2 = -om[1][2] * dyp_p;
            s2 = fmaf(om[1][0], dyp_m, s2);
            s2 = fmaf(om[2][1], dxp[2], s2);
            s2 = fmaf(-om[0][1], dxp[0], s2);
            // the base profiles' share of S
            const float dpb = __ldg(&rc[(size_t)RC_DPB * Ny + j]), dpp = __ldg(&rc[(size_t)RC_DPP * Ny + j]);
            const float dpm = __ldg(&rc[(size_t)RC_DPM * Ny + j]), dwb = __ldg(&rc[(size_t)RC_DWB * Ny + j]);
            const float dwp = __ldg(&rc[(size_t)RC_DWP * Ny + j]), dwm = __ldg(&rc[(size_t)RC_DWM * Ny + j]);
            float s3 = -2.f * dpb * dxo[1];
            s3 = fmaf(-dpp, dxo[2], s3);
            s3 = fmaf(-dpm, dxo[0], s3);
            s3 = fmaf(2.f * dwb, dxp[1], s3);
            s3 = fmaf(dwp, dxp[2], s3);
            s3 = fmaf(dwm, dxp[0], s3);
            const float lapx = fmaf(-2.f, wc, om[1][2] + om[1][0]);
            const float ap = __ldg(&rc[(size_t)RC_AP * Ny + j]), am = __ldg(&rc[(size_t)RC_AM * Ny + j]);
            const float cj = __ldg(&rc[(size_t)RC_CJ * Ny + j]);
            rhs = fmaf(p.nu_dx2, lapx, rhs);
            rhs = fmaf(ap, om[2][1] - wc, rhs);
            rhs = fmaf(-am, wc - om[0][1], rhs);
            rhs = fmaf(cj, (s1 + s2) + s3, rhs);
        }
        const size_t id = (size_t)j * Nx + i;
        if (p.rhs_out) p.rhs_out[id] = rhs;
        float wnew;
        if (p.stage == 1) wnew = fmaf(dt, rhs, wc);
        else if (p.stage == 2) wnew = 0.75f * p.w_n[id] + 0.25f * fmaf(dt, rhs, wc);
        else wnew = (1.0f / 3.0f) * p.w_n[id] + (2.0f / 3.0f) * fmaf(dt, rhs, wc);
        p.w_out[id] = wnew;
    }
}

// ---- FP32 row transforms, FP64 spectral buffer ----
struct Fft32Params {
    const float* src;          // forward: rows of w'
    cpx<double>* hat;          // [Ny][Hp], FP64
    float* psi;                // inverse output psi'
    float* w;                  // inverse: w'^(s+1), whose wall rows the Thom closure sets
    const cpx<float>* tw;      // per-pass twiddles of the radix-16 plan (p16_twiddle_table), FP32
    const cpx<float>* wN;      // M + 1 split/merge twiddles, FP32
    const double* dy_edge;
    Ctl* ctl;
    int Nx, Ny, Hp, rows_per_cta, do_thom, advance, free_slip;
    double wall_bot, wall_top;  // [Thom(psibar) - wbar] at the walls (no slip), -wbar (free slip)
};

__host__ __device__ constexpr size_t fft32_smem_bytes(int M) { return (size_t)ip_size(M) * 8; }

template <int M>
static __global__ void __launch_bounds__(IP_NT) k_fft_fwd32(Fft32Params p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<float>* buf = reinterpret_cast<cpx<float>*>(smem_raw);
    const int j = 1 + blockIdx.x;                       // interior rows
    if (j > p.Ny - 2) return;
    const float2* row = reinterpret_cast<const float2*>(p.src + (size_t)j * p.Nx);
    constexpr int R0 = p16_plan<M>::R(0), NB0 = M / R0;
    // pass 0 from global (radix-16 plan of fft_rows.cuh): thread t transforms t + NB0 r
#pragma unroll 1
    for (int b0 = 0; b0 < NB0; b0 += IP_NT) {
        const int t = b0 + (int)threadIdx.x;
        if (NB0 % IP_NT != 0 && t >= NB0) break;
        cpx<float> v[R0];
#pragma unroll
        for (int r = 0; r < R0; ++r) {
            const float2 z = __ldg(row + t + NB0 * r);
            v[r] = {z.x, z.y};
        }
        dftR<float, R0, false>(v);
        const int p0 = dit16_pos<M>(t);
#pragma unroll
        for (int q = 0; q < R0; ++q) buf[ip_idx(p0 + q)] = v[q];
    }
    __syncthreads();
    p16_passes_from<float, M, 1, false, IP_NT>(buf, p.tw);
    // the split step for the pair (k, M - k) (see k_fft_fwd)
    double2* dst = reinterpret_cast<double2*>(p.hat + (size_t)j * p.Hp);
    for (int k = threadIdx.x; k <= M / 2; k += IP_NT) {
        const int kb = (k == 0 ? 0 : M - k);
        const cpx<float> a = buf[ip_idx(k)];
        const cpx<float> b = buf[ip_idx(kb)];
        const cpx<float> sm = {0.5f * (a.x + b.x), 0.5f * (a.y - b.y)};
        const cpx<float> df = {0.5f * (a.x - b.x), 0.5f * (a.y + b.y)};
        const cpx<float> X = cadd(sm, cmul(ldtw(p.wN, k), mul_mi(df)));
        dst[k] = make_double2((double)X.x, (double)X.y);
        if (k < M / 2) {
            const int m = M - k;
            const cpx<float> Y = cadd(cpx<float>{sm.x, -sm.y}, cmul(ldtw(p.wN, m), cpx<float>{df.y, df.x}));
            dst[m] = make_double2((double)Y.x, (double)Y.y);
        }
    }
}

template <int M>
static __global__ void __launch_bounds__(IP_NT, 5) k_ifft_thom32(Fft32Params p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<float>* buf = reinterpret_cast<cpx<float>*>(smem_raw);
    const int Nx = p.Nx, Ny = p.Ny;
    int j0, j1;
    band_of(blockIdx.x, gridDim.x, p.rows_per_cta, Ny, j0, j1);
    constexpr float scale = 1.0f / (float)M;
    constexpr int R0 = p16_plan<M>::R(0), NB0 = M / R0;
    for (int j = j0; j < j1; ++j) {
        float* dst = p.psi + (size_t)j * Nx;
        if (j == 0 || j == Ny - 1) {                    // psi' = 0 on the walls
            for (int i = threadIdx.x; i < Nx; i += IP_NT) dst[i] = 0.f;
            continue;
        }
        // pass 0 from global with the merge (see k_ifft_thom)
        const double2* X = reinterpret_cast<const double2*>(p.hat + (size_t)j * p.Hp);
#pragma unroll 1
        for (int b0 = 0; b0 < NB0; b0 += IP_NT) {
            const int t = b0 + (int)threadIdx.x;
            if (NB0 % IP_NT != 0 && t >= NB0) break;
            cpx<float> v[R0];
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int n = t + NB0 * r;
                const double2 av = __ldcs(X + n), bv = __ldcs(X + (M - n));
                const cpx<float> a = {(float)av.x, (float)av.y}, b = {(float)bv.x, -(float)bv.y};
                const cpx<float> E = {0.5f * (a.x + b.x), 0.5f * (a.y + b.y)};
                const cpx<float> D = {0.5f * (a.x - b.x), 0.5f * (a.y - b.y)};
                v[r] = cadd(E, mul_pi(cmulc(D, ldtw(p.wN, n))));
            }
            dftR<float, R0, true>(v);
            const int p0 = dit16_pos<M>(t);
#pragma unroll
            for (int q = 0; q < R0; ++q) buf[ip_idx(p0 + q)] = v[q];
        }
        __syncthreads();
        p16_passes_from<float, M, 1, true, IP_NT>(buf, p.tw);
        for (int n = threadIdx.x; n < M; n += IP_NT) {
            const cpx<float> z = buf[ip_idx(n)];
            reinterpret_cast<float2*>(dst)[n] = make_float2(z.x * scale, z.y * scale);
        }
        __syncthreads();
    }
    if (p.do_thom) {
        // w'_wall = [Thom(psibar) - wbar]_wall - (A psi'_1 + B psi'_2) (src/ops.cu:114-151 on the split)
        for (int side = 0; side < 2; ++side) {
            const bool top = side == 1;
            if (!(top ? (j0 <= Ny - 3 && j1 >= Ny - 1) : (j0 <= 1 && j1 >= 3))) continue;
            const double d1 = top ? p.dy_edge[Ny - 2] : p.dy_edge[0];
            const double d2 = top ? p.dy_edge[Ny - 3] : p.dy_edge[1];
            const float A = (float)(2.0 * (1.0 / (d1 * d1) + 1.0 / (d1 * d2)));
            const float B = (float)((-2.0) * d1 / (d2 * (d1 + d2) * (d1 + d2)));
            const float base = (float)(top ? p.wall_top : p.wall_bot);     // -wbar_wall with free-slip walls
            const float* r1 = p.psi + (size_t)(top ? Ny - 2 : 1) * Nx;
            const float* r2 = p.psi + (size_t)(top ? Ny - 3 : 2) * Nx;
            float* wr = p.w + (size_t)(top ? Ny - 1 : 0) * Nx;
            for (int i = threadIdx.x; i < Nx; i += IP_NT)
                wr[i] = p.free_slip ? base : base - (A * __ldcg(&r1[i]) + B * __ldcg(&r2[i]));
        }
    }
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
            p.ctl->ifft_done = 0;
            advance_time(p.ctl);
        }
    }
}

// ---- max |u|, |v|, |v| a of psibar + psi' ----
// The item layout of k_maxuv_dt: (column strip, row band) items, a window of rows j-1, j, j+1
// in registers down the band, MX_U rows loaded at a time; here a thread holds 4 columns (one
// 16-byte load per row; Nx is a power of two >= 4), so a strip is MX32_COLS columns, and the x
// neighbours c-1 and c+4 come from the adjacent lanes.
struct Max32Params {
    MaxParams base;          // a_node, partials, control block, dt constants, items (base.psi unused)
    const float* psi;        // psi'
    const float* dpsibar;    // [Ny]: psibar_{j+1} - psibar_{j-1} (the RC_DPB row constant)
};
constexpr int MX32_COLS = 1024;

static __global__ void __launch_bounds__(256, 3) k_maxuv32(Max32Params q) {
    const MaxParams& p = q.base;
    const int Nx = p.Nx, Ny = p.Ny;
    const int lane = threadIdx.x & 31;
    double um = 0.0, vm = 0.0, vmm = 0.0;
    float probe = 0.f;
    const double cy = 0.5 * p.inv_deta, cx = 0.5 * p.inv_dx;
    const int nitems = p.nstrips * p.nbands;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int strip = item % p.nstrips, band = item / p.nstrips;
        const int c0 = strip * MX32_COLS + 4 * (int)threadIdx.x;
        const bool act = c0 < Nx;
        const int cs = act ? c0 : 0;
        const int cl = cs > 0 ? cs - 1 : Nx - 1, cr = cs + 4 < Nx ? cs + 4 : 0;
        const int j0 = 1 + band * p.band_rows, j1 = min(Ny - 1, j0 + p.band_rows);
        const bool ldl = act && lane == 0, ldr = act && (lane == 31 || c0 + 4 >= Nx);
        auto ld4 = [&](int row) { return __ldg(reinterpret_cast<const float4*>(q.psi + (size_t)row * Nx + cs)); };
        float4 w0 = ld4(j0 - 1), w1 = ld4(j0);
        for (int j = j0; j < j1; j += MX_U) {
            float4 nx[MX_U];
            float el[MX_U], er[MX_U], db[MX_U];
            double an[MX_U];
#pragma unroll
            for (int u = 0; u < MX_U; ++u) {
                const int jc = min(j + u, j1 - 1);
                nx[u] = ld4(jc + 1);
                const float* rc = q.psi + (size_t)jc * Nx;
                el[u] = ldl ? __ldg(rc + cl) : 0.f;
                er[u] = ldr ? __ldg(rc + cr) : 0.f;
                db[u] = __ldg(&q.dpsibar[jc]);
                an[u] = __ldg(&p.a_node[jc]);
            }
#pragma unroll
            for (int u = 0; u < MX_U; ++u) {
                const float4 wc = (u == 0) ? w1 : nx[u - 1];
                const float4 wm = (u == 0) ? w0 : (u == 1 ? w1 : nx[u - 2]);
                const float sl = __shfl_up_sync(0xffffffffu, wc.w, 1);
                const float sr = __shfl_down_sync(0xffffffffu, wc.x, 1);
                const float xl = ldl ? el[u] : sl, xr = ldr ? er[u] : sr;
                if (j + u >= j1 || !act) continue;
                const float d = db[u];
                const float e0 = (nx[u].x - wm.x) + d, e1 = (nx[u].y - wm.y) + d;
                const float e2 = (nx[u].z - wm.z) + d, e3 = (nx[u].w - wm.w) + d;
                const float f0 = wc.y - xl, f1 = wc.z - wc.x, f2 = wc.w - wc.y, f3 = xr - wc.z;
                const float dym = fmaxf(fmaxf(fabsf(e0), fabsf(e1)), fmaxf(fabsf(e2), fabsf(e3)));
                const float dxm = fmaxf(fmaxf(fabsf(f0), fabsf(f1)), fmaxf(fabsf(f2), fabsf(f3)));
                probe += ((e0 + e1) + (e2 + e3)) + ((f0 + f1) + (f2 + f3));
                const double a = an[u];
                const double av = (double)dxm * cx;
                um = fmax(um, a * ((double)dym * cy));
                vm = fmax(vm, av);
                vmm = fmax(vmm, av * a);
            }
            w0 = nx[MX_U - 2]; w1 = nx[MX_U - 1];
        }
    }
    const int nonfinite = !(probe - probe == 0.f) || !(um <= 1e300) || !(vm <= 1e300);
    maxuv_finish(p, um, vm, vmm, nonfinite);
}

}  // namespace nse2d
