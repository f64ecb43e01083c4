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
//   - Stage (k_stage32_tma; k_stage32 below 256 columns): the Arakawa sum S of the full fields
//     is S'(psi', w') plus base terms
//     that are FP64 row differences times x-differences of the fluctuations (the x-differences
//     of the base vanish):
//       -2 D psibar Dx w'_j - d+ psibar Dx w'_{j+1} - d- psibar Dx w'_{j-1}
//       +2 D wbar Dx psi'_j + d+ wbar Dx psi'_{j+1} + d- wbar Dx psi'_{j-1},
//     D f = f_{j+1} - f_{j-1}, d+ f = f_{j+1} - f_j, d- f = f_j - f_{j-1}; the base's Laplacian,
//     forcing and drag enter as one FP64 row constant R_j.
//   - Poisson: FP32 row transforms (k_fft_fwd32 / k_ifft_thom32) and an FP32 spectral buffer; the
//     tridiagonal solve widens the spectra on load and runs in FP64 with the FP64 elimination table
//     (homogeneous Dirichlet for psi', including kx = 0). Rounding the right-hand side and the
//     solution to FP32 perturbs psi' by ~1e-8 relative at every kx, while an FP32 table or FP32
//     sweeps would lose 1e-6 .. 1e-4 at the low kx, whose operators are badly conditioned.
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

// The row constants of an interior row j that the stage reads.
struct Rc32Row {
    float dpb, dpp, dpm, dwb, dwp, dwm, ap, am, cj;
};
__device__ __forceinline__ Rc32Row rc32_row(const float* rc, int Ny, int j) {
    Rc32Row k;
    k.dpb = __ldg(&rc[(size_t)RC_DPB * Ny + j]); k.dpp = __ldg(&rc[(size_t)RC_DPP * Ny + j]);
    k.dpm = __ldg(&rc[(size_t)RC_DPM * Ny + j]); k.dwb = __ldg(&rc[(size_t)RC_DWB * Ny + j]);
    k.dwp = __ldg(&rc[(size_t)RC_DWP * Ny + j]); k.dwm = __ldg(&rc[(size_t)RC_DWM * Ny + j]);
    k.ap = __ldg(&rc[(size_t)RC_AP * Ny + j]); k.am = __ldg(&rc[(size_t)RC_AM * Ny + j]);
    k.cj = __ldg(&rc[(size_t)RC_CJ * Ny + j]);
    return k;
}

// rhs of one interior point from its 3 x 3 neighbourhood: S'(psi', w') + the base profiles'
// share of S, the mapped Laplacian and the forcing row constant (already in rhs). p_xm, p_xp,
// p_ym, p_yp are psi' at x-1, x+1, y-1, y+1 (likewise o_ for w'); dxp/dxo[r] the x differences
// of rows j-1, j, j+1. Both FP32 stage kernels call it, so they give the same bits.
__device__ __forceinline__ float stage32_rhs_interior(float rhs, float wc, float p_xm, float p_xp, float p_ym,
                                                      float p_yp, float dyp_m, float dyp_c, float dyp_p,
                                                      const float (&dxp)[3], float o_xm, float o_xp, float o_ym,
                                                      float o_yp, float dyo_m, float dyo_c, float dyo_p,
                                                      const float (&dxo)[3], float nu_dx2, const Rc32Row& k) {
    float s1 = dxp[1] * dyo_c;
    s1 = fmaf(-dyp_c, dxo[1], s1);
    s1 = fmaf(p_xp, dyo_p, s1);
    s1 = fmaf(-p_xm, dyo_m, s1);
    s1 = fmaf(-p_yp, dxo[2], s1);
    s1 = fmaf(p_ym, dxo[0], s1);
    float s2 = -o_xp * dyp_p;
    s2 = fmaf(o_xm, dyp_m, s2);
    s2 = fmaf(o_yp, dxp[2], s2);
    s2 = fmaf(-o_ym, dxp[0], s2);
    // the base profiles' share of S
    float s3 = -2.f * k.dpb * dxo[1];
    s3 = fmaf(-k.dpp, dxo[2], s3);
    s3 = fmaf(-k.dpm, dxo[0], s3);
    s3 = fmaf(2.f * k.dwb, dxp[1], s3);
    s3 = fmaf(k.dwp, dxp[2], s3);
    s3 = fmaf(k.dwm, dxp[0], s3);
    const float lapx = fmaf(-2.f, wc, o_xp + o_xm);
    rhs = fmaf(nu_dx2, lapx, rhs);
    rhs = fmaf(k.ap, o_yp - wc, rhs);
    rhs = fmaf(-k.am, wc - o_ym, rhs);
    return fmaf(k.cj, (s1 + s2) + s3, rhs);
}

static __global__ void __launch_bounds__(256) k_stage32(Stage32Params p) {
    pdl_begin();
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
            const Rc32Row k = rc32_row(rc, Ny, j);
            rhs = stage32_rhs_interior(rhs, wc, ps[1][0], ps[1][2], ps[0][1], ps[2][1], dyp_m, dyp_c, dyp_p, dxp,
                                       om[1][0], om[1][2], om[0][1], om[2][1], dyo_m, dyo_c, dyo_p, dxo, p.nu_dx2, k);
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

// ---- k_stage32_tma: persistent CTAs, halos moved by the tensor memory accelerator ----
// The scheme of the FP64 k_stage_tma with FP32 boxes: tiles of S32_TX x S32_TY points, the halo
// boxes of psi' and w'^(s) (S32_W x S32_H, starting at column x0 - 4 so that x is a multiple of
// 16 bytes) and the w'^n tile box of the next tile in flight while the current one is
// computed; the periodic columns -1 and Nx of the first and last tile column are patched with
// plain loads. Warp g takes tile rows 4g .. 4g + 3, lane l the columns x0 + 4l .. x0 + 4l + 3: a
// row of the window (columns x - 1 .. x + 4) is three 16-byte shared loads, the four points
// share their y differences, and the results leave as 16-byte stores. A wait that does not
// complete within kTmaWaitLimit polls sets bit 1 of the error flags and ends the CTA.
constexpr int S32_TX = 128, S32_TY = 32, S32_W = S32_TX + 8, S32_H = S32_TY + 2, S32_RPT = 4;
constexpr int S32_FIELD = ((S32_H * S32_W * 4 + 127) / 128) * 128;
constexpr int S32_WN = S32_TX * S32_TY * 4;
constexpr int S32_BUF = 2 * S32_FIELD + S32_WN;
constexpr unsigned S32_TX_BYTES = 2u * S32_H * S32_W * 4;
static_assert(8 * S32_RPT == S32_TY && 32 * 4 == S32_TX, "4 columns x 32 lanes, 4 rows x 8 warps");
__host__ __device__ constexpr size_t stage32_tma_smem_bytes() { return 2 * (size_t)S32_BUF + 128; }

struct Stage32Maps {
    CUtensorMap psi, w;      // halo boxes (S32_W x S32_H)
    CUtensorMap wn;          // w'^n tile box (S32_TX x S32_TY), stages 2 and 3
};

// srow[q][r]: the row constant q (RC_*) of tile row r, staged by the kernel for the tile.
__device__ __forceinline__ void stage32_tile4(const Stage32Params& p, float dt, const float* sp, const float* so,
                                              const float* swn, int x0, int y0, const float (*srow)[S32_TY]) {
    const int Nx = p.Nx, Ny = p.Ny;
    const int l = threadIdx.x & 31, g = threadIdx.x >> 5;
    const int ly0 = g * S32_RPT;                        // tile row ly <-> box row ly + 1
    float P[3][6], O[3][6];                             // rows j-1, j, j+1 x columns x0+4l-1 .. x0+4l+4
    float dxp[4][3], dxo[4][3];                         // per point, rows j-1, j, j+1
    auto ld_row = [&](const float* f, int r, float (&v)[6]) {
        const float4* q = reinterpret_cast<const float4*>(f + r * S32_W + 4 * l);
        const float4 a = q[0], b = q[1], c = q[2];
        v[0] = a.w; v[1] = b.x; v[2] = b.y; v[3] = b.z; v[4] = b.w; v[5] = c.x;
    };
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        ld_row(sp, ly0 + r, P[r + 1]);
        ld_row(so, ly0 + r, O[r + 1]);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            dxp[k][r + 1] = P[r + 1][k + 2] - P[r + 1][k];
            dxo[k][r + 1] = O[r + 1][k + 2] - O[r + 1][k];
        }
    }
#pragma unroll
    for (int q = 0; q < S32_RPT; ++q) {
        const int ly = ly0 + q, j = y0 + ly;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            P[0][c] = P[1][c]; P[1][c] = P[2][c];
            O[0][c] = O[1][c]; O[1][c] = O[2][c];
        }
        ld_row(sp, ly + 2, P[2]);
        ld_row(so, ly + 2, O[2]);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            dxp[k][0] = dxp[k][1]; dxp[k][1] = dxp[k][2]; dxp[k][2] = P[2][k + 2] - P[2][k];
            dxo[k][0] = dxo[k][1]; dxo[k][1] = dxo[k][2]; dxo[k][2] = O[2][k + 2] - O[2][k];
        }
        if (j >= Ny) break;
        const float fr = srow[RC_R][ly];
        float rhs[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) rhs[k] = fmaf(-p.lin_drag, O[1][k + 1], fr);
        if (j != 0 && j != Ny - 1) {
            float dyo[6], dyp[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) { dyo[c] = O[2][c] - O[0][c]; dyp[c] = P[2][c] - P[0][c]; }
            Rc32Row kr;
            kr.dpb = srow[RC_DPB][ly]; kr.dpp = srow[RC_DPP][ly]; kr.dpm = srow[RC_DPM][ly];
            kr.dwb = srow[RC_DWB][ly]; kr.dwp = srow[RC_DWP][ly]; kr.dwm = srow[RC_DWM][ly];
            kr.ap = srow[RC_AP][ly]; kr.am = srow[RC_AM][ly]; kr.cj = srow[RC_CJ][ly];
#pragma unroll
            for (int k = 0; k < 4; ++k)
                rhs[k] = stage32_rhs_interior(rhs[k], O[1][k + 1], P[1][k], P[1][k + 2], P[0][k + 1], P[2][k + 1],
                                              dyp[k], dyp[k + 1], dyp[k + 2], dxp[k], O[1][k], O[1][k + 2],
                                              O[0][k + 1], O[2][k + 1], dyo[k], dyo[k + 1], dyo[k + 2], dxo[k],
                                              p.nu_dx2, kr);
        }
        const size_t id = (size_t)j * Nx + x0 + 4 * l;
        if (p.rhs_out) *reinterpret_cast<float4*>(p.rhs_out + id) = make_float4(rhs[0], rhs[1], rhs[2], rhs[3]);
        float wn[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) wn[k] = fmaf(dt, rhs[k], O[1][k + 1]);
        if (p.stage > 1) {
            const float4 n4 = *reinterpret_cast<const float4*>(swn + ly * S32_TX + 4 * l);
            const float nn[4] = {n4.x, n4.y, n4.z, n4.w};
#pragma unroll
            for (int k = 0; k < 4; ++k)
                wn[k] = (p.stage == 2) ? 0.75f * nn[k] + 0.25f * wn[k] : (1.0f / 3.0f) * nn[k] + (2.0f / 3.0f) * wn[k];
        }
        *reinterpret_cast<float4*>(p.w_out + id) = make_float4(wn[0], wn[1], wn[2], wn[3]);
    }
}

static __global__ void __launch_bounds__(256, 2) k_stage32_tma(const __grid_constant__ Stage32Maps maps, Stage32Params p) {
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    pdl_begin();
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ float srow[2][RC32_N][S32_TY];          // per buffer: the row constants of its tile
    unsigned char* smem_raw = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);
    const int Nx = p.Nx, Ny = p.Ny;
    const int tiles_x = Nx / S32_TX, ntiles = tiles_x * ((Ny + S32_TY - 1) / S32_TY);
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        fence_proxy_async_smem();
    }
    __syncthreads();
    auto issue = [&](int tile, int b) {
        const int tx = tile % tiles_x, ty = tile / tiles_x;
        unsigned char* dst = smem_raw + b * S32_BUF;
        mbar_expect_tx(&bars[b], S32_TX_BYTES + (p.stage > 1 ? (unsigned)S32_WN : 0u));
        tma_load_2d(dst, &maps.psi, tx * S32_TX - 4, ty * S32_TY - 1, &bars[b]);
        tma_load_2d(dst + S32_FIELD, &maps.w, tx * S32_TX - 4, ty * S32_TY - 1, &bars[b]);
        if (p.stage > 1) tma_load_2d(dst + 2 * S32_FIELD, &maps.wn, tx * S32_TX, ty * S32_TY, &bars[b]);
    };
    const float dt = (float)p.ctl->dt;
    int k = 0;
    if (threadIdx.x == 0 && (int)blockIdx.x < ntiles) issue(blockIdx.x, 0);
    // one barrier per tile, as in k_stage_tma
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++k) {
        const int b = k & 1;
        const int next = tile + gridDim.x;
        const int tx = tile % tiles_x, ty = tile / tiles_x;
        const int x0 = tx * S32_TX, y0 = ty * S32_TY;
        for (int e = threadIdx.x; e < RC32_N * S32_TY; e += blockDim.x) {   // the tile rows' constants
            const int q = e / S32_TY, r = e % S32_TY;
            srow[b][q][r] = __ldg(&p.rc[(size_t)q * Ny + min(y0 + r, Ny - 1)]);
        }
        const bool ok = __syncthreads_and(mbar_wait_bounded(&bars[b], (k >> 1) & 1));
        if (!ok) {                                       // nothing else is in flight
            if (threadIdx.x == 0) atomicOr(const_cast<int*>(&p.ctl->nonfinite), 2);
            return;
        }
        if (threadIdx.x == 0 && next < ntiles) issue(next, b ^ 1);
        float* sp = reinterpret_cast<float*>(smem_raw + b * S32_BUF);
        float* so = reinterpret_cast<float*>(smem_raw + b * S32_BUF + S32_FIELD);
        if (tx == 0 || tx == tiles_x - 1) {
            // periodic halo columns: box column 3 is x = -1, box column S32_TX + 4 is x = Nx
            for (int r = threadIdx.x; r < S32_H; r += blockDim.x) {
                const int gy = y0 - 1 + r;
                if (gy < 0 || gy >= Ny) continue;
                if (tx == 0) {
                    sp[r * S32_W + 3] = __ldg(&p.psi[(size_t)gy * Nx + Nx - 1]);
                    so[r * S32_W + 3] = __ldg(&p.w_in[(size_t)gy * Nx + Nx - 1]);
                }
                if (tx == tiles_x - 1) {
                    sp[r * S32_W + S32_TX + 4] = __ldg(&p.psi[(size_t)gy * Nx]);
                    so[r * S32_W + S32_TX + 4] = __ldg(&p.w_in[(size_t)gy * Nx]);
                }
            }
            __syncthreads();                             // tx is the same for the whole CTA
        }
        stage32_tile4(p, dt, sp, so, reinterpret_cast<const float*>(smem_raw + b * S32_BUF + 2 * S32_FIELD), x0, y0,
                      srow[b]);
        fence_proxy_async_smem();                        // reads of buffer b before its next TMA write
    }
}

// ---- FP32 row transforms, FP32 spectral buffer ----
struct Fft32Params {
    const float* src;          // forward: rows of w'
    cpx<float>* hat;           // [Ny][Hp], FP32
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
    pdl_begin();
    cpx<float>* buf = reinterpret_cast<cpx<float>*>(smem_raw);
    constexpr int R0 = p16_plan<M>::R(0), NB0 = M / R0;
    const int je = p.Ny - 1;                            // interior rows 1 .. Ny-2, strided over one wave of CTAs
    for (int j = 1 + blockIdx.x; j < je; j += gridDim.x) {
        const float2* row = reinterpret_cast<const float2*>(p.src + (size_t)j * p.Nx);
        // pass 0 from global (radix-16 plan of fft_rows.cuh): thread t transforms t + NB0 r
#pragma unroll 1
        for (int b0 = 0; b0 < NB0; b0 += IP_NT) {
            const int t = b0 + (int)threadIdx.x;
            if (NB0 % IP_NT != 0 && t >= NB0) break;
            cpx<float> v[R0];
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const float2 z = ld_na(row + t + NB0 * r);
                v[r] = {z.x, z.y};
            }
            dftR<float, R0, false>(v);
            const int p0 = dit16_pos<M>(t);
#pragma unroll
            for (int q = 0; q < R0; ++q) buf[ip_idx<M>(p0 + q)] = v[q];
        }
        __syncthreads();
        if constexpr (M == 16 * IP_NT) {                // the fused last pass and split (see k_fft_fwd)
            float2* dst = reinterpret_cast<float2*>(p.hat + (size_t)j * p.Hp);
            p16_pass<float, M, 1, false, IP_NT>(buf, p.tw);
            __syncthreads();
            fwd_last_pass_split<float, M>(buf, p.tw, p.wN, dst);
        } else {
            p16_passes_from<float, M, 1, false, IP_NT>(buf, p.tw);
            // the split step for the pair (k, M - k) (see k_fft_fwd)
            float2* dst = reinterpret_cast<float2*>(p.hat + (size_t)j * p.Hp);
            auto split = [&](int k, const cpx<float>& wk) {             // wk = W^k / 2 (see k_fft_fwd)
                const int kb = (k == 0 ? 0 : M - k);
                const cpx<float> a = buf[ip_idx<M>(k)];
                const cpx<float> b = buf[ip_idx<M>(kb)];
                const cpx<float> sm = {0.5f * (a.x + b.x), 0.5f * (a.y - b.y)};
                const cpx<float> df = {a.x - b.x, a.y + b.y};
                const cpx<float> X = cadd(sm, cmul(wk, mul_mi(df)));
                dst[k] = make_float2(X.x, X.y);
                if (k < M / 2) {
                    const int m = M - k;
                    const cpx<float> wm = {-wk.x, wk.y};                          // W^{M-k} = -conj(W^k)
                    const cpx<float> Y = cadd(cpx<float>{sm.x, -sm.y}, cmul(wm, cpx<float>{df.y, df.x}));
                    dst[m] = make_float2(Y.x, Y.y);
                }
            };
            for (int k = threadIdx.x; k <= M / 2; k += IP_NT) {
                const cpx<float> w1 = ldtw(p.wN, k);
                split(k, cpx<float>{0.5f * w1.x, 0.5f * w1.y});
            }
        }
        __syncthreads();                                // the split reads before the next row's pass 0
    }
}

template <int M>
static __global__ void __launch_bounds__(IP_NT, 5) k_ifft_thom32(Fft32Params p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_begin();
    cpx<float>* buf = reinterpret_cast<cpx<float>*>(smem_raw);
    const int Nx = p.Nx, Ny = p.Ny;
    int j0, j1;
    band_of(blockIdx.x, gridDim.x, p.rows_per_cta, Ny, j0, j1);
    constexpr float scale = 0.5f / (float)M;            // the merge forms 2 Z_n (see k_ifft_thom)
    constexpr int R0 = p16_plan<M>::R(0), NB0 = M / R0;
    constexpr bool kPairLanes = (NB0 == IP_NT) && (R0 == 16) && (IP_NT == 128);   // M = 2048
    for (int j = j0; j < j1; ++j) {
        float* dst = p.psi + (size_t)j * Nx;
        if (j == 0 || j == Ny - 1) {                    // psi' = 0 on the walls
            for (int i = threadIdx.x; i < Nx; i += IP_NT) dst[i] = 0.f;
            continue;
        }
        // pass 0 from global with the merge (see k_ifft_thom)
        const float2* X = reinterpret_cast<const float2*>(p.hat + (size_t)j * p.Hp);
        if constexpr (kPairLanes) {
            // mirror lanes, as in k_ifft_thom: lanes 0..15 of warp w take butterflies 16 w + l,
            // lanes 16..31 the mirrors 128 - b (64 for lane 16 of warp 0); each lane loads its
            // own 16 points and takes the mirror points X_{M-n} by shuffle
            const int w = (int)threadIdx.x >> 5, l = (int)threadIdx.x & 31;
            int b = (l < 16) ? 16 * w + l : 128 - (16 * w + l - 16);
            if (b == 128) b = 64;
            float2 x[16];
#pragma unroll
            for (int r = 0; r < 16; ++r) x[r] = __ldcs(X + b + 128 * r);
            float2 xM = make_float2(0.f, 0.f);
            if (b == 0) xM = __ldcs(X + M);
            const cpx<float> wt = ldtw(p.wN, b);        // W_{2M}^{b + 128 r} = W_{2M}^b e^{-i pi r/16}
            auto merge = [&](const float2& av, const float2& bv, int r) {
                const cpx<float> a = {av.x, av.y}, c = {bv.x, -bv.y};
                const cpx<float> E = {a.x + c.x, a.y + c.y};
                const cpx<float> D = {a.x - c.x, a.y - c.y};
                return cadd(E, mul_pi(cmulc(D, r == 0 ? wt : cmul(wt, w32<float>(r)))));
            };
            cpx<float> v[16];
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int r2 = 15 - r;
                float2 ma, mb;                           // the mirrors of the points r and 15 - r
                ma.x = __shfl_xor_sync(0xffffffffu, x[r2].x, 16);
                ma.y = __shfl_xor_sync(0xffffffffu, x[r2].y, 16);
                mb.x = __shfl_xor_sync(0xffffffffu, x[r].x, 16);
                mb.y = __shfl_xor_sync(0xffffffffu, x[r].y, 16);
                if (b == 64) { ma = x[r2]; mb = x[r]; }
                if (b == 0) { ma = (r == 0) ? xM : x[16 - r]; mb = x[r + 1]; }
                v[r] = merge(x[r], ma, r);
                v[r2] = merge(x[r2], mb, r2);
            }
            dftR<float, 16, true>(v);
            const int p0 = dit16_pos<M>(b);
#pragma unroll
            for (int q = 0; q < 16; ++q) buf[ip_idx<M>(p0 + q)] = v[q];
        } else {
#pragma unroll 1
            for (int b0 = 0; b0 < NB0; b0 += IP_NT) {
                const int t = b0 + (int)threadIdx.x;
                if (NB0 % IP_NT != 0 && t >= NB0) break;
                cpx<float> v[R0];
#pragma unroll
                for (int r = 0; r < R0; ++r) {
                    const int n = t + NB0 * r;
                    const float2 av = __ldcs(X + n), bv = __ldcs(X + (M - n));
                    const cpx<float> a = {av.x, av.y}, b = {bv.x, -bv.y};
                    const cpx<float> E = {a.x + b.x, a.y + b.y};
                    const cpx<float> D = {a.x - b.x, a.y - b.y};
                    v[r] = cadd(E, mul_pi(cmulc(D, ldtw(p.wN, n))));
                }
                dftR<float, R0, true>(v);
                const int p0 = dit16_pos<M>(t);
#pragma unroll
                for (int q = 0; q < R0; ++q) buf[ip_idx<M>(p0 + q)] = v[q];
            }
        }
        __syncthreads();
        if constexpr (p16_plan<M>::P >= 2) {
            // the last pass stores z_n straight from registers (see k_ifft_thom)
            p16_passes_to<float, M, 1, true, IP_NT>(buf, p.tw, [&](int n, const cpx<float>& z) {
                reinterpret_cast<float2*>(dst)[n] = make_float2(z.x * scale, z.y * scale);
            });
        } else {
            p16_passes_from<float, M, 1, true, IP_NT>(buf, p.tw);
            for (int n = threadIdx.x; n < M; n += IP_NT) {
                const cpx<float> z = buf[ip_idx<M>(n)];
                reinterpret_cast<float2*>(dst)[n] = make_float2(z.x * scale, z.y * scale);
            }
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
            // the loads of 8 columns per thread in flight before any store (one CTA writes the row)
            for (int i0 = threadIdx.x; i0 < Nx; i0 += 8 * IP_NT) {
                float a1[8], a2[8];
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const int i = i0 + c * IP_NT;
                    if (i < Nx) { a1[c] = __ldcg(&r1[i]); a2[c] = __ldcg(&r2[i]); }
                }
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const int i = i0 + c * IP_NT;
                    if (i < Nx) wr[i] = p.free_slip ? base : base - (A * a1[c] + B * a2[c]);
                }
            }
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
// The item layout of k_maxuv_dt with 4 columns per lane (one 16-byte load per row; Nx is a
// power of two >= 4): lanes 1..30 own a warp's 120 columns, lanes 0 and 31 hold their outer
// neighbours, and the next four rows are in flight while the current ones are reduced.
struct Max32Params {
    MaxParams base;          // a_node, control block, dt constants, items (base.psi unused)
    const float* psi;        // psi'
    const float* dpsibar;    // [Ny]: psibar_{j+1} - psibar_{j-1} (the RC_DPB row constant)
};
constexpr int MX32_WCOLS = 120, MX32_COLS = 8 * MX32_WCOLS;

static __global__ void __launch_bounds__(256, 3) k_maxuv32(Max32Params q) {
    pdl_begin();
    const MaxParams& p = q.base;
    const int Nx = p.Nx, Ny = p.Ny;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double um = 0.0, vm = 0.0, vmm = 0.0;
    float probe = 0.f;
    const double cy = 0.5 * p.inv_deta, cx = 0.5 * p.inv_dx;
    const int nitems = p.nstrips * p.nbands;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int strip = item % p.nstrips, band = item / p.nstrips;
        const int c = strip * MX32_COLS + warp * MX32_WCOLS + 4 * (lane - 1);
        const bool own = lane >= 1 && lane <= 30 && c < Nx;
        const int ca = ((c % Nx) + Nx) % Nx;
        const int j0 = 1 + band * p.band_rows, j1 = min(Ny - 1, j0 + p.band_rows);
        auto row = [&](const float4& wm, const float4& wc, const float4& wp, double a, float d) {
            const float xl = __shfl_up_sync(0xffffffffu, wc.w, 1);
            const float xr = __shfl_down_sync(0xffffffffu, wc.x, 1);
            if (own) {
                const float e0 = (wp.x - wm.x) + d, e1 = (wp.y - wm.y) + d;
                const float e2 = (wp.z - wm.z) + d, e3 = (wp.w - wm.w) + d;
                const float f0 = wc.y - xl, f1 = wc.z - wc.x, f2 = wc.w - wc.y, f3 = xr - wc.z;
                const float dym = fmaxf(fmaxf(fabsf(e0), fabsf(e1)), fmaxf(fabsf(e2), fabsf(e3)));
                const float dxm = fmaxf(fmaxf(fabsf(f0), fabsf(f1)), fmaxf(fabsf(f2), fabsf(f3)));
                probe += ((e0 + e1) + (e2 + e3)) + ((f0 + f1) + (f2 + f3));
                const double av = (double)dxm * cx;
                um = nn_max(um, a * ((double)dym * cy));
                vm = nn_max(vm, av);
                vmm = nn_max(vmm, av * a);
            }
        };
        const size_t nx1 = (size_t)Nx;
        const float* rp = q.psi + (size_t)(j0 - 1) * Nx + ca;
        float4 wm = __ldg(reinterpret_cast<const float4*>(rp));
        float4 wc = __ldg(reinterpret_cast<const float4*>(rp + nx1));
        rp += 2 * nx1;
        int j = j0;
        float4 n0, n1, n2, n3;
        auto load4 = [&](const float* r) {
            n0 = __ldg(reinterpret_cast<const float4*>(r));
            n1 = __ldg(reinterpret_cast<const float4*>(r + nx1));
            n2 = __ldg(reinterpret_cast<const float4*>(r + 2 * nx1));
            n3 = __ldg(reinterpret_cast<const float4*>(r + 3 * nx1));
        };
        if (j + 4 <= j1) load4(rp);
        for (; j + 4 <= j1; j += 4) {
            const float4 c0 = n0, c1 = n1, c2 = n2, c3 = n3;
            const double a0 = __ldg(&p.a_node[j]), a1 = __ldg(&p.a_node[j + 1]);
            const double a2 = __ldg(&p.a_node[j + 2]), a3 = __ldg(&p.a_node[j + 3]);
            const float d0 = __ldg(&q.dpsibar[j]), d1 = __ldg(&q.dpsibar[j + 1]);
            const float d2 = __ldg(&q.dpsibar[j + 2]), d3 = __ldg(&q.dpsibar[j + 3]);
            rp += 4 * nx1;
            if (j + 8 <= j1) load4(rp);
            row(wm, wc, c0, a0, d0);
            row(wc, c0, c1, a1, d1);
            row(c0, c1, c2, a2, d2);
            row(c1, c2, c3, a3, d3);
            wm = c2; wc = c3;
        }
        for (; j < j1; ++j) {
            const float4 c0 = __ldg(reinterpret_cast<const float4*>(rp));
            rp += nx1;
            row(wm, wc, c0, __ldg(&p.a_node[j]), __ldg(&q.dpsibar[j]));
            wm = wc; wc = c0;
        }
    }
    const int nonfinite = !(probe - probe == 0.f) || !(um <= 1e300) || !(vm <= 1e300);
    maxuv_finish(p, um, vm, vmm, nonfinite);
}

}  // namespace nse2d
