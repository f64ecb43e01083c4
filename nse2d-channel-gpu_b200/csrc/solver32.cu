// Host side of the FP32-bulk variant (precision 32): buffers, the split of the FP64 initial
// state into FP64 base profiles and FP32 fluctuations, the export back to FP64 fields, and the
// enqueueing of one step. The kernels and the reasoning are in bulk32.cuh. Written for this
// project.
#include <algorithm>
#include <cmath>
#include <vector>

#include "nse2d_internal.h"
#include "bulk32.cuh"

namespace nse2d {

template <typename T> static int alloc(T** p, size_t n) {
    NSE_CUDA_TRY(cudaMalloc((void**)p, n * sizeof(T) + 16));
    NSE_CUDA_TRY(cudaMemset(*p, 0, n * sizeof(T) + 16));
    return 0;
}

int setup32(Context* c) {
    const size_t N = c->N;
    if (alloc(&c->wf, N) || alloc(&c->w1f, N) || alloc(&c->w2f, N) || alloc(&c->psif, N) || alloc(&c->rhsf, N) ||
        alloc(&c->wbar, (size_t)c->Ny) || alloc(&c->psibar, (size_t)c->Ny) || alloc(&c->rc32, (size_t)RC32_N * c->Ny) ||
        alloc(&c->hat32, (size_t)c->Ny * c->Hp))
        return -1;
    // FP32 twiddles: the FP64 values rounded, in the same per-pass layout
    const long double PI = 3.141592653589793238462643383279502884L;
    const int M = c->M;
    std::vector<cpx<float>> full(M), wN(M + 1), tw;
    for (int t = 0; t < M; ++t) {
        const long double a = -2.0L * PI * (long double)t / (long double)M;
        full[t] = {(float)cosl(a), (float)sinl(a)};
    }
    for (int k = 0; k <= M; ++k) {
        const long double a = -PI * (long double)k / (long double)M;
        wN[k] = {(float)cosl(a), (float)sinl(a)};
    }
    full[0] = {1.f, 0.f};
    if (M % 4 == 0) { full[M / 4] = {0.f, -1.f}; full[M / 2] = {-1.f, 0.f}; full[3 * M / 4] = {0.f, 1.f}; }
    wN[0] = {1.f, 0.f};
    wN[M] = {-1.f, 0.f};
    if (M % 2 == 0) wN[M / 2] = {0.f, -1.f};
    p16_twiddle_table(M, full.data(), tw);
    if (alloc(&c->twf, tw.size()) || alloc(&c->wNf, wN.size())) return -1;
    NSE_CUDA_TRY(cudaMemcpy(c->twf, tw.data(), tw.size() * sizeof(tw[0]), cudaMemcpyHostToDevice));
    NSE_CUDA_TRY(cudaMemcpy(c->wNf, wN.data(), wN.size() * sizeof(wN[0]), cudaMemcpyHostToDevice));
    int per_sm = 0;
    NSE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_maxuv32, 256, 0));
    c->maxuv32_ctas = std::max(per_sm, 1) * c->num_sms;
    // stage kernel: the persistent TMA form when every tile row holds two or more tiles
    c->stage32_tma = c->stage32_tma_ok = (c->Nx >= 2 * S32_TX);
    if (c->stage32_tma) {
        const int Nx = c->Nx, Ny = c->Ny;
        if (encode_map_2d(&c->tm32_psi, c->psif, true, Nx, Ny, S32_W, S32_H) ||
            encode_map_2d(&c->tm32_w[0], c->wf, true, Nx, Ny, S32_W, S32_H) ||
            encode_map_2d(&c->tm32_w[1], c->w1f, true, Nx, Ny, S32_W, S32_H) ||
            encode_map_2d(&c->tm32_w[2], c->w2f, true, Nx, Ny, S32_W, S32_H) ||
            encode_map_2d(&c->tm32_wn, c->wf, true, Nx, Ny, S32_TX, S32_TY))
            return -1;
        int per = 0;
        NSE_CUDA_TRY(cudaFuncSetAttribute(k_stage32_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)stage32_tma_smem_bytes()));
        NSE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_stage32_tma, 256, stage32_tma_smem_bytes()));
        if (per < 1) {
            set_error("k_stage32_tma cannot be resident");
            return -1;
        }
        const int ntiles = (Nx / S32_TX) * ((Ny + S32_TY - 1) / S32_TY);
        c->stage32_tma_grid = std::min(ntiles, per * c->num_sms);
    }
    return 0;
}

void destroy32(Context* c) {
    for (void* p : {(void*)c->wf, (void*)c->w1f, (void*)c->w2f, (void*)c->psif, (void*)c->rhsf, (void*)c->wbar,
                    (void*)c->psibar, (void*)c->rc32, (void*)c->twf, (void*)c->wNf, (void*)c->hat32})
        if (p) cudaFree(p);
}

// FP64 w, psi of the context -> base profiles, fluctuations, row constants, wall constants.
int split32(Context* c, cudaStream_t s) {
    const int Ny = c->Ny;
    k_split32<<<std::min(Ny, 8 * c->num_sms), 256, 0, s>>>(c->w, c->psi, c->Nx, Ny, c->wbar, c->psibar, c->wf, c->psif);
    NSE_CUDA_TRY(cudaGetLastError());
    k_rowconst32<<<(Ny + 127) / 128, 128, 0, s>>>(c->rt, c->wbar, c->psibar, Ny, 0.25 * c->inv_dx * c->inv_deta, c->nu,
                                                 c->inv_deta2, c->cfg.lin_drag, c->rc32);
    NSE_CUDA_TRY(cudaGetLastError());
    std::vector<double> wb(Ny), pb(Ny);
    NSE_CUDA_TRY(cudaMemcpyAsync(wb.data(), c->wbar, Ny * sizeof(double), cudaMemcpyDeviceToHost, s));
    NSE_CUDA_TRY(cudaMemcpyAsync(pb.data(), c->psibar, Ny * sizeof(double), cudaMemcpyDeviceToHost, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    // [Thom(psibar) - wbar] at the walls (src/ops.cu:114-151), or -wbar with free-slip walls
    auto thom = [&](bool top) {
        const double d1 = top ? c->h_dy_edge[Ny - 2] : c->h_dy_edge[0];
        const double d2 = top ? c->h_dy_edge[Ny - 3] : c->h_dy_edge[1];
        const double A = 2.0 * (1.0 / (d1 * d1) + 1.0 / (d1 * d2));
        const double B = (-2.0) * d1 / (d2 * (d1 + d2) * (d1 + d2));
        const double pw = top ? c->psi_top : c->psi_bot;
        const double p1 = top ? pb[Ny - 2] : pb[1], p2 = top ? pb[Ny - 3] : pb[2];
        return -(A * (p1 - pw) + B * (p2 - pw));
    };
    c->wall_bot32 = (c->cfg.free_slip ? 0.0 : thom(false)) - wb[0];
    c->wall_top32 = (c->cfg.free_slip ? 0.0 : thom(true)) - wb[Ny - 1];
    return 0;
}

// The context's FP64 fields from the split state (and the stored stage rhs, with_rhs).
int export32(Context* c, bool with_rhs, cudaStream_t s) {
    const int grid = 8 * c->num_sms;
    k_join32<<<grid, 256, 0, s>>>(c->wbar, c->wf, c->w, c->Nx, c->Ny);
    k_join32<<<grid, 256, 0, s>>>(c->psibar, c->psif, c->psi, c->Nx, c->Ny);
    if (with_rhs) k_widen32<<<grid, 256, 0, s>>>(c->rhsf, c->rhs, c->N);
    NSE_CUDA_TRY(cudaGetLastError());
    return 0;
}

static Fft32Params fft32_params(Context* c) {
    Fft32Params p{};
    p.hat = c->hat32; p.tw = c->twf; p.wN = c->wNf; p.dy_edge = c->rt.dy_edge; p.ctl = c->ctl;
    p.Nx = c->Nx; p.Ny = c->Ny; p.Hp = c->Hp; p.free_slip = c->cfg.free_slip;
    p.wall_bot = c->wall_bot32; p.wall_top = c->wall_top32;
    return p;
}

template <int M> static int fft32_fwd_t(Context* c, Fft32Params& p, cudaStream_t s) {
    const size_t sm = fft32_smem_bytes(M);
    NSE_CUDA_TRY(cudaFuncSetAttribute(k_fft_fwd32<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per_sm = 0;                                      // one wave of CTAs over the interior rows
    NSE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fft_fwd32<M>, IP_NT, sm));
    const int grid = std::max(1, std::min(c->Ni, std::max(per_sm, 1) * c->num_sms));
    return launch_step_kernel(c, k_fft_fwd32<M>, dim3(grid), dim3(IP_NT), sm, s, nullptr, p);
}
template <int M> static int fft32_inv_t(Context* c, Fft32Params& p, cudaStream_t s) {
    const size_t sm = fft32_smem_bytes(M);
    NSE_CUDA_TRY(cudaFuncSetAttribute(k_ifft_thom32<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    p.rows_per_cta = 3;
    return launch_step_kernel(c, k_ifft_thom32<M>, dim3(std::max(1, c->Ny / 3)), dim3(IP_NT), sm, s, nullptr, p);
}

#define NSE_FFT32_DISPATCH(FN)                                                     \
    switch (c->M) {                                                                \
        case 2: return FN<2>(c, p, s);       case 4: return FN<4>(c, p, s);        \
        case 8: return FN<8>(c, p, s);       case 16: return FN<16>(c, p, s);      \
        case 32: return FN<32>(c, p, s);     case 64: return FN<64>(c, p, s);      \
        case 128: return FN<128>(c, p, s);   case 256: return FN<256>(c, p, s);    \
        case 512: return FN<512>(c, p, s);   case 1024: return FN<1024>(c, p, s);  \
        case 2048: return FN<2048>(c, p, s); case 4096: return FN<4096>(c, p, s);  \
        case 8192: return FN<8192>(c, p, s);                                       \
        default: set_error("no FFT kernel for M = %d", c->M); return -1;           \
    }

static int fft32_fwd(Context* c, const float* src, cudaStream_t s) {
    Fft32Params p = fft32_params(c);
    p.src = src;
    NSE_FFT32_DISPATCH(fft32_fwd_t)
}

static int fft32_inv(Context* c, float* w_out, bool advance, cudaStream_t s) {
    Fft32Params p = fft32_params(c);
    p.psi = c->psif;
    p.w = w_out;
    p.do_thom = 1;
    p.advance = advance ? 1 : 0;
    NSE_FFT32_DISPATCH(fft32_inv_t)
}

int step32_impl(Context* c, cudaStream_t s, bool store_rhs, cudaEvent_t* ev) {
    int k = 0;
    auto mark = [&]() -> int {
        if (ev) NSE_CUDA_TRY(cudaEventRecord(ev[k++], s));
        return 0;
    };
    if (mark()) return -1;
    if (c->cfg.adapt) {
        Max32Params q{};
        MaxParams& p = q.base;
        p.a_node = c->rt.a_node; p.ctl = c->ctl;
        p.Nx = c->Nx; p.Ny = c->Ny; p.adapt = 1; p.set_dt = 1;
        p.inv_dx = c->inv_dx; p.inv_deta = c->inv_deta; p.cfl = c->cfg.cfl; p.cvisc = c->cfg.cvisc;
        p.dx = c->dx; p.deta = c->deta; p.nu = c->nu; p.inv_dx2 = c->inv_dx2; p.inv_dymin2 = c->inv_dymin2;
        p.dt_max = c->cfg.dt_max;
        q.psi = c->psif;
        q.dpsibar = c->rc32 + (size_t)RC_DPB * c->Ny;
        int grid = 1;
        maxuv_plan(p, c->maxuv32_ctas, c->maxuv32_ctas, grid, MX32_COLS);
        if (launch_step_kernel(c, k_maxuv32, dim3(grid), dim3(256), 0, s, nullptr, q) || mark()) return -1;
    }
    float* wst[3] = {c->w1f, c->w2f, c->wf};
    const float* win[3] = {c->wf, c->w1f, c->w2f};
    const dim3 grid((c->Nx + ST_TX - 1) / ST_TX, (c->Ny + ST_TY - 1) / ST_TY);
    for (int st = 1; st <= 3; ++st) {
        Stage32Params sp{};
        sp.psi = c->psif; sp.w_in = win[st - 1]; sp.w_n = c->wf; sp.w_out = wst[st - 1];
        sp.rhs_out = (store_rhs && st == 3) ? c->rhsf : nullptr;
        sp.rc = c->rc32; sp.ctl = c->ctl; sp.Nx = c->Nx; sp.Ny = c->Ny; sp.stage = st;
        sp.nu_dx2 = (float)(c->nu * c->inv_dx2); sp.lin_drag = (float)c->cfg.lin_drag;
        if (c->stage32_tma) {
            Stage32Maps maps;
            maps.psi = c->tm32_psi;
            maps.w = c->tm32_w[st - 1];          // w'^(s): wf, w1f, w2f in stages 1, 2, 3
            maps.wn = c->tm32_wn;
            if (launch_step_kernel(c, k_stage32_tma, dim3(c->stage32_tma_grid), dim3(256), stage32_tma_smem_bytes(), s,
                                   nullptr, maps, sp))
                return -1;
        } else {
            if (launch_step_kernel(c, k_stage32, grid, dim3(256), 0, s, nullptr, sp)) return -1;
        }
        if (mark()) return -1;
        if (fft32_fwd(c, wst[st - 1], s) || mark()) return -1;
        for (int i = 0; i < thomas_launches(c); ++i)
            if (launch_thomas_part(c, i, s, true) || mark()) return -1;
        if (fft32_inv(c, wst[st - 1], st == 3, s) || mark()) return -1;
    }
    return 0;
}

const char* step32_kernel_name(const Context* c, int k) {
    if (c->cfg.adapt) {
        if (k == 0) return "k_maxuv32";
        --k;
    }
    const int per = 3 + thomas_launches(c);
    if (k < 0 || k >= 3 * per) return "";
    const int i = k % per;
    if (i == 0) return c->stage32_tma ? "k_stage32_tma" : "k_stage32";
    if (i == 1) return "k_fft_fwd32";
    if (i == per - 1) return "k_ifft_thom32";
    return thomas_kernel_name(c, i - 2);
}

}  // namespace nse2d
