// The learned subgrid closure: a small CNN whose 3x3 convolutions run as BF16 GEMMs on the
// tensor cores (tcgen05, FP32 accumulate), its backward pass, AdamW, and the coarse-grid data
// generator (box filter). Written for this project; the reference has no closure model.
//
// Model. Input: the coarse fields omega and psi, scaled by fixed factors, 2 channels. Three
// 3x3 convolutions 2 -> H -> H -> 1 (ReLU after the first two), periodic in x and zero-padded
// beyond the walls. Output: tau / tau_scale, the subgrid term of the Jacobian,
//   tau = filter(J(psi, omega)) - J(filter psi, filter omega),
// which the coarse solver subtracts from its rhs on interior rows.
//
// Layout. A pixel p = j Nx + i; activations are BF16 [P_pad][C] (channels contiguous), P_pad a
// multiple of 128. A convolution is im2col (A[p][k], k = tap C + c, tap = 3 (dy + 1) + dx + 1,
// K padded to a multiple of 64) and the GEMM Z = A . W^T + b with W [N_pad][K] (N_pad a
// multiple of 16); the GEMM's epilogue writes Z (FP32, kept for the backward pass) and
// ReLU(Z) in BF16, the next layer's input.
//
// Backward (loss = mean over interior pixels of (z - tau/tau_scale)^2):
//   dW[n][k] = sum_p dZ[p][n] A[p][k] and db[n] = sum_p dZ[p][n] on the CUDA cores (per-block
//   partials folded in a fixed order, so the gradients do not depend on scheduling);
//   dA = dZ . W on the tensor cores (dZ in BF16, padded to 64 channels; W^T kept in BF16);
//   col2im gathers dA back to the pixels of the layer input and applies ReLU'.
// AdamW updates FP32 master weights and re-exports the BF16 W and W^T.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "nse2d_internal.h"
#include "tc_gemm.cuh"
#include "../../include/nse2d.h"

namespace nse2d {

__device__ int g_tc_err;                  // error flag of the tensor-core GEMM's bounded waits

namespace {

constexpr int CN_LAYERS = 3;
constexpr int CN_CIN = 2;
constexpr int CN_KD = 64;                 // reduction width of the input-gradient GEMM (channels padded)
constexpr int CN_WG_PB = 64;              // pixels per block of the weight-gradient reduction
constexpr int CN_NT = 256;

int round_up(int x, int m) { return (x + m - 1) / m * m; }

}  // namespace

struct Cnn {
    int Nx = 0, Ny = 0, P = 0, Ppad = 0, hidden = 0, Pint = 0;
    int cin[CN_LAYERS], cout[CN_LAYERS], npad[CN_LAYERS], K[CN_LAYERS];
    float* w32[CN_LAYERS] = {};           // [npad][K] master weights (padding stays zero)
    float* b32[CN_LAYERS] = {};           // [npad]
    float* gw[CN_LAYERS] = {};
    float* gb[CN_LAYERS] = {};
    float* mw[CN_LAYERS] = {};
    float* vw[CN_LAYERS] = {};
    float* mb[CN_LAYERS] = {};
    float* vb[CN_LAYERS] = {};
    __nv_bfloat16* wbf[CN_LAYERS] = {};   // [npad][K]
    __nv_bfloat16* wtbf[CN_LAYERS] = {};  // [K][64]: W^T, channels padded with zeros
    __nv_bfloat16* h[CN_LAYERS] = {};     // layer input: h[0] [Ppad][2], h[l] [Ppad][npad[l-1]]
    __nv_bfloat16* A = nullptr;           // im2col of the current layer [Ppad][Kmax]
    float* z[CN_LAYERS] = {};             // pre-activations [Ppad][npad]
    float* dz = nullptr;                  // [Ppad][64]
    __nv_bfloat16* dzb = nullptr;         // [Ppad][64]
    float* dA = nullptr;                  // [Ppad][Kmax]
    float* part = nullptr;                // weight-gradient partials [nblk][npad K + npad]
    float* lpart = nullptr;               // loss partials [ceil(Ppad / CN_NT)]
    float* loss = nullptr;                // [1]
    int* err = nullptr;
    double in_w = 1.0, in_psi = 1.0, out_tau = 1.0;
    long long step = 0;
};

int tc_gemm_launch(const TcGemmParams& p0, cudaStream_t s);

namespace {

template <typename T> int cn_alloc(T** p, size_t n) {
    NSE_CUDA_TRY(cudaMalloc((void**)p, n * sizeof(T) + 16));
    NSE_CUDA_TRY(cudaMemset(*p, 0, n * sizeof(T) + 16));
    return 0;
}

__global__ void k_pack_input(const double* w, const double* psi, __nv_bfloat16* h0, int P, int Ppad, double sw, double sp) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= Ppad) return;
    const bool in = p < P;
    h0[2 * p] = __float2bfloat16_rn(in ? (float)(w[p] * sw) : 0.f);
    h0[2 * p + 1] = __float2bfloat16_rn(in ? (float)(psi[p] * sp) : 0.f);
}

// A[p][k] for one 8-wide chunk of k per thread; taps outside the walls read zero, x is periodic.
__global__ void k_im2col(const __nv_bfloat16* h, int C, int Nx, int Ny, int P, int Ppad, int K, __nv_bfloat16* A) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nch = K / 8;
    if (t >= (long long)Ppad * nch) return;
    const int p = (int)(t / nch), k0 = (int)(t % nch) * 8;
    const int j = p / Nx, i = p - j * Nx;
    __align__(16) __nv_bfloat16 v[8];
    if ((C & 7) == 0 && k0 < 9 * C) {                    // the chunk is 8 channels of one tap
        const int tap = k0 / C, c = k0 - tap * C;
        const int jj = j + tap / 3 - 1, ii = i + tap % 3 - 1;
        if (p < P && jj >= 0 && jj < Ny) {
            const int iw = ii < 0 ? ii + Nx : (ii >= Nx ? ii - Nx : ii);
            *reinterpret_cast<uint4*>(v) = *reinterpret_cast<const uint4*>(h + ((size_t)jj * Nx + iw) * C + c);
        } else {
            *reinterpret_cast<uint4*>(v) = make_uint4(0, 0, 0, 0);
        }
    } else {
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int k = k0 + e;
            float x = 0.f;
            if (p < P && k < 9 * C) {
                const int tap = k / C, c = k - tap * C;
                const int jj = j + tap / 3 - 1, ii = i + tap % 3 - 1;
                if (jj >= 0 && jj < Ny) {
                    const int iw = ii < 0 ? ii + Nx : (ii >= Nx ? ii - Nx : ii);
                    x = __bfloat162float(h[((size_t)jj * Nx + iw) * C + c]);
                }
            }
            v[e] = __float2bfloat16_rn(x);
        }
    }
    *reinterpret_cast<uint4*>(A + (size_t)p * K + k0) = *reinterpret_cast<const uint4*>(v);
}

// tau = tau_scale z[p][0] on interior rows, 0 on the walls
__global__ void k_unpack_output(const float* z, int ldz, double* tau, int Nx, int Ny, double ts) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= Nx * Ny) return;
    const int j = p / Nx;
    tau[p] = (j == 0 || j == Ny - 1) ? 0.0 : ts * (double)z[(size_t)p * ldz];
}

// loss partials and dZ of the output layer: d = z - tau / tau_scale on interior pixels
__global__ void __launch_bounds__(CN_NT) k_loss(const float* z, int ldz, const double* tau, double inv_ts, int Nx, int Ny,
                                                int Ppad, float inv_pint, float* dz, __nv_bfloat16* dzb, float* lpart) {
    __shared__ float red[CN_NT];
    const int p = blockIdx.x * CN_NT + threadIdx.x;
    float l = 0.f;
    if (p < Ppad) {
        float g = 0.f;
        const int j = p / Nx;
        if (p < Nx * Ny && j != 0 && j != Ny - 1) {
            const float d = z[(size_t)p * ldz] - (float)(tau[p] * inv_ts);
            l = d * d;
            g = 2.f * d * inv_pint;
        }
        for (int c = 0; c < CN_KD; ++c) {
            dz[(size_t)p * CN_KD + c] = c == 0 ? g : 0.f;
            dzb[(size_t)p * CN_KD + c] = __float2bfloat16_rn(c == 0 ? g : 0.f);
        }
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int s = CN_NT / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) lpart[blockIdx.x] = red[0];
}

__global__ void k_fold(const float* part, int nblk, int nout, float* out, float scale) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nout) return;
    float s = 0.f;
    for (int b = 0; b < nblk; ++b) s += part[(size_t)b * nout + o];
    out[o] = s * scale;
}

// Per-block partial sums of dW[n][k] = sum_p dz[p][n] A[p][k] (o < npad K) and db[n] (o >= npad K)
// over CN_WG_PB pixels; dz has row stride CN_KD.
__global__ void __launch_bounds__(CN_NT) k_wgrad(const float* dz, const __nv_bfloat16* A, int npad, int K, float* part) {
    extern __shared__ __align__(16) unsigned char wg_smem[];
    float* sdz = reinterpret_cast<float*>(wg_smem);                                  // [PB][npad]
    __nv_bfloat16* sA = reinterpret_cast<__nv_bfloat16*>(sdz + CN_WG_PB * npad);      // [PB][K]
    const int p0 = blockIdx.x * CN_WG_PB;
    for (int e = threadIdx.x; e < CN_WG_PB * npad; e += CN_NT) {
        const int r = e / npad, n = e - r * npad;
        sdz[e] = dz[(size_t)(p0 + r) * CN_KD + n];
    }
    for (int e = threadIdx.x; e < CN_WG_PB * K / 8; e += CN_NT) {
        const int r = e / (K / 8), c = e - r * (K / 8);
        reinterpret_cast<uint4*>(sA)[e] = reinterpret_cast<const uint4*>(A + (size_t)(p0 + r) * K)[c];
    }
    __syncthreads();
    const int nout = npad * K + npad;
    float* out = part + (size_t)blockIdx.x * nout;
    for (int o = threadIdx.x; o < nout; o += CN_NT) {
        float s = 0.f;
        if (o < npad * K) {
            const int n = o / K, k = o - n * K;
            for (int r = 0; r < CN_WG_PB; ++r) s = fmaf(sdz[r * npad + n], __bfloat162float(sA[r * K + k]), s);
        } else {
            const int n = o - npad * K;
            for (int r = 0; r < CN_WG_PB; ++r) s += sdz[r * npad + n];
        }
        out[o] = s;
    }
}

// dh[q][c] = sum over taps of dA[q - tap offset][tap C + c] (source rows inside the walls), then
// ReLU' of the layer below: dz[q][c] = dh (z_prev > 0); channels >= C written as zero.
__global__ void k_col2im_relu(const float* dA, int K, int C, const float* zprev, int ldzp, int Nx, int Ny, int Ppad,
                              float* dz, __nv_bfloat16* dzb) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)Ppad * CN_KD) return;
    const int q = (int)(t / CN_KD), c = (int)(t % CN_KD);
    float g = 0.f;
    if (q < Nx * Ny && c < C) {
        const int j = q / Nx, i = q - j * Nx;
        float s = 0.f;
#pragma unroll
        for (int tap = 0; tap < 9; ++tap) {
            const int dy = tap / 3 - 1, dx = tap % 3 - 1;
            const int jp = j - dy;
            if (jp < 0 || jp >= Ny) continue;
            int ip = i - dx;
            ip = ip < 0 ? ip + Nx : (ip >= Nx ? ip - Nx : ip);
            s += dA[((size_t)jp * Nx + ip) * K + tap * C + c];
        }
        g = zprev[(size_t)q * ldzp + c] > 0.f ? s : 0.f;
    }
    dz[t] = g;
    dzb[t] = __float2bfloat16_rn(g);
}

__global__ void k_adamw(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                        float wd, float bc1, float bc2) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const float gg = g[e];
    const float mm = b1 * m[e] + (1.f - b1) * gg;
    const float vv = b2 * v[e] + (1.f - b2) * gg * gg;
    m[e] = mm;
    v[e] = vv;
    const float mh = mm / bc1, vh = vv / bc2;
    w[e] -= lr * (mh / (sqrtf(vh) + eps) + wd * w[e]);
}

__global__ void k_export_w(const float* w, int npad, int K, __nv_bfloat16* wbf, __nv_bfloat16* wtbf) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= K * CN_KD) return;
    const int k = e / CN_KD, n = e - k * CN_KD;
    if (n < npad) {
        const __nv_bfloat16 b = __float2bfloat16_rn(w[(size_t)n * K + k]);
        wbf[(size_t)n * K + k] = b;
        wtbf[e] = b;
    } else {
        wtbf[e] = __float2bfloat16_rn(0.f);
    }
}

// Top-hat filter of a fine field onto a coarse grid whose nodes are every rx-th column and
// ry-th row of the fine one: the mean over fine columns rx i + d and rows ry j + e, |d| <= rx/2,
// |e| <= ry/2, with half weight at |d| = rx/2 and |e| = ry/2; periodic in x; rows beyond the
// walls are left out and the weights renormalised.
__global__ void k_box_filter(const double* f, int Nxf, int Nyf, double* c, int Nxc, int Nyc) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= Nxc * Nyc) return;
    const int j = p / Nxc, i = p - j * Nxc;
    const int rx = Nxf / Nxc, ry = (Nyf - 1) / (Nyc - 1);
    const int hx = rx / 2, hy = ry / 2;
    double s = 0.0, ws = 0.0;
    for (int e = -hy; e <= hy; ++e) {
        const int jf = ry * j + e;
        if (jf < 0 || jf >= Nyf) continue;
        const double we = (hy > 0 && (e == -hy || e == hy)) ? 0.5 : 1.0;
        for (int d = -hx; d <= hx; ++d) {
            int ifn = rx * i + d;
            ifn = ((ifn % Nxf) + Nxf) % Nxf;
            const double wd = (hx > 0 && (d == -hx || d == hx)) ? 0.5 : 1.0;
            s += we * wd * f[(size_t)jf * Nxf + ifn];
            ws += we * wd;
        }
    }
    c[p] = s / ws;
}

int grid_of(long long n, int nt = CN_NT) { return (int)((n + nt - 1) / nt); }

int gemm(Cnn* n, const __nv_bfloat16* A, const __nv_bfloat16* B, const float* bias, float* Cf, __nv_bfloat16* Cb, int M,
         int N, int K, int ldc, int relu, cudaStream_t s) {
    TcGemmParams p{};
    p.A = A; p.B = B; p.bias = bias; p.Cf = Cf; p.Cb = Cb; p.err = n ? n->err : nullptr;
    p.M = M; p.N = N; p.K = K; p.ldc = ldc; p.relu = relu;
    return tc_gemm_launch(p, s);
}

int export_layer(Cnn* n, int l, cudaStream_t s) {
    k_export_w<<<grid_of((long long)n->K[l] * CN_KD), CN_NT, 0, s>>>(n->w32[l], n->npad[l], n->K[l], n->wbf[l], n->wtbf[l]);
    NSE_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace

// ---- shared with the solver and the ABI ----

int tc_gemm_launch(const TcGemmParams& p0, cudaStream_t s) {
    TcGemmParams p = p0;
    if (p.M <= 0 || p.M % TG_BM != 0 || p.N < 16 || p.N > 256 || p.N % 16 != 0 || p.K < TG_BK || p.K % TG_BK != 0 ||
        p.ldc < p.N) {
        set_error("tensor-core GEMM: M = %d (multiple of 128), N = %d (16..256, multiple of 16), K = %d (multiple of 64), "
                  "ldc = %d (>= N)", p.M, p.N, p.K, p.ldc);
        return -1;
    }
    if ((reinterpret_cast<uintptr_t>(p.A) | reinterpret_cast<uintptr_t>(p.B)) % 16 != 0) {
        set_error("tensor-core GEMM: A and B must be 16-byte aligned");
        return -1;
    }
    if (!p.err) {
        void* e = nullptr;
        NSE_CUDA_TRY(cudaGetSymbolAddress(&e, g_tc_err));
        p.err = static_cast<int*>(e);
    }
    k_tc_gemm<<<p.M / TG_BM, TG_THREADS, tg_smem_bytes(p.N), s>>>(p);
    NSE_CUDA_TRY(cudaGetLastError());
    return 0;
}

int tc_gemm_setup() {
    NSE_CUDA_TRY(cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tg_smem_bytes(256)));
    return 0;
}

// Forward pass from (w, psi) on the coarse grid; with tau != null also writes tau (FP64).
int cnn_forward(Cnn* n, const double* w, const double* psi, double* tau, cudaStream_t s) {
    k_pack_input<<<grid_of(n->Ppad), CN_NT, 0, s>>>(w, psi, n->h[0], n->P, n->Ppad, 1.0 / n->in_w, 1.0 / n->in_psi);
    NSE_CUDA_TRY(cudaGetLastError());
    for (int l = 0; l < CN_LAYERS; ++l) {
        k_im2col<<<grid_of((long long)n->Ppad * (n->K[l] / 8)), CN_NT, 0, s>>>(n->h[l], n->cin[l], n->Nx, n->Ny, n->P, n->Ppad,
                                                                              n->K[l], n->A);
        NSE_CUDA_TRY(cudaGetLastError());
        const bool last = (l == CN_LAYERS - 1);
        if (gemm(n, n->A, n->wbf[l], n->b32[l], n->z[l], last ? nullptr : n->h[l + 1], n->Ppad, n->npad[l], n->K[l],
                 n->npad[l], 1, s))
            return -1;
    }
    if (tau) {
        k_unpack_output<<<grid_of(n->P), CN_NT, 0, s>>>(n->z[CN_LAYERS - 1], n->npad[CN_LAYERS - 1], tau, n->Nx, n->Ny,
                                                        n->out_tau);
        NSE_CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

// Loss against tau_target (FP64 [Ny][Nx]) and the gradients of every layer (after cnn_forward).
int cnn_backward(Cnn* n, const double* tau_target, cudaStream_t s) {
    const int nlb = (n->Ppad + CN_NT - 1) / CN_NT;
    k_loss<<<nlb, CN_NT, 0, s>>>(n->z[CN_LAYERS - 1], n->npad[CN_LAYERS - 1], tau_target, 1.0 / n->out_tau, n->Nx, n->Ny,
                                 n->Ppad, 1.f / (float)n->Pint, n->dz, n->dzb, n->lpart);
    NSE_CUDA_TRY(cudaGetLastError());
    k_fold<<<1, 32, 0, s>>>(n->lpart, nlb, 1, n->loss, 1.f / (float)n->Pint);
    NSE_CUDA_TRY(cudaGetLastError());
    for (int l = CN_LAYERS - 1; l >= 0; --l) {
        // the layer's im2col again (only one A buffer is kept)
        k_im2col<<<grid_of((long long)n->Ppad * (n->K[l] / 8)), CN_NT, 0, s>>>(n->h[l], n->cin[l], n->Nx, n->Ny, n->P, n->Ppad,
                                                                              n->K[l], n->A);
        NSE_CUDA_TRY(cudaGetLastError());
        const int nblk = n->Ppad / CN_WG_PB, nout = n->npad[l] * n->K[l] + n->npad[l];
        const size_t sm = (size_t)CN_WG_PB * n->npad[l] * 4 + (size_t)CN_WG_PB * n->K[l] * 2;
        k_wgrad<<<nblk, CN_NT, sm, s>>>(n->dz, n->A, n->npad[l], n->K[l], n->part);
        NSE_CUDA_TRY(cudaGetLastError());
        // fold: weights then biases (the partial layout is [blk][npad K | npad])
        k_fold<<<grid_of(nout), CN_NT, 0, s>>>(n->part, nblk, nout, n->dA, 1.f);
        NSE_CUDA_TRY(cudaGetLastError());
        NSE_CUDA_TRY(cudaMemcpyAsync(n->gw[l], n->dA, sizeof(float) * n->npad[l] * n->K[l], cudaMemcpyDeviceToDevice, s));
        NSE_CUDA_TRY(cudaMemcpyAsync(n->gb[l], n->dA + (size_t)n->npad[l] * n->K[l], sizeof(float) * n->npad[l],
                                     cudaMemcpyDeviceToDevice, s));
        if (l == 0) break;
        // dA = dZ . W: N tiles of at most 256 columns of K
        for (int c0 = 0; c0 < n->K[l]; c0 += 256) {
            const int nc = std::min(256, n->K[l] - c0);
            if (gemm(n, n->dzb, n->wtbf[l] + (size_t)c0 * CN_KD, nullptr, n->dA + c0, nullptr, n->Ppad, nc, CN_KD, n->K[l], 0, s))
                return -1;
        }
        k_col2im_relu<<<grid_of((long long)n->Ppad * CN_KD), CN_NT, 0, s>>>(n->dA, n->K[l], n->cin[l], n->z[l - 1],
                                                                             n->npad[l - 1], n->Nx, n->Ny, n->Ppad, n->dz, n->dzb);
        NSE_CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

int cnn_adamw(Cnn* n, float lr, float wd, cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    n->step += 1;
    const float bc1 = 1.f - powf(b1, (float)n->step), bc2 = 1.f - powf(b2, (float)n->step);
    for (int l = 0; l < CN_LAYERS; ++l) {
        const int nw = n->npad[l] * n->K[l];
        k_adamw<<<grid_of(nw), CN_NT, 0, s>>>(n->w32[l], n->gw[l], n->mw[l], n->vw[l], nw, lr, b1, b2, eps, wd, bc1, bc2);
        k_adamw<<<1, CN_NT, 0, s>>>(n->b32[l], n->gb[l], n->mb[l], n->vb[l], n->npad[l], lr, b1, b2, eps, 0.f, bc1, bc2);
        NSE_CUDA_TRY(cudaGetLastError());
        if (export_layer(n, l, s)) return -1;
    }
    return 0;
}

bool cnn_matches(const Cnn* n, int Nx, int Ny) { return n && n->Nx == Nx && n->Ny == Ny; }

void cnn_free(Cnn* n) {
    if (!n) return;
    for (int l = 0; l < CN_LAYERS; ++l) {
        cudaFree(n->w32[l]); cudaFree(n->b32[l]); cudaFree(n->gw[l]); cudaFree(n->gb[l]);
        cudaFree(n->mw[l]); cudaFree(n->vw[l]); cudaFree(n->mb[l]); cudaFree(n->vb[l]);
        cudaFree(n->wbf[l]); cudaFree(n->wtbf[l]); cudaFree(n->h[l]); cudaFree(n->z[l]);
    }
    cudaFree(n->A); cudaFree(n->dz); cudaFree(n->dzb); cudaFree(n->dA); cudaFree(n->part); cudaFree(n->lpart);
    cudaFree(n->loss); cudaFree(n->err);
    delete n;
}

int cnn_create(int Nx, int Ny, int hidden, Cnn** out) {
    *out = nullptr;
    if (Nx < 4 || Ny < 5 || hidden < 16 || hidden > 64 || hidden % 16 != 0) {
        set_error("nse2d_cnn_create: Nx >= 4, Ny >= 5, hidden a multiple of 16 in [16, 64]");
        return -1;
    }
    if (tc_gemm_setup()) return -1;
    Cnn* n = new Cnn();
    n->Nx = Nx; n->Ny = Ny; n->P = Nx * Ny; n->Ppad = round_up(n->P, 128); n->hidden = hidden; n->Pint = Nx * (Ny - 2);
    const int ch[CN_LAYERS + 1] = {CN_CIN, hidden, hidden, 1};
    int kmax = 0, nmax = 0;
    for (int l = 0; l < CN_LAYERS; ++l) {
        n->cin[l] = (l == 0) ? CN_CIN : round_up(ch[l], 16);
        n->cout[l] = ch[l + 1];
        n->npad[l] = round_up(ch[l + 1], 16);
        n->K[l] = round_up(9 * n->cin[l], 64);
        kmax = std::max(kmax, n->K[l]);
        nmax = std::max(nmax, n->npad[l] * n->K[l] + n->npad[l]);
    }
    auto fail = [&]() { cnn_free(n); return -1; };
    for (int l = 0; l < CN_LAYERS; ++l) {
        const size_t nw = (size_t)n->npad[l] * n->K[l];
        if (cn_alloc(&n->w32[l], nw) || cn_alloc(&n->b32[l], n->npad[l]) || cn_alloc(&n->gw[l], nw) ||
            cn_alloc(&n->gb[l], n->npad[l]) || cn_alloc(&n->mw[l], nw) || cn_alloc(&n->vw[l], nw) ||
            cn_alloc(&n->mb[l], n->npad[l]) || cn_alloc(&n->vb[l], n->npad[l]) || cn_alloc(&n->wbf[l], nw) ||
            cn_alloc(&n->wtbf[l], (size_t)n->K[l] * CN_KD) || cn_alloc(&n->h[l], (size_t)n->Ppad * n->cin[l]) ||
            cn_alloc(&n->z[l], (size_t)n->Ppad * n->npad[l]))
            return fail();
    }
    if (cn_alloc(&n->A, (size_t)n->Ppad * kmax) || cn_alloc(&n->dz, (size_t)n->Ppad * CN_KD) ||
        cn_alloc(&n->dzb, (size_t)n->Ppad * CN_KD) || cn_alloc(&n->dA, std::max((size_t)n->Ppad * kmax, (size_t)nmax)) ||
        cn_alloc(&n->part, (size_t)(n->Ppad / CN_WG_PB) * nmax) || cn_alloc(&n->lpart, (size_t)(n->Ppad + CN_NT - 1) / CN_NT) ||
        cn_alloc(&n->loss, 1) || cn_alloc(&n->err, 1))
        return fail();
    size_t wg_max = 0;
    for (int l = 0; l < CN_LAYERS; ++l)
        wg_max = std::max(wg_max, (size_t)CN_WG_PB * n->npad[l] * 4 + (size_t)CN_WG_PB * n->K[l] * 2);
    if (cudaFuncSetAttribute(k_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wg_max) != cudaSuccess) {
        set_error("nse2d_cnn_create: %s", cudaGetErrorString(cudaGetLastError()));
        return fail();
    }
    *out = n;
    return 0;
}

}  // namespace nse2d

using namespace nse2d;

struct nse2d_cnn {
    Cnn* n;
};

extern "C" {

int nse2d_gemm_bf16(const void* A, const void* B, const float* bias, float* Cf, void* Cb, int M, int N, int K, int ldc,
                    int relu, cudaStream_t s) {
    if (tc_gemm_setup()) return -1;
    void* e = nullptr;
    NSE_CUDA_TRY(cudaGetSymbolAddress(&e, g_tc_err));
    NSE_CUDA_TRY(cudaMemsetAsync(e, 0, sizeof(int), s));
    TcGemmParams p{};
    p.A = static_cast<const __nv_bfloat16*>(A);
    p.B = static_cast<const __nv_bfloat16*>(B);
    p.bias = bias;
    p.Cf = Cf;
    p.Cb = static_cast<__nv_bfloat16*>(Cb);
    p.err = static_cast<int*>(e);
    p.M = M; p.N = N; p.K = K; p.ldc = ldc; p.relu = relu;
    if (tc_gemm_launch(p, s)) return -1;
    int h = 0;
    NSE_CUDA_TRY(cudaMemcpyAsync(&h, e, sizeof(int), cudaMemcpyDeviceToHost, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    if (h) { set_error("tensor-core GEMM: an mbarrier wait ran out"); return -1; }
    return 0;
}

int nse2d_box_filter(const double* fine, int Nxf, int Nyf, double* coarse, int Nxc, int Nyc, cudaStream_t s) {
    if (!fine || !coarse || Nxc <= 0 || Nyc < 2 || Nxf % Nxc != 0 || (Nyf - 1) % (Nyc - 1) != 0) {
        set_error("nse2d_box_filter: Nxf must be a multiple of Nxc and Nyf - 1 of Nyc - 1");
        return -1;
    }
    k_box_filter<<<grid_of((long long)Nxc * Nyc), CN_NT, 0, s>>>(fine, Nxf, Nyf, coarse, Nxc, Nyc);
    NSE_CUDA_TRY(cudaGetLastError());
    return 0;
}

int nse2d_cnn_create(int Nx, int Ny, int hidden, nse2d_cnn** out) {
    if (!out) { set_error("nse2d_cnn_create: null output"); return -1; }
    *out = nullptr;
    Cnn* n = nullptr;
    if (cnn_create(Nx, Ny, hidden, &n)) return -1;
    *out = new nse2d_cnn{n};
    return 0;
}

int nse2d_cnn_destroy(nse2d_cnn* c) {
    if (!c) return 0;
    cnn_free(c->n);
    delete c;
    return 0;
}

int nse2d_cnn_layer_shape(nse2d_cnn* c, int layer, int* cin, int* cout) {
    if (!c || layer < 0 || layer >= CN_LAYERS) { set_error("nse2d_cnn_layer_shape: bad layer"); return -1; }
    if (cin) *cin = layer == 0 ? CN_CIN : c->n->cout[layer - 1];
    if (cout) *cout = c->n->cout[layer];
    return 0;
}

int nse2d_cnn_set_params(nse2d_cnn* c, int layer, const float* w, const float* b) {
    if (!c || layer < 0 || layer >= CN_LAYERS || !w || !b) { set_error("nse2d_cnn_set_params: bad arguments"); return -1; }
    Cnn* n = c->n;
    const int ci = layer == 0 ? CN_CIN : n->cout[layer - 1], co = n->cout[layer], K = n->K[layer], np = n->npad[layer];
    std::vector<float> wp((size_t)np * K, 0.f), bp(np, 0.f);
    for (int o = 0; o < co; ++o) {
        for (int tap = 0; tap < 9; ++tap)
            for (int ch = 0; ch < ci; ++ch) wp[(size_t)o * K + tap * n->cin[layer] + ch] = w[((size_t)o * 9 + tap) * ci + ch];
        bp[o] = b[o];
    }
    NSE_CUDA_TRY(cudaMemcpy(n->w32[layer], wp.data(), wp.size() * 4, cudaMemcpyHostToDevice));
    NSE_CUDA_TRY(cudaMemcpy(n->b32[layer], bp.data(), bp.size() * 4, cudaMemcpyHostToDevice));
    NSE_CUDA_TRY(cudaMemset(n->mw[layer], 0, wp.size() * 4));
    NSE_CUDA_TRY(cudaMemset(n->vw[layer], 0, wp.size() * 4));
    NSE_CUDA_TRY(cudaMemset(n->mb[layer], 0, bp.size() * 4));
    NSE_CUDA_TRY(cudaMemset(n->vb[layer], 0, bp.size() * 4));
    if (export_layer(n, layer, 0)) return -1;
    NSE_CUDA_TRY(cudaDeviceSynchronize());
    return 0;
}

static int get_layer(Cnn* n, int layer, const float* dw, const float* db, float* w, float* b) {
    const int ci = layer == 0 ? CN_CIN : n->cout[layer - 1], co = n->cout[layer], K = n->K[layer], np = n->npad[layer];
    std::vector<float> wp((size_t)np * K), bp(np);
    NSE_CUDA_TRY(cudaDeviceSynchronize());
    NSE_CUDA_TRY(cudaMemcpy(wp.data(), dw, wp.size() * 4, cudaMemcpyDeviceToHost));
    NSE_CUDA_TRY(cudaMemcpy(bp.data(), db, bp.size() * 4, cudaMemcpyDeviceToHost));
    for (int o = 0; o < co; ++o) {
        if (w)
            for (int tap = 0; tap < 9; ++tap)
                for (int ch = 0; ch < ci; ++ch) w[((size_t)o * 9 + tap) * ci + ch] = wp[(size_t)o * K + tap * n->cin[layer] + ch];
        if (b) b[o] = bp[o];
    }
    return 0;
}

int nse2d_cnn_get_params(nse2d_cnn* c, int layer, float* w, float* b) {
    if (!c || layer < 0 || layer >= CN_LAYERS) { set_error("nse2d_cnn_get_params: bad layer"); return -1; }
    return get_layer(c->n, layer, c->n->w32[layer], c->n->b32[layer], w, b);
}

int nse2d_cnn_get_grads(nse2d_cnn* c, int layer, float* w, float* b) {
    if (!c || layer < 0 || layer >= CN_LAYERS) { set_error("nse2d_cnn_get_grads: bad layer"); return -1; }
    return get_layer(c->n, layer, c->n->gw[layer], c->n->gb[layer], w, b);
}

int nse2d_cnn_set_scales(nse2d_cnn* c, double w_scale, double psi_scale, double tau_scale) {
    if (!c || !(w_scale > 0) || !(psi_scale > 0) || !(tau_scale > 0)) { set_error("nse2d_cnn_set_scales: scales must be > 0"); return -1; }
    c->n->in_w = w_scale; c->n->in_psi = psi_scale; c->n->out_tau = tau_scale;
    return 0;
}

int nse2d_set_closure(nse2d_ctx* ctx, nse2d_cnn* net) {
    if (!ctx || !ctx->c) { set_error("nse2d_set_closure: null context"); return -1; }
    Context* c = ctx->c;
    if (!net) { c->closure_net = nullptr; return 0; }
    if (!cnn_matches(net->n, c->Nx, c->Ny)) {
        set_error("nse2d_set_closure: the model is for %dx%d, the context is %dx%d", net->n->Nx, net->n->Ny, c->Nx, c->Ny);
        return -1;
    }
    if (c->prec32) { set_error("nse2d_set_closure: the closure runs with precision 64"); return -1; }
    if (!c->closure_tau) {
        NSE_CUDA_TRY(cudaMalloc((void**)&c->closure_tau, c->N * sizeof(double)));
        NSE_CUDA_TRY(cudaMemset(c->closure_tau, 0, c->N * sizeof(double)));
    }
    if (c->run_exec) { cudaGraphExecDestroy(c->run_exec); c->run_exec = nullptr; }
    if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
    c->closure_net = net->n;
    return 0;
}

int nse2d_cnn_forward(nse2d_cnn* c, const double* w, const double* psi, double* tau, cudaStream_t s) {
    if (!c || !w || !psi) { set_error("nse2d_cnn_forward: null argument"); return -1; }
    return cnn_forward(c->n, w, psi, tau, s);
}

int nse2d_cnn_gradients(nse2d_cnn* c, const double* w, const double* psi, const double* tau_target, float* loss,
                        cudaStream_t s) {
    if (!c || !w || !psi || !tau_target) { set_error("nse2d_cnn_gradients: null argument"); return -1; }
    if (cnn_forward(c->n, w, psi, nullptr, s) || cnn_backward(c->n, tau_target, s)) return -1;
    if (loss) {
        NSE_CUDA_TRY(cudaMemcpyAsync(loss, c->n->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
        NSE_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return 0;
}

int nse2d_cnn_train_step(nse2d_cnn* c, const double* w, const double* psi, const double* tau_target, float lr,
                         float weight_decay, float* loss, cudaStream_t s) {
    if (nse2d_cnn_gradients(c, w, psi, tau_target, nullptr, s)) return -1;
    if (cnn_adamw(c->n, lr, weight_decay, s)) return -1;
    if (loss) {
        NSE_CUDA_TRY(cudaMemcpyAsync(loss, c->n->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
        NSE_CUDA_TRY(cudaStreamSynchronize(s));
        int e = 0;
        NSE_CUDA_TRY(cudaMemcpy(&e, c->n->err, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) { set_error("nse2d_cnn_train_step: a tensor-core wait ran out"); return -1; }
    }
    return 0;
}

}  // extern "C"
