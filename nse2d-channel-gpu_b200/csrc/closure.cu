// The learned subgrid closure: a small CNN whose 3x3 convolutions run as BF16 GEMMs on the
// tensor cores (tcgen05, FP32 accumulate), its backward pass, AdamW, and the coarse-grid data
// generator (box filter). Written for this project; the reference has no closure model.
//
// Model. Inputs per point: the coarse omega, psi, u, v (each divided by a fixed scale) and y,
// 5 channels. Four 3x3 convolutions 5 -> H -> H -> H -> 1, GELU (tanh form) after the first
// three, periodic in x and zero-padded beyond the walls. Output: tau / tau_scale, the subgrid
// term of the Jacobian,
//   tau = filter(J(psi, omega)) - J(filter psi, filter omega),
// which the coarse solver subtracts from its rhs on interior rows. A batch is B whole coarse
// fields side by side; every field keeps its own periodic x and its own walls.
//
// Layout. A pixel p = b Nx Ny + j Nx + i; activations are BF16 [P_pad][C] (channels
// contiguous), P_pad a multiple of 128. A convolution is im2col (A[p][k], k = tap C + c,
// tap = 3 (dy + 1) + dx + 1, K padded to a multiple of 64) and the GEMM Z = A . W^T + b with
// W [N_pad][K] (N_pad a multiple of 16); the GEMM's epilogue writes Z (FP32, kept for the
// backward pass) and GELU(Z) in BF16, the next layer's input.
//
// Backward (loss = mean over interior pixels of (z - tau/tau_scale)^2):
//   dW[n][k] = sum_p dZ[p][n] A[p][k] and db[n] = sum_p dZ[p][n] on the CUDA cores (per-block
//   partials folded in a fixed order, so the gradients do not depend on scheduling);
//   dA = dZ . W on the tensor cores (dZ in BF16, padded to 64 channels; W^T kept in BF16);
//   col2im gathers dA back to the pixels of the layer input and multiplies by GELU'(z).
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

constexpr int CN_LAYERS = 4;
constexpr int CN_CIN = 5;                 // omega, psi, u, v, y
constexpr int CN_KD = 64;                 // reduction width of the input-gradient GEMM (channels padded)
constexpr int CN_WG_PB = 64;              // pixels per block of the weight-gradient reduction
constexpr int CN_NT = 256;
constexpr int CN_ACT = 2;                 // GELU

int round_up(int x, int m) { return (x + m - 1) / m * m; }

}  // namespace

struct Cnn {
    int Nx = 0, Ny = 0, nxy = 0, hidden = 0, max_batch = 0;
    int nb = 1, P = 0, Ppad = 0;          // the current batch
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
    __nv_bfloat16* h[CN_LAYERS] = {};     // layer input: h[0] [Ppad][5], h[l] [Ppad][npad[l-1]]
    __nv_bfloat16* A = nullptr;           // im2col of the current layer [Ppad][Kmax]
    float* z[CN_LAYERS] = {};             // pre-activations [Ppad][npad]
    float* dz = nullptr;                  // [Ppad][64]
    __nv_bfloat16* dzb = nullptr;         // [Ppad][64]
    float* dA = nullptr;                  // [Ppad][Kmax]
    float* part = nullptr;                // weight-gradient partials [nblk][npad K + npad]
    float* lpart = nullptr;               // loss partials [ceil(Ppad / CN_NT)]
    float* loss = nullptr;                // [1]
    double* y = nullptr;                  // [Ny] wall-normal coordinate (the fifth input)
    int* idx = nullptr;                   // [max_batch] sample of every batch slot
    int* err = nullptr;
    double in_scale[CN_CIN - 1] = {1.0, 1.0, 1.0, 1.0};
    double out_tau = 1.0;
    int wall_rows = 1;                    // rows next to each wall (the wall row included) with tau = 0
    double gain = 1.0;                    // factor on the applied tau
    bool row_mean = false;                // apply the x-mean of tau on every row (the mean-flow part)
    long long step = 0;
};

int tc_gemm_launch(const TcGemmParams& p0, cudaStream_t s);

namespace {

template <typename T> int cn_alloc(T** p, size_t n) {
    NSE_CUDA_TRY(cudaMalloc((void**)p, n * sizeof(T) + 16));
    NSE_CUDA_TRY(cudaMemset(*p, 0, n * sizeof(T) + 16));
    return 0;
}

struct PackSrc {
    const double* w;         // [S][Ny][Nx]; batch slot b reads sample idx[b]
    const double* psi;
    const double* u;
    const double* v;
    const int* idx;          // [nb]
    const double* y;         // [Ny]
    double s0, s1, s2, s3;   // 1 / scale of omega, psi, u, v
};

// the 5 input channels of every pixel of the batch (zero on padding pixels)
__global__ void k_pack_input(PackSrc q, __nv_bfloat16* h0, int nxy, int Nx, int P, int Ppad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= Ppad) return;
    float v[CN_CIN] = {0.f, 0.f, 0.f, 0.f, 0.f};
    if (p < P) {
        const int b = p / nxy, r = p - b * nxy;
        const size_t src = (size_t)q.idx[b] * nxy + r;
        v[0] = (float)(q.w[src] * q.s0);
        v[1] = (float)(q.psi[src] * q.s1);
        v[2] = (float)(q.u[src] * q.s2);
        v[3] = (float)(q.v[src] * q.s3);
        v[4] = (float)q.y[r / Nx];
    }
#pragma unroll
    for (int c = 0; c < CN_CIN; ++c) h0[(size_t)p * CN_CIN + c] = __float2bfloat16_rn(v[c]);
}

// A[p][k] for one 8-wide chunk of k per thread; taps outside the walls of the pixel's own field
// read zero, x is periodic within the field.
__global__ void k_im2col(const __nv_bfloat16* h, int C, int Nx, int Ny, int P, int Ppad, int K, __nv_bfloat16* A) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nch = K / 8;
    if (t >= (long long)Ppad * nch) return;
    const int p = (int)(t / nch), k0 = (int)(t % nch) * 8;
    const int nxy = Nx * Ny;
    const int b = p / nxy, r = p - b * nxy;
    const int j = r / Nx, i = r - j * Nx;
    const size_t base = (size_t)b * nxy;
    __align__(16) __nv_bfloat16 v[8];
    if ((C & 7) == 0 && k0 < 9 * C) {                    // the chunk is 8 channels of one tap
        const int tap = k0 / C, c = k0 - tap * C;
        const int jj = j + tap / 3 - 1, ii = i + tap % 3 - 1;
        if (p < P && jj >= 0 && jj < Ny) {
            const int iw = ii < 0 ? ii + Nx : (ii >= Nx ? ii - Nx : ii);
            *reinterpret_cast<uint4*>(v) = *reinterpret_cast<const uint4*>(h + (base + (size_t)jj * Nx + iw) * C + c);
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
                    x = __bfloat162float(h[(base + (size_t)jj * Nx + iw) * C + c]);
                }
            }
            v[e] = __float2bfloat16_rn(x);
        }
    }
    *reinterpret_cast<uint4*>(A + (size_t)p * K + k0) = *reinterpret_cast<const uint4*>(v);
}

// tau = tau_scale z[p][0] away from the walls, 0 on the wall_rows rows next to each wall
// (batch slot 0)
__global__ void k_unpack_output(const float* z, int ldz, double* tau, int Nx, int Ny, double ts, int wall_rows) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= Nx * Ny) return;
    const int j = p / Nx;
    tau[p] = (j < wall_rows || j >= Ny - wall_rows) ? 0.0 : ts * (double)z[(size_t)p * ldz];
}

// the x-mean of tau on every row: one CTA per row
__global__ void __launch_bounds__(CN_NT) k_unpack_row_mean(const float* z, int ldz, double* tau, int Nx, int Ny, double ts,
                                                           int wall_rows) {
    __shared__ double red[CN_NT];
    const int j = blockIdx.x;
    double sum = 0.0;
    for (int i = threadIdx.x; i < Nx; i += CN_NT) sum += (double)z[((size_t)j * Nx + i) * ldz];
    red[threadIdx.x] = sum;
    __syncthreads();
    for (int st = CN_NT / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    const double m = (j < wall_rows || j >= Ny - wall_rows) ? 0.0 : ts * red[0] / (double)Nx;
    for (int i = threadIdx.x; i < Nx; i += CN_NT) tau[(size_t)j * Nx + i] = m;
}

// loss partials and dZ of the output layer: d = z - tau / tau_scale on interior pixels
__global__ void __launch_bounds__(CN_NT) k_loss(const float* z, int ldz, const double* tau, const int* idx, double inv_ts,
                                                int Nx, int Ny, int P, int Ppad, int wall_rows, float inv_pint, float* dz,
                                                __nv_bfloat16* dzb, float* lpart) {
    __shared__ float red[CN_NT];
    const int p = blockIdx.x * CN_NT + threadIdx.x;
    const int nxy = Nx * Ny;
    float l = 0.f;
    if (p < Ppad) {
        float g = 0.f;
        if (p < P) {
            const int b = p / nxy, r = p - b * nxy, j = r / Nx;
            if (j >= wall_rows && j < Ny - wall_rows) {
                const float d = z[(size_t)p * ldz] - (float)(tau[(size_t)idx[b] * nxy + r] * inv_ts);
                l = d * d;
                g = 2.f * d * inv_pint;
            }
        }
        for (int c = 0; c < CN_KD; ++c) {
            dz[(size_t)p * CN_KD + c] = c == 0 ? g : 0.f;
            dzb[(size_t)p * CN_KD + c] = __float2bfloat16_rn(c == 0 ? g : 0.f);
        }
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int st = CN_NT / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
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

// dh[q][c] = sum over taps of dA[q - tap offset][tap C + c] (source rows inside the walls of the
// same field), then the activation's derivative of the layer below: dz[q][c] = dh GELU'(z_prev);
// channels >= C written as zero.
__global__ void k_col2im_act(const float* dA, int K, int C, const float* zprev, int ldzp, int Nx, int Ny, int P, int Ppad,
                             float* dz, __nv_bfloat16* dzb) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)Ppad * CN_KD) return;
    const int q = (int)(t / CN_KD), c = (int)(t % CN_KD);
    float g = 0.f;
    if (q < P && c < C) {
        const int nxy = Nx * Ny;
        const int b = q / nxy, r = q - b * nxy;
        const int j = r / Nx, i = r - j * Nx;
        const size_t base = (size_t)b * nxy;
        float s = 0.f;
#pragma unroll
        for (int tap = 0; tap < 9; ++tap) {
            const int dy = tap / 3 - 1, dx = tap % 3 - 1;
            const int jp = j - dy;
            if (jp < 0 || jp >= Ny) continue;
            int ip = i - dx;
            ip = ip < 0 ? ip + Nx : (ip >= Nx ? ip - Nx : ip);
            s += dA[(base + (size_t)jp * Nx + ip) * K + tap * C + c];
        }
        g = s * tg_gelu_grad(zprev[(size_t)q * ldzp + c]);
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
         int N, int K, int ldc, int act, cudaStream_t s) {
    TcGemmParams p{};
    p.A = A; p.B = B; p.bias = bias; p.Cf = Cf; p.Cb = Cb; p.err = n ? n->err : nullptr;
    p.M = M; p.N = N; p.K = K; p.ldc = ldc; p.act = act;
    return tc_gemm_launch(p, s);
}

int export_layer(Cnn* n, int l, cudaStream_t s) {
    k_export_w<<<grid_of((long long)n->K[l] * CN_KD), CN_NT, 0, s>>>(n->w32[l], n->npad[l], n->K[l], n->wbf[l], n->wtbf[l]);
    NSE_CUDA_TRY(cudaGetLastError());
    return 0;
}

void set_batch(Cnn* n, int nb) {
    n->nb = nb;
    n->P = nb * n->nxy;
    n->Ppad = round_up(n->P, 128);
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

// Forward pass of the current batch from the packed sources.
static int cnn_forward_batch(Cnn* n, const PackSrc& src, cudaStream_t s) {
    k_pack_input<<<grid_of(n->Ppad), CN_NT, 0, s>>>(src, n->h[0], n->nxy, n->Nx, n->P, n->Ppad);
    NSE_CUDA_TRY(cudaGetLastError());
    for (int l = 0; l < CN_LAYERS; ++l) {
        k_im2col<<<grid_of((long long)n->Ppad * (n->K[l] / 8)), CN_NT, 0, s>>>(n->h[l], n->cin[l], n->Nx, n->Ny, n->P, n->Ppad,
                                                                              n->K[l], n->A);
        NSE_CUDA_TRY(cudaGetLastError());
        const bool last = (l == CN_LAYERS - 1);
        if (gemm(n, n->A, n->wbf[l], n->b32[l], n->z[l], last ? nullptr : n->h[l + 1], n->Ppad, n->npad[l], n->K[l],
                 n->npad[l], CN_ACT, s))
            return -1;
    }
    return 0;
}

static PackSrc pack_src(const Cnn* n, const double* w, const double* psi, const double* u, const double* v) {
    PackSrc q{};
    q.w = w; q.psi = psi; q.u = u; q.v = v; q.idx = n->idx; q.y = n->y;
    q.s0 = 1.0 / n->in_scale[0]; q.s1 = 1.0 / n->in_scale[1]; q.s2 = 1.0 / n->in_scale[2]; q.s3 = 1.0 / n->in_scale[3];
    return q;
}

// Inference on one field (slot 0 of the index table is always sample 0); graph-capturable.
int cnn_forward(Cnn* n, const double* w, const double* psi, const double* u, const double* v, double* tau, cudaStream_t s) {
    set_batch(n, 1);
    if (cnn_forward_batch(n, pack_src(n, w, psi, u, v), s)) return -1;
    if (n->row_mean)
        k_unpack_row_mean<<<n->Ny, CN_NT, 0, s>>>(n->z[CN_LAYERS - 1], n->npad[CN_LAYERS - 1], tau, n->Nx, n->Ny,
                                                  n->out_tau * n->gain, n->wall_rows);
    else
        k_unpack_output<<<grid_of(n->nxy), CN_NT, 0, s>>>(n->z[CN_LAYERS - 1], n->npad[CN_LAYERS - 1], tau, n->Nx, n->Ny,
                                                          n->out_tau * n->gain, n->wall_rows);
    NSE_CUDA_TRY(cudaGetLastError());
    return 0;
}

// Loss against tau (samples idx of the batch) and the gradients of every layer (after the forward pass).
static int cnn_backward(Cnn* n, const double* tau, cudaStream_t s) {
    const int nlb = (n->Ppad + CN_NT - 1) / CN_NT;
    const int pint = n->nb * n->Nx * (n->Ny - 2 * n->wall_rows);
    k_loss<<<nlb, CN_NT, 0, s>>>(n->z[CN_LAYERS - 1], n->npad[CN_LAYERS - 1], tau, n->idx, 1.0 / n->out_tau, n->Nx, n->Ny, n->P,
                                 n->Ppad, n->wall_rows, 1.f / (float)pint, n->dz, n->dzb, n->lpart);
    NSE_CUDA_TRY(cudaGetLastError());
    k_fold<<<1, 32, 0, s>>>(n->lpart, nlb, 1, n->loss, 1.f / (float)pint);
    NSE_CUDA_TRY(cudaGetLastError());
    for (int l = CN_LAYERS - 1; l >= 0; --l) {
        // the layer's im2col again (one A buffer is kept)
        k_im2col<<<grid_of((long long)n->Ppad * (n->K[l] / 8)), CN_NT, 0, s>>>(n->h[l], n->cin[l], n->Nx, n->Ny, n->P, n->Ppad,
                                                                              n->K[l], n->A);
        NSE_CUDA_TRY(cudaGetLastError());
        const int nblk = n->Ppad / CN_WG_PB, nout = n->npad[l] * n->K[l] + n->npad[l];
        const size_t sm = (size_t)CN_WG_PB * n->npad[l] * 4 + (size_t)CN_WG_PB * n->K[l] * 2;
        k_wgrad<<<nblk, CN_NT, sm, s>>>(n->dz, n->A, n->npad[l], n->K[l], n->part);
        NSE_CUDA_TRY(cudaGetLastError());
        // fold into the scratch dA (weights then biases), then copy out
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
        k_col2im_act<<<grid_of((long long)n->Ppad * CN_KD), CN_NT, 0, s>>>(n->dA, n->K[l], n->cin[l], n->z[l - 1],
                                                                            n->npad[l - 1], n->Nx, n->Ny, n->P, n->Ppad, n->dz,
                                                                            n->dzb);
        NSE_CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

static int cnn_adamw(Cnn* n, float lr, float wd, cudaStream_t s) {
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
    cudaFree(n->loss); cudaFree(n->y); cudaFree(n->idx); cudaFree(n->err);
    delete n;
}

static int cnn_create(int Nx, int Ny, int hidden, int max_batch, const double* y_host, Cnn** out) {
    *out = nullptr;
    if (Nx < 4 || Ny < 5 || hidden < 16 || hidden > 64 || hidden % 16 != 0 || max_batch < 1 || !y_host) {
        set_error("nse2d_cnn_create: Nx >= 4, Ny >= 5, hidden a multiple of 16 in [16, 64], max_batch >= 1, y given");
        return -1;
    }
    if ((long long)max_batch * Nx * Ny > (1ll << 30)) { set_error("nse2d_cnn_create: batch too large"); return -1; }
    if (tc_gemm_setup()) return -1;
    Cnn* n = new Cnn();
    n->Nx = Nx; n->Ny = Ny; n->nxy = Nx * Ny; n->hidden = hidden; n->max_batch = max_batch;
    set_batch(n, max_batch);
    const int Pmax = n->Ppad;
    const int ch[CN_LAYERS + 1] = {CN_CIN, hidden, hidden, hidden, 1};
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
            cn_alloc(&n->wtbf[l], (size_t)n->K[l] * CN_KD) || cn_alloc(&n->h[l], (size_t)Pmax * n->cin[l]) ||
            cn_alloc(&n->z[l], (size_t)Pmax * n->npad[l]))
            return fail();
    }
    if (cn_alloc(&n->A, (size_t)Pmax * kmax) || cn_alloc(&n->dz, (size_t)Pmax * CN_KD) ||
        cn_alloc(&n->dzb, (size_t)Pmax * CN_KD) || cn_alloc(&n->dA, std::max((size_t)Pmax * kmax, (size_t)nmax)) ||
        cn_alloc(&n->part, (size_t)(Pmax / CN_WG_PB) * nmax) || cn_alloc(&n->lpart, (size_t)(Pmax + CN_NT - 1) / CN_NT) ||
        cn_alloc(&n->loss, 1) || cn_alloc(&n->y, Ny) || cn_alloc(&n->idx, max_batch) || cn_alloc(&n->err, 1))
        return fail();
    if (cudaMemcpy(n->y, y_host, sizeof(double) * Ny, cudaMemcpyHostToDevice) != cudaSuccess) {
        set_error("nse2d_cnn_create: y upload");
        return fail();
    }
    size_t wg_max = 0;
    for (int l = 0; l < CN_LAYERS; ++l)
        wg_max = std::max(wg_max, (size_t)CN_WG_PB * n->npad[l] * 4 + (size_t)CN_WG_PB * n->K[l] * 2);
    if (cudaFuncSetAttribute(k_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wg_max) != cudaSuccess) {
        set_error("nse2d_cnn_create: %s", cudaGetErrorString(cudaGetLastError()));
        return fail();
    }
    set_batch(n, 1);
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
    p.M = M; p.N = N; p.K = K; p.ldc = ldc; p.act = relu ? 1 : 0;
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

int nse2d_cnn_create(int Nx, int Ny, int hidden, int max_batch, const double* y, nse2d_cnn** out) {
    if (!out) { set_error("nse2d_cnn_create: null output"); return -1; }
    *out = nullptr;
    Cnn* n = nullptr;
    if (cnn_create(Nx, Ny, hidden, max_batch, y, &n)) return -1;
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
    n->step = 0;
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

int nse2d_cnn_set_scales(nse2d_cnn* c, const double* in_scales, double tau_scale) {
    if (!c || !in_scales || !(tau_scale > 0)) { set_error("nse2d_cnn_set_scales: bad arguments"); return -1; }
    for (int k = 0; k < CN_CIN - 1; ++k) {
        if (!(in_scales[k] > 0)) { set_error("nse2d_cnn_set_scales: scales must be > 0"); return -1; }
        c->n->in_scale[k] = in_scales[k];
    }
    c->n->out_tau = tau_scale;
    return 0;
}

int nse2d_cnn_set_application(nse2d_cnn* c, int wall_rows, double gain, int row_mean) {
    if (!c || wall_rows < 1 || 2 * wall_rows >= c->n->Ny - 1 || !(gain >= 0.0)) {
        set_error("nse2d_cnn_set_application: wall_rows in [1, (Ny - 1) / 2), gain >= 0");
        return -1;
    }
    c->n->wall_rows = wall_rows;
    c->n->gain = gain;
    c->n->row_mean = row_mean != 0;
    return 0;
}

int nse2d_set_closure(nse2d_ctx* ctx, nse2d_cnn* net, int every_stage) {
    if (!ctx || !ctx->c) { set_error("nse2d_set_closure: null context"); return -1; }
    Context* c = ctx->c;
    if (c->run_exec) { cudaGraphExecDestroy(c->run_exec); c->run_exec = nullptr; }
    if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
    if (!net) { c->closure_net = nullptr; return 0; }
    if (!cnn_matches(net->n, c->Nx, c->Ny)) {
        set_error("nse2d_set_closure: the model is for %dx%d, the context is %dx%d", net->n->Nx, net->n->Ny, c->Nx, c->Ny);
        return -1;
    }
    if (c->prec32) { set_error("nse2d_set_closure: the closure runs with precision 64"); return -1; }
    if (!c->closure_tau) {
        NSE_CUDA_TRY(cudaMalloc((void**)&c->closure_tau, 3 * c->N * sizeof(double)));
        NSE_CUDA_TRY(cudaMemset(c->closure_tau, 0, 3 * c->N * sizeof(double)));
    }
    c->closure_net = net->n;
    c->closure_every_stage = every_stage != 0;
    return 0;
}

int nse2d_cnn_forward(nse2d_cnn* c, const double* w, const double* psi, const double* u, const double* v, double* tau,
                      cudaStream_t s) {
    if (!c || !w || !psi || !u || !v || !tau) { set_error("nse2d_cnn_forward: null argument"); return -1; }
    return cnn_forward(c->n, w, psi, u, v, tau, s);
}

static int batch_setup(Cnn* n, const int* idx, int nb, cudaStream_t s) {
    if (!idx || nb < 1 || nb > n->max_batch) { set_error("nse2d_cnn: batch of %d (1..%d)", nb, n->max_batch); return -1; }
    for (int b = 0; b < nb; ++b)
        if (idx[b] < 0) { set_error("nse2d_cnn: negative sample index"); return -1; }
    set_batch(n, nb);
    NSE_CUDA_TRY(cudaMemcpyAsync(n->idx, idx, sizeof(int) * nb, cudaMemcpyHostToDevice, s));
    return 0;
}

int nse2d_cnn_gradients(nse2d_cnn* c, const double* w, const double* psi, const double* u, const double* v,
                        const double* tau, const int* idx, int nb, float* loss, cudaStream_t s) {
    if (!c || !w || !psi || !u || !v || !tau) { set_error("nse2d_cnn_gradients: null argument"); return -1; }
    Cnn* n = c->n;
    if (batch_setup(n, idx, nb, s)) return -1;
    const int rc = (cnn_forward_batch(n, pack_src(n, w, psi, u, v), s) || cnn_backward(n, tau, s)) ? -1 : 0;
    // slot 0 back to sample 0 for inference
    const int zero = 0;
    NSE_CUDA_TRY(cudaMemcpyAsync(n->idx, &zero, sizeof(int), cudaMemcpyHostToDevice, s));
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    if (rc) return -1;
    if (loss) NSE_CUDA_TRY(cudaMemcpy(loss, n->loss, sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}

int nse2d_cnn_train_step(nse2d_cnn* c, const double* w, const double* psi, const double* u, const double* v,
                         const double* tau, const int* idx, int nb, float lr, float weight_decay, float* loss,
                         cudaStream_t s) {
    if (nse2d_cnn_gradients(c, w, psi, u, v, tau, idx, nb, loss, s)) return -1;
    if (cnn_adamw(c->n, lr, weight_decay, s)) return -1;
    NSE_CUDA_TRY(cudaStreamSynchronize(s));
    int e = 0;
    NSE_CUDA_TRY(cudaMemcpy(&e, c->n->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) { set_error("nse2d_cnn_train_step: a tensor-core wait ran out"); return -1; }
    return 0;
}

}  // extern "C"
