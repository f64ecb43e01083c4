// BF16 GEMM on the 5th-generation tensor cores (tcgen05) for the learned closure's
// convolutions, written for this project: C[M][N] = A[M][K] . B[N][K]^T, FP32 accumulate.
//
// A and B are row-major with K contiguous ("K-major"), BF16. M is a multiple of 128, N a
// multiple of 16 in [16, 256], K a multiple of 64 (callers pad with zeros). One CTA of 4 warps
// owns 128 rows of C and all N columns; the accumulator lives in tensor memory (TMEM, 128 lanes
// x N 32-bit columns) and never touches registers until the epilogue.
//
// Per K-block of 64:
//   - all threads copy the A tile (128 x 64) and the B tile (N x 64) with 16-byte cp.async into
//     the no-swizzle "core matrix" layout the MMA reads: 8 rows x 16 bytes per 128-byte core
//     matrix, core matrices ordered [row group][k chunk], so that the byte step between the two
//     k halves of one MMA (LBO) is 128 and between 8-row groups (SBO) is 8 x 128;
//   - the copies of block kb+1 go to the other of two buffers while block kb is multiplied;
//   - one thread issues four tcgen05.mma (M = 128, N, K = 16) and tcgen05.commit, which arrives
//     on the buffer's mbarrier when the MMAs have read it.
// After the last block all threads wait on that barrier; warp w reads TMEM lanes 32w..32w+31
// (rows of C) with tcgen05.ld 32x32b.x16 and applies the epilogue: + bias[n], an activation,
// FP32 and/or BF16 stores (the BF16 output after the activation: ReLU or GELU).
//
// Every mbarrier wait is bounded. A wait that runs out sets *err and the CTA still waits
// (bounded) for its MMAs before it frees its TMEM and returns.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace nse2d {

constexpr int TG_BM = 128;               // rows of C per CTA
constexpr int TG_BK = 64;                // K per block
constexpr int TG_THREADS = 128;
constexpr unsigned TG_WAIT_LIMIT = 1u << 24;

__host__ __device__ constexpr size_t tg_buf_bytes(int N) { return (size_t)(TG_BM + N) * TG_BK * 2; }
__host__ __device__ constexpr size_t tg_smem_bytes(int N) { return 2 * tg_buf_bytes(N) + 128; }

struct TcGemmParams {
    const __nv_bfloat16* A;  // [M][K]
    const __nv_bfloat16* B;  // [N][K]
    const float* bias;       // [N] or null
    float* Cf;               // [M][ldc] FP32 (pre-activation) or null
    __nv_bfloat16* Cb;       // [M][ldc] BF16 (after the activation) or null
    int* err;                // set to 1 by a wait that ran out
    int M, N, K, ldc;
    int act;                 // activation of the BF16 output: 0 none, 1 ReLU, 2 GELU (tanh form)
};

// GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))), and its derivative.
__device__ __forceinline__ float tg_gelu(float x) {
    const float u = 0.7978845608028654f * fmaf(0.044715f * x, x * x, x);
    return 0.5f * x * (1.f + tanhf(u));
}
__device__ __forceinline__ float tg_gelu_grad(float x) {
    const float u = 0.7978845608028654f * fmaf(0.044715f * x, x * x, x);
    const float t = tanhf(u);
    return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * 0.7978845608028654f * fmaf(0.134145f, x * x, 1.f);
}

__device__ __forceinline__ uint32_t tg_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor, no swizzle, K-major: start, LBO, SBO in 16-byte units, version 1.
__device__ __forceinline__ uint64_t tg_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, M = 128.
__host__ __device__ constexpr uint32_t tg_idesc(int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(TG_BM >> 4) << 24);
}

__device__ __forceinline__ void tg_cp16(uint32_t s, const void* g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void tg_bar_init(uint64_t* b) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(tg_smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool tg_bar_wait(uint64_t* b, unsigned parity) {
    for (unsigned it = 0; it < TG_WAIT_LIMIT; ++it) {
        unsigned ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(ok) : "r"(tg_smem_u32(b)), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}

// Copies block kb of A (rows m0..m0+127) and B into the core-matrix layout of buffer sA/sB.
__device__ __forceinline__ void tg_load_block(const TcGemmParams& p, int m0, int kb, uint32_t sA, uint32_t sB) {
    const int k0 = kb * TG_BK;
    for (int ch = threadIdx.x; ch < TG_BM * 8; ch += TG_THREADS) {       // 8 chunks of 16 bytes per row
        const int r = ch >> 3, c = ch & 7;
        tg_cp16(sA + (uint32_t)((((r >> 3) * 8 + c) << 7) + ((r & 7) << 4)), p.A + (size_t)(m0 + r) * p.K + k0 + c * 8);
    }
    for (int ch = threadIdx.x; ch < p.N * 8; ch += TG_THREADS) {
        const int r = ch >> 3, c = ch & 7;
        tg_cp16(sB + (uint32_t)((((r >> 3) * 8 + c) << 7) + ((r & 7) << 4)), p.B + (size_t)r * p.K + k0 + c * 8);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

static __global__ void __launch_bounds__(TG_THREADS) k_tc_gemm(TcGemmParams p) {
    extern __shared__ __align__(16) unsigned char tg_smem[];
    __shared__ __align__(8) uint64_t mma_bar[2];
    __shared__ uint32_t tmem_base;
    unsigned char* sm = tg_smem + ((128u - (tg_smem_u32(tg_smem) & 127u)) & 127u);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TG_BM;
    const int nk = p.K / TG_BK;
    const uint32_t ncols = p.N <= 32 ? 32u : (p.N <= 64 ? 64u : (p.N <= 128 ? 128u : 256u));
    const uint32_t buf = (uint32_t)tg_buf_bytes(p.N);
    const uint32_t s0 = tg_smem_u32(sm);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(tg_smem_u32(&tmem_base)), "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        tg_bar_init(&mma_bar[0]);
        tg_bar_init(&mma_bar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base;
    bool ok = true;
    tg_load_block(p, m0, 0, s0, s0 + TG_BM * TG_BK * 2);
    const uint32_t idesc = tg_idesc(p.N);
    for (int kb = 0; kb < nk; ++kb) {
        const int b = kb & 1;
        if (kb + 1 < nk) {
            // the other buffer was read by the MMAs of block kb-1
            if (kb >= 1) ok &= tg_bar_wait(&mma_bar[b ^ 1], (unsigned)(((kb - 1) >> 1) & 1));
            const uint32_t sb = s0 + (uint32_t)(b ^ 1) * buf;
            tg_load_block(p, m0, kb + 1, sb, sb + TG_BM * TG_BK * 2);
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");    // copies visible to the tensor core
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t sa = s0 + (uint32_t)b * buf, sbm = sa + TG_BM * TG_BK * 2;
#pragma unroll
            for (int kk = 0; kk < TG_BK / 16; ++kk) {
                const uint64_t da = tg_desc(sa + kk * 256, 128, 1024);
                const uint64_t db = tg_desc(sbm + kk * 256, 128, 1024);
                const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
                asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                             " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                             ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                         ::"r"(tg_smem_u32(&mma_bar[b])) : "memory");
        }
    }
    // the last commit covers every MMA of this CTA
    const int last = nk - 1;
    ok &= tg_bar_wait(&mma_bar[last & 1], (unsigned)((last >> 1) & 1));
    if (!ok) {
        atomicOr(p.err, 1);
        tg_bar_wait(&mma_bar[last & 1], (unsigned)((last >> 1) & 1));
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    // epilogue: row m0 + 32 warp + lane, 16 columns per TMEM load
    const int row = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < p.N; c0 += 16) {
        uint32_t v[16];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
                     : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                       "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                     : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (row < p.M) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float z = __uint_as_float(v[i]);
                if (p.bias) z += p.bias[c0 + i];
                if (p.Cf) p.Cf[(size_t)row * p.ldc + c0 + i] = z;
                if (p.Cb) {
                    const float a = p.act == 1 ? fmaxf(z, 0.f) : (p.act == 2 ? tg_gelu(z) : z);
                    p.Cb[(size_t)row * p.ldc + c0 + i] = __float2bfloat16_rn(a);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(ncols) : "memory");
}

}  // namespace nse2d
