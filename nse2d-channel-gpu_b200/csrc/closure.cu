// The learned subgrid closure: BF16 convolution layers on the tensor cores (tcgen05, FP32
// accumulate), their backward pass, AdamW, and the coarse-grid data generator. Written for
// this project; the reference has no closure model.
#include <cstdint>

#include "common.cuh"
#include "tc_gemm.cuh"
#include "../../include/nse2d.h"

namespace nse2d {
namespace {

__device__ int g_tc_err;                  // error flag of the tensor-core GEMM's bounded waits

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
    const size_t smem = tg_smem_bytes(p.N);
    NSE_CUDA_TRY(cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_tc_gemm<<<p.M / TG_BM, TG_THREADS, smem, s>>>(p);
    NSE_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace
}  // namespace nse2d

using namespace nse2d;

extern "C" {

int nse2d_gemm_bf16(const void* A, const void* B, const float* bias, float* Cf, void* Cb, int M, int N, int K, int ldc,
                    int relu, cudaStream_t s) {
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

}  // extern "C"
