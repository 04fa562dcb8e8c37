// Learned initialiser: tensor-core GEMM entry point (the convolution-as-GEMM layers
// and their training are built on it).
#include <cuda_bf16.h>

#include <new>

#include "gemm_tc.cuh"
#include "internal.h"

namespace mi {
namespace {

template <int NT>
cudaError_t launch_gemm(int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, float* C,
                        int ldc, unsigned int* err, cudaStream_t st) {
    const size_t sm = tc::gemm_smem<NT>();
    cudaError_t e = cudaFuncSetAttribute(tc::k_gemm_tn<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    dim3 grid((M + tc::TILE_M - 1) / tc::TILE_M, (N + NT - 1) / NT);
    tc::k_gemm_tn<NT><<<grid, tc::THREADS, sm, st>>>(M, N, K, A, lda, B, ldb, C, ldc, err);
    return cudaGetLastError();
}

}  // namespace

// C[M×N] = A[M×K]·B[N×K]ᵀ on the stream; the N tile follows N.
cudaError_t gemm_bf16_tn(int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb,
                         float* C, int ldc, unsigned int* err, cudaStream_t st) {
    if (N <= 16) return launch_gemm<16>(M, N, K, A, lda, B, ldb, C, ldc, err, st);
    if (N <= 32) return launch_gemm<32>(M, N, K, A, lda, B, ldb, C, ldc, err, st);
    if (N <= 64) return launch_gemm<64>(M, N, K, A, lda, B, ldb, C, ldc, err, st);
    return launch_gemm<128>(M, N, K, A, lda, B, ldb, C, ldc, err, st);
}

}  // namespace mi

extern "C" {

mi_status mi_gemm_bf16_tn(mi_context* ctx, int M, int N, int K, const void* A, int lda, const void* B, int ldb,
                          float* C, int ldc) {
    if (!ctx || M < 1 || N < 1 || K < 1 || !A || !B || !C || lda < K || ldb < K || ldc < N)
        return MI_ERR_INVALID_ARGUMENT;
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    unsigned int* err = nullptr;
    MI_CHECK_CUDA(ctx, cudaMalloc(&err, sizeof(unsigned int)));
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(unsigned int), ctx->stream);
    if (e == cudaSuccess)
        e = mi::gemm_bf16_tn(M, N, K, static_cast<const __nv_bfloat16*>(A), lda, static_cast<const __nv_bfloat16*>(B),
                             ldb, C, ldc, err, ctx->stream);
    unsigned int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(err);
    if (e != cudaSuccess) return mi::cuda_status(ctx, e, "mi_gemm_bf16_tn");
    if (h) return mi::set_error(ctx, MI_ERR_TIMEOUT, "tensor-core GEMM: an mbarrier wait gave up");
    return MI_OK;
}

}  // extern "C"
