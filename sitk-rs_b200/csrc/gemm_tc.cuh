// BF16 × BF16 → FP32 GEMM on the 5th-generation tensor cores (tcgen05), for the
// learned initialiser's convolution-as-GEMM layers:
//
//     C[M×N] = A[M×K] · B[N×K]ᵀ     (A and B row-major with K contiguous: "TN")
//
// One CTA of 128 threads computes a 128 × NT tile of C. Per K step of 64 the threads
// copy the A and B tiles into shared memory in the canonical K-major, no-swizzle
// layout (8-row × 16-byte core matrices: core (row group r, k chunk c) at
// (8r + c)·128 bytes, so the leading-dimension offset between k chunks is 128 B and
// the stride between row groups 1024 B), fence them for the async proxy, and one
// thread issues four tcgen05.mma (K = 16 each) accumulating in tensor memory (128
// lanes × NT FP32 columns) and commits them to an mbarrier that every thread waits on
// — with a bounded number of polls — before the tiles are overwritten. The epilogue
// reads the accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31) and
// stores FP32 C. Out-of-range rows, columns and k are zero-filled, so M, N and K are
// arbitrary. Descriptor formats follow the PTX ISA (tcgen05 shared-memory matrix
// descriptor and kind::f16 instruction descriptor).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mi {
namespace tc {

constexpr int TILE_M = 128;
constexpr int TILE_K = 64;
constexpr int THREADS = 128;
constexpr unsigned int WAIT_POLLS = 1u << 26;  // mbarrier polls before giving up

// shared-memory matrix descriptor: start >> 4, LBO >> 4 at 16, SBO >> 4 at 32,
// version 1 at 46, no swizzle (layout type 0 at 61)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D FP32 (bits 4-5 = 1), A BF16 (bits 7-9 = 1),
// B BF16 (bits 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
__host__ __device__ constexpr uint32_t instr_desc(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Copies rows [r0, r0 + rows) × k [k0, k0 + 64) of a row-major bf16 matrix (leading
// dimension ld, valid extent nrows × K) into the core-matrix layout at `tile`.
template <int ROWS>
__device__ __forceinline__ void load_tile(const __nv_bfloat16* __restrict__ g, int ld, int nrows, int K, int r0, int k0,
                                          uint8_t* tile) {
    constexpr int CHUNKS = ROWS * (TILE_K / 8);
    const bool vec_ok = (ld % 8) == 0 && (((uintptr_t)g) & 15) == 0;
#pragma unroll 4
    for (int q = threadIdx.x; q < CHUNKS; q += THREADS) {
        const int row = q >> 3, c = q & 7;
        const int gr = r0 + row, gk = k0 + c * 8;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (gr < nrows) {
            const __nv_bfloat16* src = g + (size_t)gr * ld + gk;
            if (vec_ok && gk + 8 <= K) {
                v = *reinterpret_cast<const uint4*>(src);
            } else {
                unsigned short e[8];
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    e[j] = gk + j < K ? __bfloat16_as_ushort(src[j]) : (unsigned short)0;
                v.x = e[0] | ((uint32_t)e[1] << 16);
                v.y = e[2] | ((uint32_t)e[3] << 16);
                v.z = e[4] | ((uint32_t)e[5] << 16);
                v.w = e[6] | ((uint32_t)e[7] << 16);
            }
        }
        const int off = (((row >> 3) * 8 + c) << 7) + ((row & 7) << 4);
        *reinterpret_cast<uint4*>(tile + off) = v;
    }
}

template <int NT>
__global__ void __launch_bounds__(THREADS)
k_gemm_tn(int M, int N, int K, const __nv_bfloat16* __restrict__ A, int lda, const __nv_bfloat16* __restrict__ B,
          int ldb, float* __restrict__ C, int ldc, unsigned int* __restrict__ err) {
    static_assert(NT >= 16 && NT <= 256 && NT % 16 == 0, "N tile");
    constexpr uint32_t COLS = NT <= 32 ? 32 : (NT <= 64 ? 64 : (NT <= 128 ? 128 : 256));
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* As = smem;                         // 128 × 64 bf16 = 16 KB
    uint8_t* Bs = smem + TILE_M * TILE_K * 2;   // NT × 64 bf16
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * TILE_M, n0 = blockIdx.y * NT;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = instr_desc(TILE_M, NT);
    const uint32_t a_addr = smem_u32(As), b_addr = smem_u32(Bs);
    uint32_t phase = 0;
    bool ok = true;

    // split K: slice blockIdx.z of gridDim.z covers k tiles [kt0, kt1) and writes its
    // partial product to the blockIdx.z-th M × ldc block of C
    const int ktiles = (K + TILE_K - 1) / TILE_K;
    const int per = (ktiles + (int)gridDim.z - 1) / (int)gridDim.z;
    const int kt0 = (int)blockIdx.z * per, kt1 = min(ktiles, kt0 + per);
    C += (size_t)blockIdx.z * (size_t)M * (size_t)ldc;
    for (int kt = kt0; kt < kt1 && ok; ++kt) {  // `ok` is uniform over the CTA
        load_tile<TILE_M>(A, lda, M, K, m0, kt * TILE_K, As);
        load_tile<NT>(B, ldb, N, K, n0, kt * TILE_K, Bs);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int s = 0; s < TILE_K / 16; ++s) {
                // k step s reads k chunks 2s and 2s + 1: 256 bytes further per step
                const uint64_t ad = smem_desc(a_addr + s * 256, 128, 1024);
                const uint64_t bd = smem_desc(b_addr + s * 256, 128, 1024);
                const uint32_t acc = (kt > kt0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
                    "}" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&mbar))
                         : "memory");
        }
        // the tiles may be overwritten only once the MMAs that read them are done
        uint32_t done = 0;
        for (unsigned int polls = 0; polls < WAIT_POLLS; ++polls) {
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.b32 %0, 1, 0, p;\n\t"
                "}"
                : "=r"(done)
                : "r"(smem_u32(&mbar)), "r"(phase)
                : "memory");
            if (done) break;
        }
        // a CTA-wide decision, so every thread leaves the loop (or not) together
        ok = __syncthreads_and(done != 0) != 0;
        if (!ok && threadIdx.x == 0) atomicOr(err, 1u);
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }

    if (ok) {
        // epilogue: warp w reads TMEM lanes 32w..32w+31 (rows m0 + 32w + lane)
        const int row = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < NT; c0 += 8) {
            uint32_t r[8];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int col = n0 + c0 + j;
                    // an empty K slice wrote no accumulator: its partial product is 0
                    if (col < N) C[(size_t)row * ldc + col] = kt1 > kt0 ? __uint_as_float(r[j]) : 0.0f;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(COLS));
}

template <int NT>
constexpr size_t gemm_smem() {
    return (size_t)(TILE_M + NT) * TILE_K * 2;
}

}  // namespace tc
}  // namespace mi
