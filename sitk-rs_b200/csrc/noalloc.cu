// Mattes value for callers that cannot allocate device memory.
//
// Some callers of this library may not call cudaMalloc at all: an application that
// embeds the metric and hands it a fixed device-memory budget up front (it owns every
// buffer, and a library that allocates on its own breaks that accounting), or a
// real-time loop that must not reach the allocator (cudaMalloc and cudaFree may
// synchronise the device and take milliseconds). mi_metric_value_noalloc serves them.
// It evaluates the metric value over device buffers the caller owns, and its only
// scratch — the joint histogram the passes accumulate into, plus one word that counts
// rejected sample indices — lives in one file-scope `static __device__` array of a
// fixed size (MI_NOALLOC_MAX_BINS bins), which every GPU that loads the library holds
// until the process exits.
//
// The array is shared by every call on a device and keeps the last call's contents,
// so each call clears it on its own stream before use; two calls whose work overlaps
// on the GPU (different streams, or different host threads on one stream without
// ordering) race on it and must be serialised by the caller.
//
// The caller's sample list lives in device memory, so the host cannot check it: the
// histogram pass skips every index at or beyond the fixed grid's voxel count (it
// reads neither the fixed volume nor the moving volume for it) and counts it, and the
// tail then reports the call as failed through the result (value NaN, valid count
// minus the number of rejected indices).
//
// The histogram pass here decides every sample with the exact FP64 chain of
// sampler.cuh (exact_index / exact_value) and reads the fixed value directly, so it
// needs neither the moving volume's texture nor the per-sample fixed bins that the
// metric object builds at creation.

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <mutex>

#include "internal.h"
#include "sampler.cuh"

namespace mi {
void index_to_physical(const mi_geometry& g, double* m);
bool invert3(const double* m, double* inv);
}  // namespace mi

namespace {

constexpr int NA_BLOCK = 256;
constexpr int NA_SCRATCH = MI_NOALLOC_MAX_BINS * MI_NOALLOC_MAX_BINS + MI_NOALLOC_MAX_BINS + 1;

// The scratch: joint histogram (B² taps in 2^-k fixed point), the fixed marginal
// (B counts), then the count of rejected sample indices, u64.
static __device__ __align__(256) unsigned long long g_noalloc_hist[NA_SCRATCH];

// Device address of g_noalloc_hist per device, looked up once per device with that
// device current (a host reference to the symbol is only a host-side stand-in). The
// address belongs to the device's primary context: after cudaDeviceReset the module
// is loaded again and this cached address is stale, so a process that resets a device
// must not call mi_metric_value_noalloc on it afterwards.
std::mutex g_setup_mutex;
unsigned long long* g_hist_addr[256] = {};

mi_status scratch_address(mi_context* ctx, unsigned long long** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (ctx->device < 0 || ctx->device >= 256) return MI_ERR_INVALID_ARGUMENT;
    if (!g_hist_addr[ctx->device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_hist);
        if (e != cudaSuccess) return mi::cuda_status(ctx, e, "cudaGetSymbolAddress(g_noalloc_hist)");
        g_hist_addr[ctx->device] = static_cast<unsigned long long*>(p);
    }
    *out = g_hist_addr[ctx->device];
    return MI_OK;
}

__global__ void __launch_bounds__(NA_BLOCK)
k_noalloc_hist(mi::SamplerParams P, const float* __restrict__ fixed, const float* __restrict__ moving,
               const uint32_t* __restrict__ samples, uint32_t n, uint32_t nvox, float hist_scale,
               unsigned long long* __restrict__ hist) {
    extern __shared__ unsigned int nsh[];
    const int B = P.bins;
    const int nb = B * B + B;
    // the shared histogram, then the CTA's count of rejected indices
    for (int i = threadIdx.x; i <= nb; i += blockDim.x) nsh[i] = 0u;
    __syncthreads();
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
        const uint32_t flat = samples ? samples[s] : s;
        if (flat >= nvox) {
            // not a voxel of the fixed grid: neither volume is read for it
            atomicAdd(nsh + nb, 1u);
            continue;
        }
        uint32_t i, j, k;
        mi::grid_index(P, flat, i, j, k);
        double c[3];
        mi::exact_index(P, i, j, k, c);
        bool inside = true;
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (!(c[d] >= -0.5 && c[d] < P.mhi[d])) inside = false;
        if (!inside) continue;
        const double mv = mi::exact_value(P, c, moving);
        if (mv < P.moving_min || mv > P.moving_max) continue;
        const double term = __dsub_rn(__ddiv_rn(mv, P.moving_bin_size), P.moving_nmin);
        const int mi_ = mi::parzen_bin(term, B);
        const int fi = mi::fixed_bin(P, fixed[flat]);
        float w[4];
        mi::bspline3_taps((float)(term - (double)mi_), w);
        unsigned int* row = nsh + fi * B + (mi_ - 1);
#pragma unroll
        for (int t = 0; t < 4; ++t)
            atomicAdd(row + t, __float_as_uint(fmaf(w[t], hist_scale, 12582912.0f)) - 0x4B400000u);
        atomicAdd(nsh + B * B + fi, 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= nb; i += blockDim.x) {
        const unsigned int v = nsh[i];
        if (v) atomicAdd(hist + i, (unsigned long long)v);
    }
}

__device__ double na_block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (warp == 0) {
        r = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
#pragma unroll
        for (int off = 16; off; off >>= 1) r += __shfl_down_sync(0xffffffffu, r, off);
        if (lane == 0) red[0] = r;
    }
    __syncthreads();
    r = red[0];
    __syncthreads();
    return r;
}

// −MI from the finished histogram (registration/mattes.rs:273-328) into result[0],
// the valid count into result[1]; NaN and minus the number of rejected sample indices
// when the pass skipped any.
__global__ void __launch_bounds__(NA_BLOCK)
k_noalloc_tail(int B, double moving_bin_size, double hist_inv, const unsigned long long* __restrict__ hist,
               double* __restrict__ result) {
    __shared__ double jp[MI_NOALLOC_MAX_BINS * MI_NOALLOC_MAX_BINS];
    __shared__ double fm[MI_NOALLOC_MAX_BINS], mm[MI_NOALLOC_MAX_BINS], lfm[MI_NOALLOC_MAX_BINS];
    __shared__ double red[32];
    const int B2 = B * B;
    const unsigned long long rejected = hist[B2 + B];
    if (rejected) {
        if (threadIdx.x == 0) {
            result[0] = __longlong_as_double(0x7ff8000000000000ll);
            result[1] = -(double)rejected;
        }
        return;
    }
    double part = 0.0, cnt = 0.0;
    for (int i = threadIdx.x; i < B2; i += blockDim.x) {
        jp[i] = (double)hist[i] * hist_inv;
        part += jp[i];
    }
    for (int i = threadIdx.x; i < B; i += blockDim.x) {
        fm[i] = (double)hist[B2 + i];
        cnt += fm[i];
    }
    const double joint_sum = na_block_sum(part, red);
    const double valid = na_block_sum(cnt, red);
    if (valid == 0.0 || joint_sum < DBL_EPSILON) {
        if (threadIdx.x == 0) {
            result[0] = DBL_MAX;
            result[1] = valid;
        }
        return;
    }
    const double inv_sum = 1.0 / joint_sum;
    for (int i = threadIdx.x; i < B2; i += blockDim.x) jp[i] *= inv_sum;
    for (int i = threadIdx.x; i < B; i += blockDim.x) {
        fm[i] *= inv_sum;
        lfm[i] = fm[i] > DBL_EPSILON ? log(fm[i]) : 0.0;
    }
    __syncthreads();
    for (int m = threadIdx.x; m < B; m += blockDim.x) {
        double acc = 0.0;
        for (int f = 0; f < B; ++f) acc += jp[f * B + m];
        mm[m] = acc;
    }
    __syncthreads();
    double sum = 0.0;
    for (int i = threadIdx.x; i < B2; i += blockDim.x) {
        const int f = i / B, m = i - f * B;
        if (fm[f] > DBL_EPSILON && mm[m] > DBL_EPSILON && jp[i] > DBL_EPSILON)
            sum += jp[i] * (log(jp[i] / mm[m]) - lfm[f]);
    }
    const double total = na_block_sum(sum, red);
    if (threadIdx.x == 0) {
        result[0] = -total;
        result[1] = valid;
    }
}

}  // namespace

extern "C" mi_status mi_metric_value_noalloc(mi_context* ctx, const float* fixed, const mi_geometry* fixed_geometry,
                                             const float* moving, const mi_geometry* moving_geometry,
                                             const uint32_t* samples, int64_t n_samples, const mi_metric_info* info,
                                             const double* stages, int nstage, double* result) {
    using namespace mi;
    if (!ctx || !fixed || !fixed_geometry || !moving || !moving_geometry || !info || !result)
        return MI_ERR_INVALID_ARGUMENT;
    if (nstage < 1 || nstage > MI_MAX_STAGES)
        return set_error(ctx, MI_ERR_POINT_MAP_STAGE_COUNT,
                         "the device replays 1 to " + std::to_string(MI_MAX_STAGES) + " point-map stages");
    if (!stages) return MI_ERR_INVALID_ARGUMENT;
    const int B = info->bins;
    if (B < 2 * PADDING + 1) return set_error(ctx, MI_ERR_TOO_FEW_HISTOGRAM_BINS, "need at least 5 histogram bins");
    if (B > MI_NOALLOC_MAX_BINS)
        return set_error(ctx, MI_ERR_TOO_MANY_HISTOGRAM_BINS,
                         "the allocation-free path's fixed scratch holds at most " +
                             std::to_string(MI_NOALLOC_MAX_BINS) + " histogram bins");
    for (int d = 0; d < 3; ++d)
        if (fixed_geometry->size[d] <= 0 || moving_geometry->size[d] <= 0)
            return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "bad geometry");
    const int64_t nvox = fixed_geometry->size[0] * fixed_geometry->size[1] * fixed_geometry->size[2];
    const int64_t mvox = moving_geometry->size[0] * moving_geometry->size[1] * moving_geometry->size[2];
    if (nvox >= ((int64_t)1 << 31) || mvox >= ((int64_t)1 << 32))
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "volume too large");
    const int64_t n = samples ? n_samples : nvox;
    if (n < 0 || n >= ((int64_t)1 << 31)) return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "bad sample count");
    if (!(info->fixed_bin_size > 0.0) || !(info->moving_bin_size > 0.0))
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "bad histogram geometry");
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    unsigned long long* hist = nullptr;
    mi_status s = scratch_address(ctx, &hist);
    if (s != MI_OK) return s;

    SamplerParams P;
    std::memset(&P, 0, sizeof(P));
    double f_i2p[9], m_i2p[9], m_p2i[9];
    index_to_physical(*fixed_geometry, f_i2p);
    index_to_physical(*moving_geometry, m_i2p);
    if (!invert3(m_i2p, m_p2i)) return set_error(ctx, MI_ERR_SINGULAR_DIRECTION, "moving direction is singular");
    P.fsize0 = fixed_geometry->size[0];
    P.fsize1 = fixed_geometry->size[1];
    P.fsize2 = fixed_geometry->size[2];
    P.div0 = make_fastdiv((uint32_t)P.fsize0);
    P.div1 = make_fastdiv((uint32_t)P.fsize1);
    for (int i = 0; i < 3; ++i) P.forigin[i] = fixed_geometry->origin[i];
    for (int i = 0; i < 9; ++i) P.fi2p[i] = f_i2p[i];
    P.nstage = nstage;
    for (int st = 0; st < nstage; ++st)
        for (int i = 0; i < 12; ++i) P.stage[st][i] = stages[st * 12 + i];
    for (int d = 0; d < 3; ++d) {
        P.msize[d] = moving_geometry->size[d];
        P.morigin[d] = moving_geometry->origin[d];
        P.mhi[d] = (double)moving_geometry->size[d] - 0.5;
    }
    P.mstride1 = moving_geometry->size[0];
    P.mstride2 = moving_geometry->size[0] * moving_geometry->size[1];
    for (int i = 0; i < 9; ++i) P.mp2i[i] = m_p2i[i];
    P.bins = B;
    P.fixed_bin_size = info->fixed_bin_size;
    P.moving_bin_size = info->moving_bin_size;
    P.fixed_nmin = info->fixed_normalized_min;
    P.moving_nmin = info->moving_normalized_min;
    P.moving_min = info->moving_min;
    P.moving_max = info->moving_max;

    int sms = ctx->num_sms > 0 ? ctx->num_sms : 1;
    int64_t want = (n + NA_BLOCK - 1) / NA_BLOCK;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * 4));
    // fixed-point scale: a CTA adds at most ceil(n / (grid·block))·block samples
    const double cta_max =
        (double)std::max<int64_t>(1, ((n + (int64_t)grid * NA_BLOCK - 1) / ((int64_t)grid * NA_BLOCK)) * NA_BLOCK);
    int kbits = 22;
    while (kbits > 0 && std::ldexp(1.0, kbits) * (2.0 / 3.0) * cta_max + cta_max >= 4294967295.0 * 0.98) --kbits;
    cudaStream_t st = ctx->stream;
    // the histogram, the marginal and the rejected-index count start at zero
    MI_CHECK_CUDA(ctx, cudaMemsetAsync(hist, 0, (size_t)(B * B + B + 1) * sizeof(unsigned long long), st));
    k_noalloc_hist<<<grid, NA_BLOCK, (size_t)(B * B + B + 1) * sizeof(unsigned int), st>>>(
        P, fixed, moving, samples, (uint32_t)n, (uint32_t)nvox, (float)std::ldexp(1.0, kbits), hist);
    k_noalloc_tail<<<1, NA_BLOCK, 0, st>>>(B, P.moving_bin_size, std::ldexp(1.0, -kbits), hist, result);
    MI_CHECK_CUDA(ctx, cudaGetLastError());
    return MI_OK;
}
