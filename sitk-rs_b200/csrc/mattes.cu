// Mattes mutual information on the device: metric set-up and the per-evaluation
// kernels.
//
// One evaluation (DeviceMattesMetric::evaluate, registration/device.rs:767-800) is
//   k_hist   pass 1: sampler → Parzen joint histogram in shared memory (per CTA,
//            2^-32 fixed point in u64, so every add is exact and the result does
//            not depend on the order), flushed into a global u64 histogram
//   k_tail   one CTA: normalisation, marginals, −MI, pRatio·nFactor table
//            (registration/mattes.rs:273-328)
//   k_deriv  pass 2: sampler with gradient → 12 moments A[d] = Σ w g_d,
//            B[d][e] = Σ w g_d (x_e − x_ref,e) with w = Σ_taps B₃′·pRatio
//            (cuda/ops/mattes.rs:319-381 is the reference's form), per-CTA partials
//            in a fixed shuffle/tree order; the last CTA to finish folds the partials
//            in CTA order and contracts them with the transform's Jacobian form
//            (registration/cuda.rs:505-524)
// and one 8·(2+P)-byte copy back. Every reduction order is a function of the
// launch shape alone, so repeated evaluations are bit-identical.

#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "internal.h"
#include "sampler.cuh"

namespace mi {

// Host geometry helpers (geometry.cpp, compiled without FP contraction).
void index_to_physical(const mi_geometry& g, double* m);
bool invert3(const double* m, double* inv);

namespace {

constexpr double FIX_SCALE = 4294967296.0;        // 2^32
constexpr double FIX_INV = 1.0 / 4294967296.0;    // 2^-32
constexpr int HIST_BLOCK = 256;
constexpr int DERIV_BLOCK = 256;
constexpr int TAIL_BLOCK = 1024;
constexpr int NMOM = 12;

struct JacobianForm {
    int nparams;
    double jac0[3 * MI_MAX_PARAMS];
    double jacc[3][3 * MI_MAX_PARAMS];
};

// ---------------------------------------------------------------------------
// Pass 1: joint histogram.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(HIST_BLOCK)
k_hist(SamplerParams P, const float* __restrict__ fixed, const float* __restrict__ moving,
       const uint8_t* __restrict__ mmask, const uint32_t* __restrict__ samples, int64_t n,
       unsigned long long* __restrict__ ghist) {
    extern __shared__ unsigned long long sh[];
    const int B = P.bins;
    const int nb = B * B + B;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) sh[i] = 0ull;
    __syncthreads();
    unsigned long long* sh_joint = sh;
    unsigned long long* sh_fixed = sh + B * B;
    unsigned int valid = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
        const uint32_t flat = samples ? __ldg(samples + s) : (uint32_t)s;
        Sample o;
        if (take_sample<false>(P, flat, fixed, moving, mmask, o) != SAMPLE_VALID) continue;
        ++valid;
        atomicAdd(&sh_fixed[o.fi], 1ull);
        unsigned long long* row = sh_joint + o.fi * B;
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int m = o.mi - 1 + t;
            const double w = bspline3((double)m - o.mterm);
            const unsigned long long q = __double2ull_rn(w * FIX_SCALE);
            if (q) atomicAdd(&row[m], q);
        }
    }
    // valid count: one atomic per warp
    unsigned int wv = valid;
#pragma unroll
    for (int off = 16; off; off >>= 1) wv += __shfl_down_sync(0xffffffffu, wv, off);
    __syncthreads();
    if ((threadIdx.x & 31) == 0 && wv) atomicAdd(&ghist[nb], (unsigned long long)wv);
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        const unsigned long long v = sh[i];
        if (v) atomicAdd(&ghist[i], v);
    }
}

// Block-wide sum of a double in a fixed order (warp shuffles, then warp 0).
__device__ double block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    double r = 0.0;
    if (warp == 0) {
        r = lane < nw ? red[lane] : 0.0;
#pragma unroll
        for (int off = 16; off; off >>= 1) r += __shfl_down_sync(0xffffffffu, r, off);
        if (lane == 0) red[0] = r;
    }
    __syncthreads();
    r = red[0];
    __syncthreads();
    return r;
}

// ---------------------------------------------------------------------------
// Tail: normalise, marginals, −MI, pRatio (registration/mattes.rs:273-328).
// tail[0] value, tail[1] valid, tail[2] degenerate flag, tail[3] joint sum;
// result[0..1] receive value and valid for the value-only path.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(TAIL_BLOCK)
k_tail(int B, double moving_bin_size, const unsigned long long* __restrict__ ghist,
       double* __restrict__ pratio, double* __restrict__ tail, double* __restrict__ result) {
    extern __shared__ double tsh[];
    double* jp = tsh;              // B*B
    double* fm = jp + B * B;       // B
    double* mm = fm + B;           // B
    double* lfm = mm + B;          // B
    double* red = lfm + B;         // 32
    const int B2 = B * B;
    const unsigned long long valid = ghist[B2 + B];
    double part = 0.0;
    for (int i = threadIdx.x; i < B2; i += blockDim.x) {
        const double v = (double)ghist[i] * FIX_INV;
        jp[i] = v;
        part += v;
    }
    for (int i = threadIdx.x; i < B; i += blockDim.x) fm[i] = (double)ghist[B2 + i];
    const double joint_sum = block_sum(part, red);
    if (valid == 0 || joint_sum < DBL_EPSILON) {
        // degenerate histogram (mattes.rs:590-609): value f64::MAX, zero derivative
        if (threadIdx.x == 0) {
            tail[0] = DBL_MAX;
            tail[1] = (double)valid;
            tail[2] = 1.0;
            tail[3] = joint_sum;
            result[0] = DBL_MAX;
            result[1] = (double)valid;
        }
        return;
    }
    const double n_factor = 1.0 / (moving_bin_size * (double)valid);
    const double inv_sum = 1.0 / joint_sum;
    for (int i = threadIdx.x; i < B2; i += blockDim.x) jp[i] *= inv_sum;
    for (int i = threadIdx.x; i < B; i += blockDim.x) {
        const double f = fm[i] * inv_sum;
        fm[i] = f;
        lfm[i] = f > DBL_EPSILON ? log(f) : 0.0;
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
        const double p = jp[i], mmv = mm[m];
        double r = 0.0;
        if (fm[f] > DBL_EPSILON && mmv > DBL_EPSILON && p > DBL_EPSILON) {
            const double lr = log(p / mmv);
            sum += p * (lr - lfm[f]);
            r = lr * n_factor;
        }
        pratio[i] = r;
    }
    const double total = block_sum(sum, red);
    if (threadIdx.x == 0) {
        tail[0] = -total;
        tail[1] = (double)valid;
        tail[2] = 0.0;
        tail[3] = joint_sum;
        result[0] = -total;
        result[1] = (double)valid;
    }
}

// ---------------------------------------------------------------------------
// Pass 2: derivative moments, with the last CTA folding and contracting.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(DERIV_BLOCK)
k_deriv(SamplerParams P, JacobianForm J, const float* __restrict__ fixed,
        const float* __restrict__ moving, const uint8_t* __restrict__ mmask,
        const uint32_t* __restrict__ samples, int64_t n, const double* __restrict__ pratio_g,
        const double* __restrict__ tail, double* __restrict__ partials,
        unsigned int* __restrict__ done_counter, double* __restrict__ result) {
    extern __shared__ double dsh[];
    const int B = P.bins;
    double* pr = dsh;                 // B*B
    double* red = dsh + B * B;        // 32 * NMOM
    __shared__ bool is_last;
    const bool degenerate = tail[2] != 0.0;
    double acc[NMOM];
#pragma unroll
    for (int i = 0; i < NMOM; ++i) acc[i] = 0.0;
    if (!degenerate) {
        for (int i = threadIdx.x; i < B * B; i += blockDim.x) pr[i] = pratio_g[i];
        __syncthreads();
        const int64_t stride = (int64_t)gridDim.x * blockDim.x;
        for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
            const uint32_t flat = samples ? __ldg(samples + s) : (uint32_t)s;
            Sample o;
            if (take_sample<true>(P, flat, fixed, moving, mmask, o) != SAMPLE_VALID) continue;
            const double* row = pr + o.fi * B;
            double w = 0.0;
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int m = o.mi - 1 + t;
                w += bspline3_deriv((double)m - o.mterm) * row[m];
            }
            if (w == 0.0) continue;
            const double dx0 = o.x[0] - P.xref[0], dx1 = o.x[1] - P.xref[1], dx2 = o.x[2] - P.xref[2];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double wg = w * o.g[d];
                acc[d] += wg;
                acc[3 + d * 3 + 0] += wg * dx0;
                acc[3 + d * 3 + 1] += wg * dx1;
                acc[3 + d * 3 + 2] += wg * dx2;
            }
        }
    }
    // CTA reduction in a fixed order: shuffles within a warp, then warp 0 over warps.
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int i = 0; i < NMOM; ++i) {
        double v = acc[i];
#pragma unroll
        for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        acc[i] = v;
    }
    if (lane == 0)
        for (int i = 0; i < NMOM; ++i) red[warp * NMOM + i] = acc[i];
    __syncthreads();
    if (threadIdx.x < NMOM) {
        double v = 0.0;
        for (int w = 0; w < nw; ++w) v += red[w * NMOM + threadIdx.x];
        partials[(int64_t)blockIdx.x * NMOM + threadIdx.x] = v;
    }
    // Last CTA to arrive folds every CTA's partials in CTA order (no waiting).
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(done_counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    __shared__ double mom[NMOM];
    if (threadIdx.x < NMOM) {
        double v = 0.0;
        for (unsigned int b = 0; b < gridDim.x; ++b)
            v += __ldcg(partials + (int64_t)b * NMOM + threadIdx.x);
        mom[threadIdx.x] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) *done_counter = 0u;
    // Contract: ∂/∂p_k = Σ_d J(x_ref)[d][k]·A_d + Σ_{d,e} C_e[d][k]·B[d][e],
    // with J(x_ref) = J(0) + Σ_e x_ref,e·C_e.
    const int np = J.nparams;
    if (threadIdx.x < np) {
        const int k = threadIdx.x;
        double dk = 0.0;
        if (!degenerate) {
            for (int d = 0; d < 3; ++d) {
                double jr = J.jac0[d * np + k];
                for (int e = 0; e < 3; ++e) jr += P.xref[e] * J.jacc[e][d * np + k];
                dk += jr * mom[d];
                for (int e = 0; e < 3; ++e) dk += J.jacc[e][d * np + k] * mom[3 + d * 3 + e];
            }
        }
        result[2 + k] = dk;
    }
    if (threadIdx.x == 0) {
        result[0] = tail[0];
        result[1] = tail[1];
    }
}

// Per-sample decisions, for the exactness tests.
__global__ void k_decisions(SamplerParams P, const float* __restrict__ fixed,
                            const float* __restrict__ moving, const uint8_t* __restrict__ mmask,
                            const uint32_t* __restrict__ samples, int64_t n,
                            int8_t* __restrict__ status, int32_t* __restrict__ fbin,
                            int32_t* __restrict__ mbin, int64_t* __restrict__ flat_out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
        const uint32_t flat = samples ? samples[s] : (uint32_t)s;
        Sample o;
        const int st = take_sample<false>(P, flat, fixed, moving, mmask, o);
        if (status) status[s] = (int8_t)st;
        if (fbin) fbin[s] = st == SAMPLE_VALID ? o.fi : -1;
        if (mbin) mbin[s] = st == SAMPLE_VALID ? o.mi : -1;
        if (flat_out) flat_out[s] = flat;
    }
}

// ---------------------------------------------------------------------------
// Set-up kernels: the draw, the fixed-mask gate, and the intensity ranges.
// ---------------------------------------------------------------------------
__global__ void k_draw_random(uint64_t seed, uint64_t voxels, int64_t count, uint32_t* out) {
    // SplitMix64 (registration/metric.rs:101-122): the i-th output follows
    // i+1 advances of the state, so draw i is mix(seed + (i+1)·γ) mod voxels.
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        uint64_t z = seed + (uint64_t)(i + 1) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        out[i] = (uint32_t)(z % voxels);
    }
}

__global__ void k_iota_stride(int64_t count, uint64_t stride_v, uint32_t* out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
        out[i] = (uint32_t)((uint64_t)i * stride_v);
}

__global__ void k_mask_flags(const uint32_t* __restrict__ idx, int64_t count,
                             const float* __restrict__ fmask, uint8_t* __restrict__ flags) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
        flags[i] = fmask[idx[i]] != 0.0f ? 1 : 0;
}

// min/max over the selected fixed samples (or all voxels) and over the moving voxels
// the moving mask admits; NaN is skipped like f64::min/max. Per-CTA partials.
__global__ void k_minmax(const float* __restrict__ vals, const uint32_t* __restrict__ idx,
                         const uint8_t* __restrict__ mask, int64_t n, float* __restrict__ out) {
    float lo = INFINITY, hi = -INFINITY;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int64_t j = idx ? (int64_t)idx[i] : i;
        if (mask && !mask[j]) continue;
        const float v = vals[j];
        lo = fminf(lo, v);
        hi = fmaxf(hi, v);
    }
    __shared__ float slo[32], shi[32];
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        lo = fminf(lo, __shfl_down_sync(0xffffffffu, lo, off));
        hi = fmaxf(hi, __shfl_down_sync(0xffffffffu, hi, off));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { slo[warp] = lo; shi[warp] = hi; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            lo = fminf(lo, slo[w]);
            hi = fmaxf(hi, shi[w]);
        }
        out[blockIdx.x * 2] = lo;
        out[blockIdx.x * 2 + 1] = hi;
    }
}

int grid_for(int64_t n, int block, int cap) {
    int64_t g = (n + block - 1) / block;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

mi_status minmax(mi_context* ctx, const float* vals, const uint32_t* idx, const uint8_t* mask,
                 int64_t n, double* lo, double* hi, bool* any) {
    const int block = 256;
    const int grid = grid_for(n, block, ctx->num_sms * 4);
    float* d = nullptr;
    MI_CHECK_CUDA(ctx, cudaMalloc(&d, (size_t)grid * 2 * sizeof(float)));
    k_minmax<<<grid, block, 0, ctx->stream>>>(vals, idx, mask, n, d);
    std::vector<float> h((size_t)grid * 2);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d, h.size() * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_status(ctx, e, "minmax");
    float l = INFINITY, u = -INFINITY;
    for (int b = 0; b < grid; ++b) {
        l = std::fmin(l, h[b * 2]);
        u = std::fmax(u, h[b * 2 + 1]);
    }
    *any = !(l == INFINITY && u == -INFINITY);
    *lo = *any ? (double)l : 0.0;
    *hi = *any ? (double)u : 0.0;
    return MI_OK;
}

void free_metric(mi_metric* m) {
    if (!m) return;
    cudaFree(m->fixed);
    cudaFree(m->moving);
    cudaFree(m->mmask);
    cudaFree(m->samples);
    cudaFree(m->ws.hist);
    cudaFree(m->ws.pratio);
    cudaFree(m->ws.tail);
    cudaFree(m->ws.partials);
    cudaFree(m->ws.result);
    cudaFree(m->ws.done_counter);
    if (m->ws.host_result) cudaFreeHost(m->ws.host_result);
    for (int i = 0; i < 5; ++i)
        if (m->ws.ev[i]) cudaEventDestroy(m->ws.ev[i]);
    delete m;
}

size_t hist_smem(int B) { return (size_t)(B * B + B) * sizeof(unsigned long long); }
size_t tail_smem(int B) { return (size_t)(B * B + 3 * B + 32) * sizeof(double); }
size_t deriv_smem(int B) { return (size_t)(B * B + 32 * NMOM) * sizeof(double); }

// Build the sample list: the strategy's draw, gated by the fixed mask, sorted
// ascending. The histogram is a sum of exact integers and so does not depend on
// the order; sorting only buys locality.
mi_status build_samples(mi_context* ctx, mi_metric* m, const mi_image* fixed_mask,
                        const mi_sampling* smp, int64_t nvox) {
    const int strategy = smp ? smp->strategy : MI_SAMPLING_NONE;
    if (strategy == MI_SAMPLING_NONE && !fixed_mask) {
        m->samples = nullptr;
        m->n_samples = nvox;
        return MI_OK;
    }
    int64_t count = 0;
    uint32_t* draw = nullptr;
    cudaStream_t st = ctx->stream;
    const int block = 256;
    if (strategy == MI_SAMPLING_NONE) {
        count = nvox;
        MI_CHECK_CUDA(ctx, cudaMalloc(&draw, (size_t)count * 4));
        k_iota_stride<<<grid_for(count, block, ctx->num_sms * 8), block, 0, st>>>(count, 1, draw);
    } else if (strategy == MI_SAMPLING_REGULAR) {
        if (!(smp->percentage > 0.0) || !std::isfinite(smp->percentage))
            return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "sampling percentage must be positive");
        int64_t stride = (int64_t)std::ceil(1.0 / smp->percentage);
        if (stride < 1) stride = 1;
        count = (nvox + stride - 1) / stride;
        MI_CHECK_CUDA(ctx, cudaMalloc(&draw, (size_t)std::max<int64_t>(count, 1) * 4));
        k_iota_stride<<<grid_for(count, block, ctx->num_sms * 8), block, 0, st>>>(count, (uint64_t)stride, draw);
    } else if (strategy == MI_SAMPLING_RANDOM) {
        if (!(smp->percentage > 0.0) || !std::isfinite(smp->percentage))
            return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "sampling percentage must be positive");
        count = (int64_t)((double)nvox * smp->percentage);
        if (count >= ((int64_t)1 << 32))
            return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "sample count exceeds 2^32");
        MI_CHECK_CUDA(ctx, cudaMalloc(&draw, (size_t)std::max<int64_t>(count, 1) * 4));
        if (count)
            k_draw_random<<<grid_for(count, block, ctx->num_sms * 8), block, 0, st>>>(smp->seed, (uint64_t)nvox, count, draw);
    } else if (strategy == MI_SAMPLING_EXPLICIT) {
        if (smp->n_indices < 0 || (smp->n_indices > 0 && !smp->indices))
            return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "explicit sampling needs an index list");
        count = smp->n_indices;
        std::vector<uint32_t> h((size_t)count);
        for (int64_t i = 0; i < count; ++i) {
            const int64_t v = smp->indices[i];
            if (v < 0 || v >= nvox)
                return set_error(ctx, MI_ERR_SAMPLE_INDEX_OUT_OF_GRID,
                                 "sample index " + std::to_string(v) + " is outside the fixed grid of " +
                                     std::to_string(nvox) + " voxels");
            h[i] = (uint32_t)v;
        }
        MI_CHECK_CUDA(ctx, cudaMalloc(&draw, (size_t)std::max<int64_t>(count, 1) * 4));
        if (count) MI_CHECK_CUDA(ctx, cudaMemcpyAsync(draw, h.data(), (size_t)count * 4, cudaMemcpyHostToDevice, st));
        MI_CHECK_CUDA(ctx, cudaStreamSynchronize(st));
    } else {
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "unknown sampling strategy");
    }
    MI_CHECK_CUDA(ctx, cudaGetLastError());

    uint32_t* kept = draw;
    int64_t nkept = count;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    if (fixed_mask && count) {
        uint8_t* flags = nullptr;
        uint32_t* out = nullptr;
        int* nsel = nullptr;
        MI_CHECK_CUDA(ctx, cudaMalloc(&flags, (size_t)count));
        MI_CHECK_CUDA(ctx, cudaMalloc(&out, (size_t)count * 4));
        MI_CHECK_CUDA(ctx, cudaMalloc(&nsel, sizeof(int)));
        k_mask_flags<<<grid_for(count, block, ctx->num_sms * 8), block, 0, st>>>(draw, count, fixed_mask->data, flags);
        MI_CHECK_CUDA(ctx, cub::DeviceSelect::Flagged(nullptr, tmp_bytes, draw, flags, out, nsel, (int)count, st));
        MI_CHECK_CUDA(ctx, cudaMalloc(&tmp, tmp_bytes));
        MI_CHECK_CUDA(ctx, cub::DeviceSelect::Flagged(tmp, tmp_bytes, draw, flags, out, nsel, (int)count, st));
        int h = 0;
        MI_CHECK_CUDA(ctx, cudaMemcpyAsync(&h, nsel, sizeof(int), cudaMemcpyDeviceToHost, st));
        MI_CHECK_CUDA(ctx, cudaStreamSynchronize(st));
        cudaFree(tmp);
        tmp = nullptr;
        cudaFree(flags);
        cudaFree(nsel);
        cudaFree(draw);
        kept = out;
        nkept = h;
    }
    if (nkept > 1) {
        uint32_t* sorted = nullptr;
        MI_CHECK_CUDA(ctx, cudaMalloc(&sorted, (size_t)nkept * 4));
        int bits = 1;
        while (bits < 32 && ((uint64_t)1 << bits) < (uint64_t)nvox) ++bits;
        tmp_bytes = 0;
        MI_CHECK_CUDA(ctx, cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, kept, sorted, (int)nkept, 0, bits, st));
        MI_CHECK_CUDA(ctx, cudaMalloc(&tmp, tmp_bytes));
        MI_CHECK_CUDA(ctx, cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, kept, sorted, (int)nkept, 0, bits, st));
        MI_CHECK_CUDA(ctx, cudaStreamSynchronize(st));
        cudaFree(tmp);
        cudaFree(kept);
        kept = sorted;
    }
    m->samples = kept;
    m->n_samples = nkept;
    return MI_OK;
}

}  // namespace

mi_status evaluate(mi_metric* m, const double* stages, int nstage, const double* jac0,
                   const double* jacc, int nparams, bool want_derivative, double* value,
                   double* derivative, int64_t* valid) {
    mi_context* ctx = m->ctx;
    if (nstage < 0 || nstage > MI_MAX_STAGES)
        return set_error(ctx, MI_ERR_POINT_MAP_STAGE_COUNT,
                         "the device replays at most " + std::to_string(MI_MAX_STAGES) + " point-map stages");
    if (nstage > 0 && !stages) return MI_ERR_INVALID_ARGUMENT;
    if (want_derivative && (nparams < 1 || nparams > MI_MAX_PARAMS || !jac0 || !jacc || !derivative))
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "bad Jacobian form");
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    SamplerParams P = m->base;
    P.nstage = nstage;
    for (int s = 0; s < nstage; ++s)
        for (int i = 0; i < 12; ++i) P.stage[s][i] = stages[s * 12 + i];
    const int B = m->bins;
    cudaStream_t st = ctx->stream;
    Workspace& ws = m->ws;
    const bool timing = ws.timing;
    if (timing) MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[0], st));
    MI_CHECK_CUDA(ctx, cudaMemsetAsync(ws.hist, 0, (size_t)(B * B + B + 1) * 8, st));
    k_hist<<<ws.grid_hist, ws.block_hist, hist_smem(B), st>>>(P, m->fixed, m->moving, m->mmask, m->samples,
                                                              m->n_samples, ws.hist);
    if (timing) MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[1], st));
    k_tail<<<1, TAIL_BLOCK, tail_smem(B), st>>>(B, P.moving_bin_size, ws.hist, ws.pratio, ws.tail, ws.result);
    if (timing) MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[2], st));
    int nout = 2;
    if (want_derivative) {
        JacobianForm J;
        J.nparams = nparams;
        for (int i = 0; i < 3 * nparams; ++i) {
            J.jac0[i] = jac0[i];
            for (int e = 0; e < 3; ++e) J.jacc[e][i] = jacc[e * 3 * nparams + i];
        }
        k_deriv<<<ws.grid_deriv, ws.block_deriv, deriv_smem(B), st>>>(
            P, J, m->fixed, m->moving, m->mmask, m->samples, m->n_samples, ws.pratio, ws.tail,
            ws.partials, ws.done_counter, ws.result);
        nout = 2 + nparams;
    }
    if (timing) MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[3], st));
    MI_CHECK_CUDA(ctx, cudaGetLastError());
    MI_CHECK_CUDA(ctx, cudaMemcpyAsync(ws.host_result, ws.result, (size_t)nout * 8, cudaMemcpyDeviceToHost, st));
    if (timing) MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[4], st));
    MI_CHECK_CUDA(ctx, cudaStreamSynchronize(st));
    if (timing) {
        float t = 0.f;
        MI_CHECK_CUDA(ctx, cudaEventElapsedTime(&t, ws.ev[0], ws.ev[4]));
        ws.ms[0] += t;
        MI_CHECK_CUDA(ctx, cudaEventElapsedTime(&t, ws.ev[0], ws.ev[1]));
        ws.ms[1] += t;
        MI_CHECK_CUDA(ctx, cudaEventElapsedTime(&t, ws.ev[1], ws.ev[2]));
        ws.ms[2] += t;
        MI_CHECK_CUDA(ctx, cudaEventElapsedTime(&t, ws.ev[2], ws.ev[3]));
        ws.ms[3] += t;
        ws.timed_evals += 1;
    }
    if (value) *value = ws.host_result[0];
    if (valid) *valid = (int64_t)ws.host_result[1];
    if (want_derivative)
        for (int k = 0; k < nparams; ++k) derivative[k] = ws.host_result[2 + k];
    return MI_OK;
}

}  // namespace mi

extern "C" {

mi_status mi_metric_create(mi_context* ctx, const mi_image* fixed, const mi_image* moving,
                           const mi_image* fixed_mask, const uint8_t* moving_mask,
                           const mi_sampling* sampling, int bins, mi_metric** out) {
    using namespace mi;
    if (!ctx || !fixed || !moving || !out) return MI_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (fixed->ctx != ctx || moving->ctx != ctx || (fixed_mask && fixed_mask->ctx != ctx))
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "images belong to another context");
    if (bins < 2 * PADDING + 1)
        return set_error(ctx, MI_ERR_TOO_FEW_HISTOGRAM_BINS,
                         "need at least " + std::to_string(2 * PADDING + 1) + " histogram bins, got " +
                             std::to_string(bins));
    if (bins > MI_MAX_BINS)
        return set_error(ctx, MI_ERR_TOO_MANY_HISTOGRAM_BINS,
                         "the shared-memory histogram holds at most " + std::to_string(MI_MAX_BINS) + " bins");
    if (fixed_mask)
        for (int d = 0; d < 3; ++d)
            if (fixed_mask->geo.size[d] != fixed->geo.size[d])
                return set_error(ctx, MI_ERR_MASK_SIZE_MISMATCH, "fixed mask size differs from the fixed image");
    const int64_t nvox = fixed->n, mvox = moving->n;
    if (nvox >= ((int64_t)1 << 32) || mvox >= ((int64_t)1 << 40))
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "volume too large for 32-bit sample indices");
    double m_i2p[9], m_p2i[9], f_i2p[9];
    index_to_physical(moving->geo, m_i2p);
    if (!invert3(m_i2p, m_p2i)) return set_error(ctx, MI_ERR_SINGULAR_DIRECTION, "moving direction is singular");
    index_to_physical(fixed->geo, f_i2p);
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));

    mi_metric* m = new (std::nothrow) mi_metric();
    if (!m) return MI_ERR_OUT_OF_MEMORY;
    m->ctx = ctx;
    m->fgeo = fixed->geo;
    m->mgeo = moving->geo;
    m->bins = bins;
    cudaStream_t st = ctx->stream;
    auto fail = [&](mi_status s) {
        cudaStreamSynchronize(st);
        free_metric(m);
        return s;
    };
#define TRY_CUDA(expr)                                                   \
    do {                                                                 \
        cudaError_t _e = (expr);                                         \
        if (_e != cudaSuccess) return fail(cuda_status(ctx, _e, #expr)); \
    } while (0)
    TRY_CUDA(cudaMalloc(&m->fixed, (size_t)nvox * 4));
    TRY_CUDA(cudaMalloc(&m->moving, (size_t)mvox * 4));
    TRY_CUDA(cudaMemcpyAsync(m->fixed, fixed->data, (size_t)nvox * 4, cudaMemcpyDeviceToDevice, st));
    TRY_CUDA(cudaMemcpyAsync(m->moving, moving->data, (size_t)mvox * 4, cudaMemcpyDeviceToDevice, st));
    if (moving_mask) {
        TRY_CUDA(cudaMalloc(&m->mmask, (size_t)mvox));
        TRY_CUDA(cudaMemcpyAsync(m->mmask, moving_mask, (size_t)mvox, cudaMemcpyHostToDevice, st));
    }
    mi_status s = build_samples(ctx, m, fixed_mask, sampling, nvox);
    if (s != MI_OK) return fail(s);

    // Histogram geometry from the sampled fixed values and the masked moving volume
    // (metric.rs:633-640, :913-924; MattesGeometry::new, mattes.rs:152-186).
    double fmin, fmax, mmin, mmax;
    bool anyf, anym;
    s = minmax(ctx, m->fixed, m->samples, nullptr, m->n_samples, &fmin, &fmax, &anyf);
    if (s != MI_OK) return fail(s);
    s = minmax(ctx, m->moving, nullptr, m->mmask, mvox, &mmin, &mmax, &anym);
    if (s != MI_OK) return fail(s);
    if (fmax - fmin <= DBL_EPSILON) return fail(set_error(ctx, MI_ERR_CONSTANT_FIXED, "constant intensity: fixed"));
    if (mmax - mmin <= DBL_EPSILON) return fail(set_error(ctx, MI_ERR_CONSTANT_MOVING, "constant intensity: moving"));
    const double denom = (double)(bins - 2 * PADDING);
    mi_metric_info& info = m->info;
    info.bins = bins;
    info.n_samples = m->n_samples;
    info.fixed_min = fmin;
    info.fixed_max = fmax;
    info.moving_min = mmin;
    info.moving_max = mmax;
    info.fixed_bin_size = (fmax - fmin) / denom;
    info.moving_bin_size = (mmax - mmin) / denom;
    info.fixed_normalized_min = fmin / info.fixed_bin_size - (double)PADDING;
    info.moving_normalized_min = mmin / info.moving_bin_size - (double)PADDING;

    SamplerParams& P = m->base;
    std::memset(&P, 0, sizeof(P));
    P.fsize0 = fixed->geo.size[0];
    P.fsize1 = fixed->geo.size[1];
    P.fsize2 = fixed->geo.size[2];
    for (int i = 0; i < 3; ++i) P.forigin[i] = fixed->geo.origin[i];
    for (int i = 0; i < 9; ++i) P.fi2p[i] = f_i2p[i];
    for (int d = 0; d < 3; ++d) {
        P.msize[d] = moving->geo.size[d];
        P.morigin[d] = moving->geo.origin[d];
        P.mhi[d] = (double)moving->geo.size[d] - 0.5;
    }
    P.mstride1 = moving->geo.size[0];
    P.mstride2 = moving->geo.size[0] * moving->geo.size[1];
    for (int i = 0; i < 9; ++i) P.mp2i[i] = m_p2i[i];
    P.has_mmask = moving_mask ? 1 : 0;
    P.bins = bins;
    P.fixed_bin_size = info.fixed_bin_size;
    P.moving_bin_size = info.moving_bin_size;
    P.fixed_nmin = info.fixed_normalized_min;
    P.moving_nmin = info.moving_normalized_min;
    P.moving_min = mmin;
    P.moving_max = mmax;
    // x_ref: the fixed grid's physical centre.
    const double mid[3] = {0.5 * (double)(P.fsize0 - 1), 0.5 * (double)(P.fsize1 - 1), 0.5 * (double)(P.fsize2 - 1)};
    for (int r = 0; r < 3; ++r)
        P.xref[r] = P.forigin[r] + f_i2p[r * 3] * mid[0] + f_i2p[r * 3 + 1] * mid[1] + f_i2p[r * 3 + 2] * mid[2];

    // Workspace and launch shapes.
    Workspace& ws = m->ws;
    const int B = bins;
    TRY_CUDA(cudaFuncSetAttribute(k_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hist_smem(B)));
    TRY_CUDA(cudaFuncSetAttribute(k_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tail_smem(B)));
    TRY_CUDA(cudaFuncSetAttribute(k_deriv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)deriv_smem(B)));
    int occ_h = 0, occ_d = 0;
    TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_h, k_hist, HIST_BLOCK, hist_smem(B)));
    TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_d, k_deriv, DERIV_BLOCK, deriv_smem(B)));
    ws.block_hist = HIST_BLOCK;
    ws.block_deriv = DERIV_BLOCK;
    ws.grid_hist = grid_for(m->n_samples, HIST_BLOCK, ctx->num_sms * std::max(occ_h, 1));
    ws.grid_deriv = grid_for(m->n_samples, DERIV_BLOCK, ctx->num_sms * std::max(occ_d, 1));
    TRY_CUDA(cudaMalloc(&ws.hist, (size_t)(B * B + B + 1) * 8));
    TRY_CUDA(cudaMalloc(&ws.pratio, (size_t)B * B * 8));
    TRY_CUDA(cudaMalloc(&ws.tail, 4 * 8));
    TRY_CUDA(cudaMalloc(&ws.partials, (size_t)ws.grid_deriv * NMOM * 8));
    TRY_CUDA(cudaMalloc(&ws.result, (2 + MI_MAX_PARAMS) * 8));
    TRY_CUDA(cudaMalloc(&ws.done_counter, sizeof(unsigned int)));
    TRY_CUDA(cudaMemsetAsync(ws.done_counter, 0, sizeof(unsigned int), st));
    TRY_CUDA(cudaMemsetAsync(ws.result, 0, (2 + MI_MAX_PARAMS) * 8, st));
    TRY_CUDA(cudaMallocHost(&ws.host_result, (2 + MI_MAX_PARAMS) * 8));
    TRY_CUDA(cudaStreamSynchronize(st));
#undef TRY_CUDA
    *out = m;
    return MI_OK;
}

mi_status mi_metric_info_get(const mi_metric* m, mi_metric_info* out) {
    if (!m || !out) return MI_ERR_INVALID_ARGUMENT;
    *out = m->info;
    return MI_OK;
}

mi_status mi_metric_destroy(mi_metric* m) {
    if (!m) return MI_ERR_INVALID_ARGUMENT;
    cudaSetDevice(m->ctx->device);
    cudaStreamSynchronize(m->ctx->stream);
    mi::free_metric(m);
    return MI_OK;
}

mi_status mi_metric_value(mi_metric* m, const double* stages, int nstage, double* value, int64_t* valid) {
    if (!m || !value) return MI_ERR_INVALID_ARGUMENT;
    return mi::evaluate(m, stages, nstage, nullptr, nullptr, 0, false, value, nullptr, valid);
}

mi_status mi_metric_value_and_derivative(mi_metric* m, int kind, const double* params, int nparams,
                                         const double* fixed_params, int nfixed, double* value,
                                         double* derivative, int64_t* valid) {
    if (!m || !params || !value || !derivative) return MI_ERR_INVALID_ARGUMENT;
    mi::AffineForm f;
    mi_status s = mi::transform_form(kind, params, nparams, fixed_params, nfixed, &f);
    if (s != MI_OK) return mi::set_error(m->ctx, s, "bad transform kind or parameter count");
    return mi::evaluate(m, f.stage, 1, f.jac0, &f.jacc[0][0], f.nparams, true, value, derivative, valid);
}

mi_status mi_metric_value_and_derivative_stages(mi_metric* m, const double* stages, int nstage,
                                                const double* jac0, const double* jac_c, int nparams,
                                                double* value, double* derivative, int64_t* valid) {
    if (!m || !value || !derivative || !jac0 || !jac_c) return MI_ERR_INVALID_ARGUMENT;
    return mi::evaluate(m, stages, nstage, jac0, jac_c, nparams, true, value, derivative, valid);
}

mi_status mi_metric_timing_enable(mi_metric* m, int enable) {
    if (!m) return MI_ERR_INVALID_ARGUMENT;
    mi::Workspace& ws = m->ws;
    if (enable && !ws.ev[0]) {
        MI_CHECK_CUDA(m->ctx, cudaSetDevice(m->ctx->device));
        for (int i = 0; i < 5; ++i) MI_CHECK_CUDA(m->ctx, cudaEventCreate(&ws.ev[i]));
    }
    ws.timing = enable != 0;
    return MI_OK;
}

mi_status mi_metric_timing_read(mi_metric* m, double* ms4, int64_t* n_evals) {
    if (!m) return MI_ERR_INVALID_ARGUMENT;
    mi::Workspace& ws = m->ws;
    if (ms4)
        for (int i = 0; i < 4; ++i) ms4[i] = ws.ms[i];
    if (n_evals) *n_evals = ws.timed_evals;
    for (int i = 0; i < 4; ++i) ws.ms[i] = 0.0;
    ws.timed_evals = 0;
    return MI_OK;
}

mi_status mi_transform_form(int kind, const double* params, int nparams, const double* fixed_params,
                            int nfixed, double* stage12, double* jac0, double* jac_c) {
    mi::AffineForm f;
    mi_status s = mi::transform_form(kind, params, nparams, fixed_params, nfixed, &f);
    if (s != MI_OK) return s;
    if (stage12) std::memcpy(stage12, f.stage, sizeof(f.stage));
    if (jac0) std::memcpy(jac0, f.jac0, sizeof(double) * 3 * f.nparams);
    if (jac_c)
        for (int e = 0; e < 3; ++e) std::memcpy(jac_c + e * 3 * f.nparams, f.jacc[e], sizeof(double) * 3 * f.nparams);
    return MI_OK;
}

mi_status mi_metric_sample_decisions(mi_metric* m, const double* stages, int nstage, int8_t* status,
                                     int32_t* fixed_bin, int32_t* moving_bin, int64_t* flat, int64_t n) {
    using namespace mi;
    if (!m) return MI_ERR_INVALID_ARGUMENT;
    mi_context* ctx = m->ctx;
    if (n < m->n_samples) return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "output arrays shorter than the sample count");
    if (nstage < 0 || nstage > MI_MAX_STAGES) return set_error(ctx, MI_ERR_POINT_MAP_STAGE_COUNT, "too many stages");
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    SamplerParams P = m->base;
    P.nstage = nstage;
    for (int s = 0; s < nstage; ++s)
        for (int i = 0; i < 12; ++i) P.stage[s][i] = stages[s * 12 + i];
    const int64_t ns = m->n_samples;
    int8_t* d_st = nullptr;
    int32_t *d_fb = nullptr, *d_mb = nullptr;
    int64_t* d_fl = nullptr;
    cudaStream_t st = ctx->stream;
    MI_CHECK_CUDA(ctx, cudaMalloc(&d_st, (size_t)std::max<int64_t>(ns, 1)));
    MI_CHECK_CUDA(ctx, cudaMalloc(&d_fb, (size_t)std::max<int64_t>(ns, 1) * 4));
    MI_CHECK_CUDA(ctx, cudaMalloc(&d_mb, (size_t)std::max<int64_t>(ns, 1) * 4));
    MI_CHECK_CUDA(ctx, cudaMalloc(&d_fl, (size_t)std::max<int64_t>(ns, 1) * 8));
    const int block = 256;
    k_decisions<<<grid_for(ns, block, ctx->num_sms * 8), block, 0, st>>>(P, m->fixed, m->moving, m->mmask,
                                                                         m->samples, ns, d_st, d_fb, d_mb, d_fl);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && status) e = cudaMemcpyAsync(status, d_st, (size_t)ns, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && fixed_bin) e = cudaMemcpyAsync(fixed_bin, d_fb, (size_t)ns * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && moving_bin) e = cudaMemcpyAsync(moving_bin, d_mb, (size_t)ns * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && flat) e = cudaMemcpyAsync(flat, d_fl, (size_t)ns * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_st);
    cudaFree(d_fb);
    cudaFree(d_mb);
    cudaFree(d_fl);
    if (e != cudaSuccess) return cuda_status(ctx, e, "mi_metric_sample_decisions");
    return MI_OK;
}

}  // extern "C"
