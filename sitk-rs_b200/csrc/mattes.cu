// Mattes mutual information on the device: metric set-up and the per-evaluation
// kernels.
//
// One evaluation (DeviceMattesMetric::evaluate, registration/device.rs:767-800) is two
// launches; the result reaches the host through mapped pinned memory, with no copy:
//   k_hist   pass 1: sampler (value and gradient) → Parzen joint histogram, per CTA
//            in shared memory as u32 fixed point (native shared atomics), flushed
//            with the joint part's column sums into global u64 counters. Integer adds
//            are exact, so the histogram does not depend on the order. Each sample also
//            leaves an 18-byte record (both Parzen bins, Parzen fraction, index-space
//            gradient) for pass 2. Samples whose decisions the fast path cannot take
//            are queued and run through the exact FP64 chain after the main loop.
//   k_deriv  launched as a programmatic dependent of k_hist. Every CTA forms the tail
//            itself from the integer histogram (registration/mattes.rs:273-328:
//            normalisation, marginals and the pRatio·nFactor table, FP64 logarithms),
//            sums the −MI slices that fall to it, then streams its records → 12
//            moments A[j] = Σ w g_j, B[j][e] = Σ w g_j (x_e − x_ref,e), w = Σ_taps
//            B₃′·pRatio (the form of the reference's mattes_deriv,
//            cuda/ops/mattes.rs:319-381), FP32 per thread and FP64 from the warp
//            reduction on, in a fixed shuffle/tree order into per-CTA partials. The last
//            CTA folds the slices and the partials in a fixed order, turns the moments
//            into physical space, contracts them with the transform's Jacobian form
//            (registration/cuda.rs:505-524), writes value, valid and derivative into the
//            host's mapped mirror with a sequence number, and clears the histogram.
// A value-only evaluation is k_hist alone: the CTA that flushes last forms the tail
// and publishes the result.
// Every reduction order is a function of the launch shape alone, so repeated
// evaluations are bit-identical. No kernel waits on another CTA.

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_run_length_encode.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <utility>

#include <cfloat>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "internal.h"
#include "sampler.cuh"
#include "eval_device.cuh"
#include "brick.cuh"
#include "tile.cuh"
#include "point_map.h"

namespace mi {

// Host geometry helpers (geometry.cpp, compiled without FP contraction).
void index_to_physical(const mi_geometry& g, double* m);
bool invert3(const double* m, double* inv);

namespace {

// ---------------------------------------------------------------------------
// Kernels. The fused evaluation is one cooperative launch:
//   histogram → grid barrier → every CTA forms the tail (CTA 0 writes value and
//   valid) and its share of the derivative moments → the last CTA to finish folds
//   the moments, writes the derivative, re-zeroes the global histogram and resets
//   the counters. The value-only form runs the tail in CTA 0 alone.
// The split form (k_hist, then k_deriv) does the same work with a kernel boundary in
// place of the barrier.
// ---------------------------------------------------------------------------
// This CTA's queue of samples for the exact chain (k_hist, k_eval: a grid-stride walk,
// so at most exq_cap = ceil(n / (grid·block))·block samples per CTA).
__device__ __forceinline__ ExactQueue exact_queue(const EvalArgs& a) {
#if MI_EXACT_DEFERRED
    return ExactQueue{a.exq + (size_t)blockIdx.x * a.exq_cap, a.exq_cap};
#else
    return ExactQueue{nullptr, 0u};
#endif
}

template <bool DERIV>
__global__ void __launch_bounds__(HIST_BLOCK, HIST_MIN_BLOCKS)
k_eval(const __grid_constant__ SamplerParams P, const __grid_constant__ JacobianForm J, EvalArgs a) {
    extern __shared__ __align__(16) unsigned char esh[];
    unsigned int* sh = reinterpret_cast<unsigned int*>(esh);
    double* dsh = reinterpret_cast<double*>(esh);
    const int B = P.bins;
    hist_phase<DERIV>(P, a, sh, grid_samples(a.n), exact_queue(a));
    if (!grid_barrier(a, 1)) return;
    TailCtx t;
    if (DERIV) {
        t = deriv_phase(P, a, dsh, grid_groups(a));
    } else {
        const TailSmem ts = tail_layout(B, esh);
        t = tail_prepare(B, P.moving_bin_size, a, ts);
        if (!t.degenerate) value_slices_share(B, a, t, ts, (int)blockIdx.x, (int)gridDim.x);
    }
    if (!last_to_arrive(a.sync)) return;
    // every CTA has left the barrier and is done with the histogram
    if (DERIV) deriv_fold(P, J, a, t, a.partials, gridDim.x);
    if (threadIdx.x < 32) fold_value(B, a, t);
    if (threadIdx.x == 0) {
        a.sync[0] = 0u;
        a.sync[2] = 0u;
    }
    for (int i = threadIdx.x; i < B * B + B; i += blockDim.x) a.ghist[i] = 0ull;
    if (a.gcols)
        for (int i = threadIdx.x; i < B; i += blockDim.x) a.gcols[i] = 0ull;
}

// Histogram pass of the split form. For a value-only evaluation (RECORD false) the CTA
// that flushes last forms the tail (tail_once) and publishes the result, so that
// evaluation is this one launch.
size_t hist_kernel_smem(int B) { return std::max(hist_smem(B), tail_once_smem(B)); }

template <bool RECORD>
__global__ void __launch_bounds__(HIST_BLOCK, HIST_MIN_BLOCKS)
k_hist(const __grid_constant__ SamplerParams P, EvalArgs a) {
    extern __shared__ __align__(16) unsigned int sh[];
    pdl_launch_dependents();
    hist_phase<RECORD, (HIST_CLUSTER > 1)>(P, a, sh, grid_samples(a.n), exact_queue(a));
    // the value+derivative evaluation's tail is formed by k_deriv's CTAs; a value-only
    // evaluation ends here, with its tail in the CTA that flushes last
    if (RECORD || !last_to_arrive(a.sync + 1)) return;
    tail_once(P.bins, P.moving_bin_size, a, reinterpret_cast<unsigned char*>(sh), true);
}

// Derivative pass of the split form, a programmatic dependent of k_hist: each CTA forms
// the tail and its value slices, then the moments of its records (stream_phase); the
// last CTA folds them, contracts them with the Jacobian form and publishes value, valid
// and derivative.
__global__ void __launch_bounds__(DERIV_BLOCK, DERIV_MIN_BLOCKS)
k_deriv(const __grid_constant__ SamplerParams P, const __grid_constant__ JacobianForm J, EvalArgs a) {
    extern __shared__ double dsh[];
    pdl_wait();
    const TailCtx t = stream_phase(P, a, dsh, grid_groups(a));
    if (!last_to_arrive(a.sync)) return;
    // every CTA has read the histogram and written its value slices and moments; the
    // last warp folds the value while the others fold the derivative
    static_assert(DERIV_BLOCK >= 18 * NMOM + 32, "deriv_fold's value warp");
    deriv_fold<true>(P, J, a, t, a.partials, gridDim.x);
    publish_seq(a, J.nparams);
    if (threadIdx.x == 0) a.sync[0] = 0u;
    for (int i = threadIdx.x; i < P.bins * P.bins + P.bins; i += blockDim.x) a.ghist[i] = 0ull;
    for (int i = threadIdx.x; i < P.bins; i += blockDim.x) a.gcols[i] = 0ull;
}

// The histogram pass with TMA-staged moving tiles (tile.cuh), one CTA per SM; a
// value-only evaluation ends with the tail in the CTA that flushes last, as in k_hist.
template <bool RECORD>
__global__ void __launch_bounds__(TILE_BLOCK, 1)
k_hist_tile(const __grid_constant__ SamplerParams P, EvalArgs a, const __grid_constant__ CUtensorMap tmap,
            TileArgs T) {
    extern __shared__ __align__(128) unsigned char tsh[];
    pdl_launch_dependents();
    tile_hist_phase<RECORD>(P, a, &tmap, T, tsh);
    if (RECORD || !last_to_arrive(a.sync + 1)) return;
    tail_once(P.bins, P.moving_bin_size, a, tsh, true);
}

// Per-sample decisions of the same sampler the kernels use, for the exactness tests.
__global__ void k_decisions(const __grid_constant__ SamplerParams P, const float* __restrict__ moving,
                            const uint8_t* __restrict__ mmask, const uint32_t* __restrict__ samples,
                            const uint8_t* __restrict__ fbin, int64_t n, int8_t* __restrict__ status,
                            int32_t* __restrict__ fb, int32_t* __restrict__ mb, int64_t* __restrict__ flat_out,
                            int8_t* __restrict__ exact_out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
        const uint32_t flat = samples ? samples[s] : (uint32_t)s;
        Sample o;
        o.exact = false;
        const int st = sample<false>(P, flat, moving, mmask, o);
        status[s] = (int8_t)st;
        fb[s] = st == SAMPLE_VALID ? (int)fbin[s] : -1;
        mb[s] = st == SAMPLE_VALID ? o.mi : -1;
        flat_out[s] = flat;
        exact_out[s] = o.exact ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------
// Set-up kernels: the draw, the fixed-mask gate, the ranges and the fixed bins.
// ---------------------------------------------------------------------------
__global__ void k_draw_random(uint64_t seed, uint64_t voxels, int64_t count, uint32_t* out) {
    // SplitMix64 (registration/metric.rs:101-122): the i-th output follows i+1
    // advances of the state, so draw i is mix(seed + (i+1)·γ) mod voxels.
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        uint64_t z = seed + (uint64_t)(i + 1) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        out[i] = (uint32_t)(z % voxels);
    }
}

// Sort key of a voxel in brick order: the fixed grid cut into bricks of 2^lb voxels
// per axis, bricks x-fastest, voxels inside a brick x-fastest.
__global__ void k_brick_key(const uint32_t* __restrict__ idx, int64_t count, int64_t nx, int64_t ny, int lb,
                            int64_t nbx, int64_t nby, unsigned long long* __restrict__ key) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = idx[t];
        const int64_t x = v % nx, row = v / nx;
        const int64_t y = row % ny, z = row / ny;
        const int64_t m = ((int64_t)1 << lb) - 1;
        const int64_t brick = ((z >> lb) * nby + (y >> lb)) * nbx + (x >> lb);
        key[t] = ((unsigned long long)brick << (3 * lb)) |
                 (unsigned long long)((((z & m) << lb | (y & m)) << lb) | (x & m));
    }
}

// Sort key of a voxel in the brick layout's order: bricks of 2^bl voxels per axis
// (x-fastest), inside a brick its 8³ sub-bricks (x-fastest), inside those the voxels
// (x-fastest). 3 ≤ bl ≤ 6.
__global__ void k_brick_key_bl(const uint32_t* __restrict__ idx, int64_t count, int64_t nx, int64_t ny, int bl,
                               int64_t nbx, int64_t nby, unsigned long long* __restrict__ key) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = idx[t];
        const int64_t x = v % nx, row = v / nx;
        const int64_t y = row % ny, z = row / ny;
        const int64_t brick = ((z >> bl) * nby + (y >> bl)) * nbx + (x >> bl);
        const int sb = bl - 3;
        const int64_t sm = ((int64_t)1 << sb) - 1;
        const int64_t sub = ((((z >> 3) & sm) << sb | ((y >> 3) & sm)) << sb) | ((x >> 3) & sm);
        const int64_t local = ((z & 7) << 6) | ((y & 7) << 3) | (x & 7);
        key[t] = ((unsigned long long)brick << (3 * bl)) | (unsigned long long)((sub << 9) | local);
    }
}

// The brick of each sample (its index in the bricks' x-fastest order).
__global__ void k_brick_of(const uint32_t* __restrict__ idx, int64_t count, int64_t nx, int64_t ny, int bl,
                           int64_t nbx, int64_t nby, uint32_t* __restrict__ bid) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = idx[t];
        const int64_t x = v % nx, row = v / nx;
        const int64_t y = row % ny, z = row / ny;
        bid[t] = (uint32_t)(((z >> bl) * nby + (y >> bl)) * nbx + (x >> bl));
    }
}

__global__ void k_run_chunks(const int* __restrict__ counts, int64_t nruns, uint32_t* __restrict__ nch) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nruns; r += (int64_t)gridDim.x * blockDim.x)
        nch[r] = (uint32_t)((counts[r] + BRICK_CHUNK - 1) / BRICK_CHUNK);
}

// Per run (a non-empty brick): its packed coordinates and the run index of each of its
// chunks.
__global__ void k_run_fill(const uint32_t* __restrict__ bid, int64_t nruns, const uint32_t* __restrict__ chunk_off,
                           const uint32_t* __restrict__ nch, int64_t nbx, int64_t nby, uint32_t* __restrict__ run_brick,
                           uint32_t* __restrict__ chunk_run) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nruns; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = bid[r];
        const int64_t bx = b % nbx, by = (b / nbx) % nby, bz = b / (nbx * nby);
        run_brick[r] = (uint32_t)(bx | (by << 10) | (bz << 20));
        for (uint32_t c = 0; c < nch[r]; ++c) chunk_run[chunk_off[r] + c] = (uint32_t)r;
    }
}

// The codes: one CTA per run, sample t of the run at padded position chunk_off·32 + t:
// its offset in the brick (bl bits per axis) and its fixed bin above them (fbin in walk
// order, or by voxel for the whole grid).
__global__ void k_scatter_codes(const uint32_t* __restrict__ samples, const uint8_t* __restrict__ fbin,
                                bool fbin_by_flat, const int* __restrict__ counts,
                                const uint32_t* __restrict__ run_start, const uint32_t* __restrict__ chunk_off,
                                int64_t nx, int64_t ny, int bl, uint32_t* __restrict__ codes) {
    const int64_t r = blockIdx.x;
    const int64_t n = counts[r];
    const int64_t s0 = run_start[r], p0 = (int64_t)chunk_off[r] * BRICK_CHUNK;
    const int64_t msk = ((int64_t)1 << bl) - 1;
    for (int64_t t = threadIdx.x; t < n; t += blockDim.x) {
        const int64_t v = samples[s0 + t];
        const int64_t x = v % nx, row = v / nx;
        const int64_t y = row % ny, z = row / ny;
        codes[p0 + t] = (uint32_t)((x & msk) | ((y & msk) << bl) | ((z & msk) << (2 * bl)) |
                                   ((int64_t)fbin[fbin_by_flat ? v : s0 + t] << (3 * bl)));
    }
}

__global__ void k_iota_stride(int64_t count, uint64_t stride_v, uint32_t* out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
        out[i] = (uint32_t)((uint64_t)i * stride_v);
}

__global__ void k_mask_flags(const uint32_t* __restrict__ idx, int64_t count, const float* __restrict__ fmask,
                             uint8_t* __restrict__ flags) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
        flags[i] = fmask[idx[i]] != 0.0f ? 1 : 0;
}

// v ← v rounded to BF16 (to nearest, ties to even; NaN stays NaN), bits[i] its upper
// 16 bits
__global__ void k_round_bf16(float* __restrict__ v, int64_t n, uint16_t* __restrict__ bits) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint16_t b = __bfloat16_as_ushort(__float2bfloat16_rn(v[i]));
        bits[i] = b;
        v[i] = __uint_as_float((uint32_t)b << 16);
    }
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
    if (lane == 0) {
        slo[warp] = lo;
        shi[warp] = hi;
    }
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

// The exact fixed Parzen bin of every sample, in sample order.
__global__ void k_fixed_bins(SamplerParams P, const float* __restrict__ fixed, const uint32_t* __restrict__ samples,
                             int64_t n, uint8_t* __restrict__ fbin) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
        const uint32_t flat = samples ? samples[s] : (uint32_t)s;
        fbin[s] = (uint8_t)fixed_bin(P, fixed[flat]);
    }
}

// Sample arrays are padded to whole groups of four (the derivative pass reads them
// with vector loads); at least one group is always allocated.
size_t pad4(int64_t n) { return (size_t)((std::max<int64_t>(n, 1) + 3) & ~(int64_t)3); }

int grid_for(int64_t n, int block, int cap) {
    int64_t g = (n + block - 1) / block;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

mi_status minmax(mi_context* ctx, const float* vals, const uint32_t* idx, const uint8_t* mask, int64_t n,
                 double* lo, double* hi, bool* any) {
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

// The global histogram's replicas: each B² joint + B counts + B column sums u64, padded
// to whole 256-byte blocks.
uint32_t ghist_rep_stride(int B) { return (uint32_t)(((size_t)B * B + 2 * B + 31) & ~(size_t)31); }
size_t ghist_bytes(int B) { return (size_t)GHIST_REPS * ghist_rep_stride(B) * sizeof(unsigned long long); }

// The split form's histogram grid: enough CTAs for the samples, at most as many as are
// resident at once, in whole thread-block clusters of HIST_CLUSTER (bounded by the
// clusters the device can hold at once with this kernel's shape).
int hist_grid(mi_context* ctx, int64_t n, int occ, int B) {
    int g = grid_for(n, HIST_BLOCK, ctx->num_sms * std::max(occ, 1));
    if (HIST_CLUSTER <= 1) return g;
    int clusters = (g + HIST_CLUSTER - 1) / HIST_CLUSTER;
    cudaLaunchConfig_t hc = {};
    hc.gridDim = dim3((unsigned)(clusters * HIST_CLUSTER));
    hc.blockDim = dim3(HIST_BLOCK);
    hc.dynamicSmemBytes = hist_kernel_smem(B);
    cudaLaunchAttribute hattr[1];
    hattr[0].id = cudaLaunchAttributeClusterDimension;
    hattr[0].val.clusterDim.x = HIST_CLUSTER;
    hattr[0].val.clusterDim.y = 1;
    hattr[0].val.clusterDim.z = 1;
    hc.attrs = hattr;
    hc.numAttrs = 1;
    int active = 0;
    if (cudaOccupancyMaxActiveClusters(&active, k_hist<true>, &hc) == cudaSuccess && active > 0)
        clusters = std::min(clusters, active);
    else
        cudaGetLastError();
    return std::max(1, clusters) * HIST_CLUSTER;
}

void free_metric(mi_metric* m) {
    if (!m) return;
    if (m->mtex) cudaDestroyTextureObject(m->mtex);
    if (m->marray) cudaFreeArray(m->marray);
    cudaFree(m->fixed);
    cudaFree(m->moving);
    cudaFree(m->mmask);
    cudaFree(m->samples);
    cudaFree(m->fbin);
    cudaFree(m->codes);
    cudaFree(m->chunk_run);
    cudaFree(m->run_brick);
    cudaFree(m->run_chunk0);
    cudaFree(m->run_start);
    cudaFree(m->ws.hist);
    cudaFree(m->ws.partials);
    cudaFree(m->ws.vsum);
    cudaFree(m->ws.exq);
    cudaFree(m->ws.result);
    cudaFree(m->ws.done_counter);
    cudaFree(m->ws.rec_bins);
    cudaFree(m->ws.rec_f);
    cudaFree(m->ws.rec_g);
    if (m->ws.host_result) cudaFreeHost(m->ws.host_result);
    for (int i = 0; i < 5; ++i)
        if (m->ws.ev[i]) cudaEventDestroy(m->ws.ev[i]);
    moments_free(m);
    cudaFree(m->bs_coef);
    cudaFree(m->bs_deriv);
    cudaFree(m->bs_order);
    cudaFree(m->bs_off);
    cudaFree(m->bs_pr);
    delete m;
}

// The brick edge of the layout: the smallest of 16, 32, 64 voxels that leaves on average
// at least 200 samples per brick (few padding lanes, few bricks per CTA), and at least
// large enough that no axis has more than 1024 bricks (the packed coordinates).
int choose_brick_bl(const int64_t* size, int64_t n) {
    const int64_t nvox = size[0] * size[1] * size[2];
    int bl = 4;
    while (bl < 6 && (double)n * (double)((int64_t)1 << (3 * bl)) < 200.0 * (double)nvox) ++bl;
    for (int d = 0; d < 3; ++d)
        while (bl < 6 && ((size[d] + ((int64_t)1 << bl) - 1) >> bl) > 1024) ++bl;
    return bl;
}

// Build the sample list: the strategy's draw, gated by the fixed mask, sorted into
// brick order (SAMPLE_BRICK_LOG2). The histogram is a sum of exact integers and so
// does not depend on the order; sorting only buys locality.
// With `bricks` (the Mattes metric) the sort key is the brick layout's (brick_key_bl):
// bricks of 2^bl voxels per axis, bl chosen from the sample density (choose_brick_bl),
// then 8³ sub-bricks, then voxels, each x-fastest; m->brick_bl records bl.
mi_status build_samples(mi_context* ctx, mi_metric* m, const mi_image* fixed_mask, const mi_sampling* smp,
                        int64_t nvox, bool bricks) {
    const int strategy = smp ? smp->strategy : MI_SAMPLING_NONE;
    if (strategy == MI_SAMPLING_NONE && !fixed_mask) {
        // the whole grid, walked in voxel order with no list (the brick layout is built
        // from a sorted list of its own, build_brick_layout)
        m->samples = nullptr;
        m->n_samples = nvox;
        if (bricks) m->brick_bl = choose_brick_bl(m->fgeo.size, nvox);
        return MI_OK;
    }
    int64_t count = 0;
    uint32_t* draw = nullptr;
    cudaStream_t st = ctx->stream;
    const int block = 256;
    if (strategy == MI_SAMPLING_NONE) {
        count = nvox;
        MI_CHECK_CUDA(ctx, cudaMalloc(&draw, pad4(count) * 4));
        k_iota_stride<<<grid_for(count, block, ctx->num_sms * 8), block, 0, st>>>(count, 1, draw);
    } else if (strategy == MI_SAMPLING_REGULAR) {
        if (!(smp->percentage > 0.0) || !std::isfinite(smp->percentage))
            return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "sampling percentage must be positive");
        int64_t stride = (int64_t)std::ceil(1.0 / smp->percentage);
        if (stride < 1) stride = 1;
        count = (nvox + stride - 1) / stride;
        MI_CHECK_CUDA(ctx, cudaMalloc(&draw, pad4(count) * 4));
        k_iota_stride<<<grid_for(count, block, ctx->num_sms * 8), block, 0, st>>>(count, (uint64_t)stride, draw);
    } else if (strategy == MI_SAMPLING_RANDOM) {
        if (!(smp->percentage > 0.0) || !std::isfinite(smp->percentage))
            return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "sampling percentage must be positive");
        count = (int64_t)((double)nvox * smp->percentage);
        if (count >= ((int64_t)1 << 31))
            return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "sample count exceeds 2^31");
        MI_CHECK_CUDA(ctx, cudaMalloc(&draw, pad4(count) * 4));
        if (count)
            k_draw_random<<<grid_for(count, block, ctx->num_sms * 8), block, 0, st>>>(smp->seed, (uint64_t)nvox,
                                                                                         count, draw);
    } else if (strategy == MI_SAMPLING_EXPLICIT) {
        if (smp->n_indices < 0 || (smp->n_indices > 0 && !smp->indices))
            return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "explicit sampling needs an index list");
        if (smp->n_indices >= ((int64_t)1 << 31))
            return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "sample count exceeds 2^31");
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
        MI_CHECK_CUDA(ctx, cudaMalloc(&draw, pad4(count) * 4));
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
        MI_CHECK_CUDA(ctx, cudaMalloc(&out, pad4(count) * 4));
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
    const int64_t fsz[3] = {m->fgeo.size[0], m->fgeo.size[1], m->fgeo.size[2]};
    if (bricks) m->brick_bl = choose_brick_bl(fsz, nkept);
    if (nkept > 1 && bricks) {
        const int bl = m->brick_bl;
        const int64_t nx = fsz[0], ny = fsz[1];
        const int64_t nbx = (nx + (1 << bl) - 1) >> bl, nby = (ny + (1 << bl) - 1) >> bl;
        const int64_t nbz = (fsz[2] + (1 << bl) - 1) >> bl;
        const uint64_t kmax = (uint64_t)(nbx * nby * nbz) << (3 * bl);
        int bits = 1;
        while (bits < 64 && ((uint64_t)1 << bits) < kmax) ++bits;
        unsigned long long *keys = nullptr, *keys_out = nullptr;
        uint32_t* sorted = nullptr;
        MI_CHECK_CUDA(ctx, cudaMalloc(&keys, (size_t)nkept * 8));
        MI_CHECK_CUDA(ctx, cudaMalloc(&keys_out, (size_t)nkept * 8));
        MI_CHECK_CUDA(ctx, cudaMalloc(&sorted, pad4(nkept) * 4));
        k_brick_key_bl<<<grid_for(nkept, block, ctx->num_sms * 8), block, 0, st>>>(kept, nkept, nx, ny, bl, nbx, nby,
                                                                                  keys);
        MI_CHECK_CUDA(ctx, cudaGetLastError());
        tmp_bytes = 0;
        MI_CHECK_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys_out, kept, sorted,
                                                           (int)nkept, 0, bits, st));
        MI_CHECK_CUDA(ctx, cudaMalloc(&tmp, tmp_bytes));
        MI_CHECK_CUDA(ctx, cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys_out, kept, sorted, (int)nkept,
                                                           0, bits, st));
        MI_CHECK_CUDA(ctx, cudaStreamSynchronize(st));
        cudaFree(tmp);
        cudaFree(keys);
        cudaFree(keys_out);
        cudaFree(kept);
        kept = sorted;
    } else if (nkept > 1 && SAMPLE_BRICK_LOG2 > 0) {
        const int lb = SAMPLE_BRICK_LOG2;
        const int64_t nx = m->fgeo.size[0], ny = m->fgeo.size[1], nz = m->fgeo.size[2];
        const int64_t nbx = (nx + (1 << lb) - 1) >> lb, nby = (ny + (1 << lb) - 1) >> lb;
        const int64_t nbz = (nz + (1 << lb) - 1) >> lb;
        const uint64_t kmax = (uint64_t)(nbx * nby * nbz) << (3 * lb);
        int bits = 1;
        while (bits < 64 && ((uint64_t)1 << bits) < kmax) ++bits;
        unsigned long long *keys = nullptr, *keys_out = nullptr;
        uint32_t* sorted = nullptr;
        MI_CHECK_CUDA(ctx, cudaMalloc(&keys, (size_t)nkept * 8));
        MI_CHECK_CUDA(ctx, cudaMalloc(&keys_out, (size_t)nkept * 8));
        MI_CHECK_CUDA(ctx, cudaMalloc(&sorted, pad4(nkept) * 4));
        k_brick_key<<<grid_for(nkept, block, ctx->num_sms * 8), block, 0, st>>>(kept, nkept, nx, ny, lb, nbx, nby, keys);
        MI_CHECK_CUDA(ctx, cudaGetLastError());
        tmp_bytes = 0;
        MI_CHECK_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys_out, kept, sorted,
                                                           (int)nkept, 0, bits, st));
        MI_CHECK_CUDA(ctx, cudaMalloc(&tmp, tmp_bytes));
        MI_CHECK_CUDA(ctx, cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys_out, kept, sorted, (int)nkept,
                                                           0, bits, st));
        MI_CHECK_CUDA(ctx, cudaStreamSynchronize(st));
        cudaFree(tmp);
        cudaFree(keys);
        cudaFree(keys_out);
        cudaFree(kept);
        kept = sorted;
    } else if (nkept > 1) {
        uint32_t* sorted = nullptr;
        MI_CHECK_CUDA(ctx, cudaMalloc(&sorted, pad4(nkept) * 4));
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

// The brick layout of the walk (build_samples with bricks; the whole grid sorted here)
// and its fixed bins: runs of samples per brick (CUB run-length encoding), each padded to whole
// chunks of 32, the codes scattered to their padded positions.
mi_status build_brick_layout(mi_context* ctx, mi_metric* m) {
    cudaStream_t st = ctx->stream;
    const int64_t n = m->n_samples;
    const int bl = m->brick_bl;
    const int64_t nx = m->fgeo.size[0], ny = m->fgeo.size[1];
    const int64_t nbx = (nx + (1 << bl) - 1) >> bl, nby = (ny + (1 << bl) - 1) >> bl;
    const int block = 256;
    if (n == 0) {
        // one chunk of padding keeps every launch shape non-empty
        m->nchunks = 1;
        m->nruns = 1;
        MI_CHECK_CUDA(ctx, cudaMalloc(&m->codes, BRICK_CHUNK * 4));
        MI_CHECK_CUDA(ctx, cudaMemsetAsync(m->codes, 0xFF, BRICK_CHUNK * 4, st));
        MI_CHECK_CUDA(ctx, cudaMalloc(&m->chunk_run, 4));
        MI_CHECK_CUDA(ctx, cudaMemsetAsync(m->chunk_run, 0, 4, st));
        MI_CHECK_CUDA(ctx, cudaMalloc(&m->run_brick, 4));
        MI_CHECK_CUDA(ctx, cudaMemsetAsync(m->run_brick, 0, 4, st));
        MI_CHECK_CUDA(ctx, cudaMalloc(&m->run_start, 4));
        MI_CHECK_CUDA(ctx, cudaMemsetAsync(m->run_start, 0, 4, st));
        const uint32_t r0[2] = {0u, 1u};
        MI_CHECK_CUDA(ctx, cudaMalloc(&m->run_chunk0, 2 * 4));
        MI_CHECK_CUDA(ctx, cudaMemcpyAsync(m->run_chunk0, r0, 2 * 4, cudaMemcpyHostToDevice, st));
        MI_CHECK_CUDA(ctx, cudaStreamSynchronize(st));
        return MI_OK;
    }
    uint32_t *bid = nullptr, *uniq = nullptr, *nch = nullptr, *chunk_off = nullptr, *run_start = nullptr;
    uint32_t* whole = nullptr;  // the whole grid's voxels in brick order (no walk list)
    int *counts = nullptr, *nruns_d = nullptr;
    void* tmp = nullptr;
    size_t tb = 0;
    auto done = [&](mi_status s) {
        cudaStreamSynchronize(st);
        cudaFree(whole);
        cudaFree(bid);
        cudaFree(uniq);
        cudaFree(nch);
        cudaFree(chunk_off);
        cudaFree(run_start);
        cudaFree(counts);
        cudaFree(nruns_d);
        cudaFree(tmp);
        return s;
    };
#define TRY_L(expr)                                                      \
    do {                                                                 \
        cudaError_t _e = (expr);                                         \
        if (_e != cudaSuccess) return done(cuda_status(ctx, _e, #expr)); \
    } while (0)
    const uint32_t* list = m->samples;
    if (!list) {
        // the whole grid: its voxels sorted by the layout's key
        unsigned long long *keys = nullptr, *keys_out = nullptr;
        uint32_t* iota = nullptr;
        const int64_t nbz = (m->fgeo.size[2] + (1 << bl) - 1) >> bl;
        const uint64_t kmax = (uint64_t)(nbx * nby * nbz) << (3 * bl);
        int bits = 1;
        while (bits < 64 && ((uint64_t)1 << bits) < kmax) ++bits;
        cudaError_t e = cudaMalloc(&keys, (size_t)n * 8);
        if (e == cudaSuccess) e = cudaMalloc(&keys_out, (size_t)n * 8);
        if (e == cudaSuccess) e = cudaMalloc(&iota, (size_t)n * 4);
        if (e == cudaSuccess) e = cudaMalloc(&whole, (size_t)n * 4);
        if (e == cudaSuccess) {
            k_iota_stride<<<grid_for(n, block, ctx->num_sms * 8), block, 0, st>>>(n, 1, iota);
            k_brick_key_bl<<<grid_for(n, block, ctx->num_sms * 8), block, 0, st>>>(iota, n, nx, ny, bl, nbx, nby, keys);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
            e = cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys_out, iota, whole, (int)n, 0, bits, st);
        if (e == cudaSuccess) e = cudaMalloc(&tmp, tb);
        if (e == cudaSuccess)
            e = cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys_out, iota, whole, (int)n, 0, bits, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(keys);
        cudaFree(keys_out);
        cudaFree(iota);
        cudaFree(tmp);
        tmp = nullptr;
        tb = 0;
        if (e != cudaSuccess) return done(cuda_status(ctx, e, "brick layout of the whole grid"));
        list = whole;
    }
    TRY_L(cudaMalloc(&bid, (size_t)n * 4));
    TRY_L(cudaMalloc(&uniq, (size_t)n * 4));
    TRY_L(cudaMalloc(&counts, (size_t)n * 4));
    TRY_L(cudaMalloc(&nruns_d, sizeof(int)));
    k_brick_of<<<grid_for(n, block, ctx->num_sms * 8), block, 0, st>>>(list, n, nx, ny, bl, nbx, nby, bid);
    TRY_L(cudaGetLastError());
    TRY_L(cub::DeviceRunLengthEncode::Encode(nullptr, tb, bid, uniq, counts, nruns_d, (int)n, st));
    TRY_L(cudaMalloc(&tmp, tb));
    TRY_L(cub::DeviceRunLengthEncode::Encode(tmp, tb, bid, uniq, counts, nruns_d, (int)n, st));
    int nruns = 0;
    TRY_L(cudaMemcpyAsync(&nruns, nruns_d, sizeof(int), cudaMemcpyDeviceToHost, st));
    TRY_L(cudaStreamSynchronize(st));
    cudaFree(tmp);
    tmp = nullptr;
    TRY_L(cudaMalloc(&nch, (size_t)nruns * 4));
    TRY_L(cudaMalloc(&chunk_off, (size_t)nruns * 4));
    TRY_L(cudaMalloc(&run_start, (size_t)nruns * 4));
    k_run_chunks<<<grid_for(nruns, block, ctx->num_sms * 8), block, 0, st>>>(counts, nruns, nch);
    TRY_L(cudaGetLastError());
    tb = 0;
    size_t tb2 = 0;
    TRY_L(cub::DeviceScan::ExclusiveSum(nullptr, tb, nch, chunk_off, nruns, st));
    TRY_L(cub::DeviceScan::ExclusiveSum(nullptr, tb2, reinterpret_cast<const uint32_t*>(counts), run_start, nruns, st));
    TRY_L(cudaMalloc(&tmp, std::max(tb, tb2)));
    TRY_L(cub::DeviceScan::ExclusiveSum(tmp, tb, nch, chunk_off, nruns, st));
    TRY_L(cub::DeviceScan::ExclusiveSum(tmp, tb2, reinterpret_cast<const uint32_t*>(counts), run_start, nruns, st));
    uint32_t last[2] = {0, 0};
    TRY_L(cudaMemcpyAsync(&last[0], chunk_off + nruns - 1, 4, cudaMemcpyDeviceToHost, st));
    TRY_L(cudaMemcpyAsync(&last[1], nch + nruns - 1, 4, cudaMemcpyDeviceToHost, st));
    TRY_L(cudaStreamSynchronize(st));
    const int64_t nchunks = (int64_t)last[0] + last[1];
    if (nchunks * BRICK_CHUNK >= ((int64_t)1 << 32))
        return done(set_error(ctx, MI_ERR_INVALID_ARGUMENT, "too many samples for the brick layout"));
    m->nchunks = nchunks;
    m->nruns = nruns;
    TRY_L(cudaMalloc(&m->codes, (size_t)nchunks * BRICK_CHUNK * 4));
    TRY_L(cudaMemsetAsync(m->codes, 0xFF, (size_t)nchunks * BRICK_CHUNK * 4, st));
    TRY_L(cudaMalloc(&m->chunk_run, (size_t)nchunks * 4));
    TRY_L(cudaMalloc(&m->run_brick, (size_t)nruns * 4));
    k_run_fill<<<grid_for(nruns, block, ctx->num_sms * 8), block, 0, st>>>(uniq, nruns, chunk_off, nch, nbx, nby,
                                                                           m->run_brick, m->chunk_run);
    TRY_L(cudaGetLastError());
    k_scatter_codes<<<(unsigned)nruns, block, 0, st>>>(list, m->fbin, m->samples == nullptr, counts, run_start,
                                                       chunk_off, nx, ny, bl, m->codes);
    TRY_L(cudaGetLastError());
    // the first sample of every run in the walk order, the first chunk of every run and
    // the chunk count after the last
    TRY_L(cudaMalloc(&m->run_start, (size_t)nruns * 4));
    TRY_L(cudaMemcpyAsync(m->run_start, run_start, (size_t)nruns * 4, cudaMemcpyDeviceToDevice, st));
    TRY_L(cudaMalloc(&m->run_chunk0, ((size_t)nruns + 1) * 4));
    TRY_L(cudaMemcpyAsync(m->run_chunk0, chunk_off, (size_t)nruns * 4, cudaMemcpyDeviceToDevice, st));
    {
        const uint32_t total = (uint32_t)nchunks;
        TRY_L(cudaMemcpyAsync(m->run_chunk0 + nruns, &total, 4, cudaMemcpyHostToDevice, st));
        TRY_L(cudaStreamSynchronize(st));
    }
#undef TRY_L
    return done(MI_OK);
}

// The tensor-map encoder of the driver (cuTensorMapEncodeTiled), found once.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// The staged-tile pass's shape (tile.cuh): whether the linear moving volume meets the
// tensor-map rules (row pitch a multiple of 16 bytes), its grid (one CTA per SM), and the
// most samples one of its threads takes: over the CTAs' contiguous chunk ranges, the
// sum over their runs of ceil(chunks / 16).
mi_status tile_setup(mi_context* ctx, mi_metric* m) {
    const int64_t nx = m->mgeo.size[0];
    m->tile_capable = nx % 4 == 0 && tensor_map_encoder() != nullptr && m->nchunks > 0;
    m->tile_grid = ctx->num_sms;
    if (!m->tile_capable) return MI_OK;
    const int64_t nch = m->nchunks;
    std::vector<uint32_t> run((size_t)nch);
    MI_CHECK_CUDA(ctx, cudaMemcpyAsync(run.data(), m->chunk_run, (size_t)nch * 4, cudaMemcpyDeviceToHost, ctx->stream));
    MI_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    int64_t most = 1;
    const int64_t G = m->tile_grid;
    for (int64_t c = 0; c < G; ++c) {
        const int64_t c0 = c * nch / G, c1 = (c + 1) * nch / G;
        int64_t sum = 0;
        for (int64_t k = c0; k < c1;) {
            int64_t e = k;
            while (e < c1 && run[(size_t)e] == run[(size_t)k]) ++e;
            sum += (e - k + TILE_CONSUMER_WARPS - 1) / TILE_CONSUMER_WARPS;
            k = e;
        }
        most = std::max(most, sum);
    }
    m->tile_per_thread = most;
    return MI_OK;
}

// The tile geometry of one evaluation (box from the brick's extent in moving index
// space, the ring's depth from the shared memory left), the tensor map re-encoded when
// the box changes. Returns false when the box does not fit two buffers.
bool tile_args(mi_metric* m, const SamplerParams& P, TileArgs& T, size_t& smem) {
    int cells[3];
    for (int d = 0; d < 3; ++d) {
        const double span = P.hi_ext[d] - P.lo_ext[d];
        if (!(span >= 0.0 && span < 240.0)) return false;
        cells[d] = (int)std::floor(span) + 3;
    }
    T.bx = (cells[0] + 3 + 3) & ~3;
    T.by = cells[1];
    T.bz = cells[2];
    if (T.bx > 256 || T.by > 256 || T.bz > 256) return false;
    T.tile_floats = (uint32_t)(T.bx * T.by * T.bz);
    T.tile_stride = (T.tile_floats + 31u) & ~31u;
    const int B = m->bins;
    const size_t hist = (hist_region_bytes(B, hist_copies(B), hist_fine_copies(B)) + 127) & ~(size_t)127;
    T.meta_off = (uint32_t)hist;
    const size_t meta = ((size_t)TILE_MAX_STAGES * sizeof(TileMeta) + 127) & ~(size_t)127;
    T.tile_off = (uint32_t)(hist + meta);
    int optin = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, m->ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const size_t tile_bytes = (size_t)T.tile_stride * 4;
    const size_t fixed = (size_t)T.tile_off + 2 * TILE_MAX_STAGES * 8;
    if ((size_t)optin <= fixed) return false;
    T.stages = (int)std::min<size_t>(TILE_MAX_STAGES, ((size_t)optin - fixed) / tile_bytes);
    if (T.stages < 2) return false;
    T.bar_off = (uint32_t)(T.tile_off + (size_t)T.stages * tile_bytes);
    smem = std::max<size_t>((size_t)T.bar_off + 2 * (size_t)T.stages * 8, tail_once_smem(B));
    if (T.bx != m->tile_box[0] || T.by != m->tile_box[1] || T.bz != m->tile_box[2]) {
        const cuuint64_t dim[3] = {(cuuint64_t)m->mgeo.size[0], (cuuint64_t)m->mgeo.size[1],
                                   (cuuint64_t)m->mgeo.size[2]};
        const cuuint64_t stride[2] = {(cuuint64_t)m->mgeo.size[0] * 4,
                                      (cuuint64_t)m->mgeo.size[0] * (cuuint64_t)m->mgeo.size[1] * 4};
        const cuuint32_t box[3] = {(cuuint32_t)T.bx, (cuuint32_t)T.by, (cuuint32_t)T.bz};
        const cuuint32_t es[3] = {1, 1, 1};
        const CUresult r = tensor_map_encoder()(reinterpret_cast<CUtensorMap*>(m->tmap), CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                                                3, m->moving, dim, stride, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            m->tile_box[0] = m->tile_box[1] = m->tile_box[2] = 0;
            return false;
        }
        m->tile_box[0] = T.bx;
        m->tile_box[1] = T.by;
        m->tile_box[2] = T.bz;
    }
    T.run_chunk0 = m->run_chunk0;
    T.err = m->ws.done_counter + 3;
    return true;
}

// Per-evaluation sampler constants: the stages and the composite map (point_map.h).
mi_status fill_params(mi_metric* m, const double* stages, int nstage, SamplerParams& P) {
    P = m->base;
    if (!point_map_fill(P, stages, nstage))
        return set_error(m->ctx, MI_ERR_INVALID_ARGUMENT, "non-finite point map");
    return MI_OK;
}

}  // namespace

mi_status evaluate(mi_metric* m, const double* stages, int nstage, const double* jac0, const double* jacc,
                   int nparams, bool want_derivative, double* value, double* derivative, int64_t* valid) {
    mi_context* ctx = m->ctx;
    // an empty list, or one longer than MI_MAX_STAGES, is refused by name
    // (cuda/ops/resident.rs:698-703 upload_point_map)
    if (nstage < 1 || nstage > MI_MAX_STAGES)
        return set_error(ctx, MI_ERR_POINT_MAP_STAGE_COUNT,
                         "the device replays 1 to " + std::to_string(MI_MAX_STAGES) + " point-map stages");
    if (!stages) return MI_ERR_INVALID_ARGUMENT;
    if (want_derivative && (nparams < 1 || nparams > MI_MAX_PARAMS || !jac0 || !jacc || !derivative))
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "bad Jacobian form");
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    SamplerParams P;
    mi_status s = fill_params(m, stages, nstage, P);
    if (s != MI_OK) return s;
    if (m->metric_kind != MI_METRIC_MATTES)
        return evaluate_moments(m, P, jac0, jacc, nparams, want_derivative, value, derivative, valid);
    const int B = m->bins;
    cudaStream_t st = ctx->stream;
    Workspace& ws = m->ws;
    const bool timing = ws.timing != 0;
    const bool per_kernel = ws.timing == 2;
    const uint32_t n = (uint32_t)m->n_samples;
    EvalArgs a;
    a.moving = m->moving;
    a.mmask = m->mmask;
    a.samples = m->samples;
    a.fbin = m->fbin;
    a.n = n;
    a.npad = (n + 3u) & ~3u;
    a.hist_scale = ws.hist_scale;
    a.fine_scale = (float)std::ldexp(1.0, ws.fine_scale_log2);
    a.fine_shift = ws.fine_scale_log2 - ws.hist_scale_log2;
    a.copies = hist_copies(B);
    a.fine_copies = hist_fine_copies(B);
    a.hist_inv = std::ldexp(1.0, -ws.fine_scale_log2);
    a.ghist = ws.hist;
    a.gcols = ws.hist + B * B + B;
    // the split form's histogram pass spreads its flush over replicas; the fused form
    // (whose CTAs each read the histogram) keeps one
    a.reps = ws.fused || want_derivative ? 1 : GHIST_REPS;
    a.rep_stride = ghist_rep_stride(B);
    a.rec_bins = want_derivative ? ws.rec_bins : nullptr;
    a.rec_f = want_derivative ? ws.rec_f : nullptr;
    a.rec_g = want_derivative ? ws.rec_g : nullptr;
    a.partials = ws.partials;
    a.vsum = ws.vsum;
    a.exq = ws.exq;
    a.exq_cap = ws.fused ? ws.exq_cap_eval : ws.exq_cap_hist;
    a.sync = ws.done_counter;
    a.result = ws.result;
    // the brick layout, for the staged-tile histogram pass
    a.codes = m->codes;
    a.chunk_run = m->chunk_run;
    a.run_brick = m->run_brick;
    a.run_start = m->run_start;
    a.nchunks = (uint32_t)m->nchunks;
    // the split form's last kernel copies the result into the mapped mirror; the
    // fused form, whose CTAs may leave early on a barrier timeout, is copied back
    a.result_host = ws.fused ? nullptr : ws.host_result_dev;
    a.seq = ++ws.seq;
    JacobianForm J;
    J.nparams = want_derivative ? nparams : 0;
    for (int i = 0; i < 3 * J.nparams; ++i) {
        J.jac0[i] = jac0[i];
        for (int e = 0; e < 3; ++e) J.jacc[e][i] = jacc[e * 3 * nparams + i];
    }
    if (timing) MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[0], st));
    if (ws.fused) {
        // one cooperative launch: every CTA resident, so the in-kernel barriers hold
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)ws.grid_eval);
        cfg.blockDim = dim3(HIST_BLOCK);
        cfg.dynamicSmemBytes = eval_smem(B);
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if (want_derivative)
            MI_CHECK_CUDA(ctx, cudaLaunchKernelEx(&cfg, k_eval<true>, P, J, a));
        else
            MI_CHECK_CUDA(ctx, cudaLaunchKernelEx(&cfg, k_eval<false>, P, J, a));
        if (per_kernel) MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[1], st));
    } else {
        TileArgs T{};
        size_t tsm = 0;
        if (ws.staging == 1 && m->tile_capable && tile_args(m, P, T, tsm)) {
            // the histogram pass with TMA-staged moving tiles, one CTA per SM
            const void* fn = want_derivative ? (const void*)k_hist_tile<true> : (const void*)k_hist_tile<false>;
            mi_status ls = raise_smem_limit(ctx, fn, tsm);
            if (ls != MI_OK) return ls;
            cudaLaunchConfig_t tc = {};
            tc.gridDim = dim3((unsigned)m->tile_grid);
            tc.blockDim = dim3(TILE_BLOCK);
            tc.dynamicSmemBytes = tsm;
            tc.stream = st;
            const CUtensorMap& tmap = *reinterpret_cast<const CUtensorMap*>(m->tmap);
            if (want_derivative)
                MI_CHECK_CUDA(ctx, cudaLaunchKernelEx(&tc, k_hist_tile<true>, P, a, tmap, T));
            else
                MI_CHECK_CUDA(ctx, cudaLaunchKernelEx(&tc, k_hist_tile<false>, P, a, tmap, T));
            ++ws.tiled_evals;
        } else {
            // thread-block clusters of HIST_CLUSTER CTAs (the grid is a multiple of it)
            cudaLaunchConfig_t hc = {};
            hc.gridDim = dim3((unsigned)ws.grid_hist);
            hc.blockDim = dim3(HIST_BLOCK);
            hc.dynamicSmemBytes = hist_kernel_smem(B);
            hc.stream = st;
            cudaLaunchAttribute hattr[1];
            hattr[0].id = cudaLaunchAttributeClusterDimension;
            hattr[0].val.clusterDim.x = HIST_CLUSTER;
            hattr[0].val.clusterDim.y = 1;
            hattr[0].val.clusterDim.z = 1;
            hc.attrs = hattr;
            hc.numAttrs = HIST_CLUSTER > 1 ? 1 : 0;
            if (want_derivative)
                MI_CHECK_CUDA(ctx, cudaLaunchKernelEx(&hc, k_hist<true>, P, a));
            else
                MI_CHECK_CUDA(ctx, cudaLaunchKernelEx(&hc, k_hist<false>, P, a));
        }
        if (per_kernel) MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[1], st));
        if (want_derivative) {
            // launched as a programmatic dependent of k_hist (no event between them), so
            // its launch overlaps k_hist's last CTAs
            cudaLaunchConfig_t cfg = {};
            cfg.stream = st;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attr[0].val.programmaticStreamSerializationAllowed = 1;
            cfg.attrs = attr;
            cfg.numAttrs = per_kernel ? 0 : 1;
            cfg.gridDim = dim3((unsigned)ws.grid_deriv);
            cfg.blockDim = dim3(DERIV_BLOCK);
            cfg.dynamicSmemBytes = stream_smem(B);
            MI_CHECK_CUDA(ctx, cudaLaunchKernelEx(&cfg, k_deriv, P, J, a));
        }
        if (per_kernel) {
            MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[2], st));
            MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[3], st));
        }
    }
    MI_CHECK_CUDA(ctx, cudaGetLastError());
    if (!a.result_host)
        MI_CHECK_CUDA(ctx, cudaMemcpyAsync(ws.host_result, ws.result, RESULT_DOUBLES * sizeof(double),
                                           cudaMemcpyDeviceToHost, st));
    if (timing) MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[4], st));
    if (a.result_host && !timing) {
        // wait for the published sequence number in the mapped mirror rather than for the
        // stream (whose last kernel may still be clearing the histogram for the next
        // evaluation); the stream is queried every 256 polls, so a failed launch still
        // ends the wait with its error, and a finished stream without the number is
        // reported as an error
        const volatile unsigned long long* words = reinterpret_cast<const volatile unsigned long long*>(ws.host_result);
        const int np = want_derivative ? nparams : 0;
        auto published = [&]() { return words[RESULT_ERR + 1] == publish_tag(a.seq, words, np); };
        for (uint32_t spin = 1;; ++spin) {
            if (published()) break;
            if ((spin & 255u) == 0u) {
                const cudaError_t q = cudaStreamQuery(st);
                if (q == cudaSuccess) {
                    if (published()) break;
                    return set_error(ctx, MI_ERR_CUDA, "the evaluation finished without publishing its result");
                }
                if (q != cudaErrorNotReady) return cuda_status(ctx, q, "cudaStreamQuery");
            }
        }
    } else {
        MI_CHECK_CUDA(ctx, cudaStreamSynchronize(st));
    }
    unsigned int err = 0;
    std::memcpy(&err, ws.host_result + RESULT_ERR, sizeof(err));
    if (err) {
        // a barrier gave up: clear the counters, the error word and the histogram
        MI_CHECK_CUDA(ctx, cudaMemsetAsync(ws.done_counter, 0, 4 * sizeof(unsigned int), st));
        MI_CHECK_CUDA(ctx, cudaMemsetAsync(ws.result, 0, RESULT_DOUBLES * sizeof(double), st));
        MI_CHECK_CUDA(ctx, cudaMemsetAsync(ws.hist, 0, ghist_bytes(B), st));
        MI_CHECK_CUDA(ctx, cudaStreamSynchronize(st));
        return set_error(ctx, MI_ERR_TIMEOUT, ws.fused ? "a grid barrier of the fused evaluation timed out"
                                                         : "a staged-tile wait of the histogram pass timed out");
    }
    if (timing) {
        float t = 0.f;
        MI_CHECK_CUDA(ctx, cudaEventElapsedTime(&t, ws.ev[0], ws.ev[4]));
        ws.ms[0] += t;
        if (per_kernel) {
            MI_CHECK_CUDA(ctx, cudaEventElapsedTime(&t, ws.ev[0], ws.ev[1]));
            ws.ms[1] += t;
            if (!ws.fused) {
                MI_CHECK_CUDA(ctx, cudaEventElapsedTime(&t, ws.ev[1], ws.ev[2]));
                ws.ms[2] += t;
                MI_CHECK_CUDA(ctx, cudaEventElapsedTime(&t, ws.ev[2], ws.ev[3]));
                ws.ms[3] += t;
            }
        }
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

mi_status mi_metric_create(mi_context* ctx, const mi_image* fixed, const mi_image* moving, const mi_image* fixed_mask,
                           const uint8_t* moving_mask, const mi_sampling* sampling, int bins, mi_metric** out) {
    return mi_metric_create_ex(ctx, fixed, moving, fixed_mask, moving_mask, sampling, bins, nullptr, out);
}

mi_status mi_metric_create_ex(mi_context* ctx, const mi_image* fixed, const mi_image* moving,
                              const mi_image* fixed_mask, const uint8_t* moving_mask, const mi_sampling* sampling,
                              int bins, const mi_metric_options* options, mi_metric** out) {
    using namespace mi;
    if (!ctx || !fixed || !moving || !out) return MI_ERR_INVALID_ARGUMENT;
    const int storage = options ? options->moving_storage : MI_STORAGE_F32;
    if (storage != MI_STORAGE_F32 && storage != MI_STORAGE_BF16)
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "moving_storage must be MI_STORAGE_F32 or MI_STORAGE_BF16");
    const int metric = options ? options->metric : MI_METRIC_MATTES;
    if (metric != MI_METRIC_MATTES && metric != MI_METRIC_MEAN_SQUARES && metric != MI_METRIC_CORRELATION)
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "unknown metric kind");
    const int texture = options ? options->texture : MI_TEXTURE_AUTO;
    if (texture != MI_TEXTURE_AUTO && texture != MI_TEXTURE_3D)
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "texture must be MI_TEXTURE_AUTO or MI_TEXTURE_3D");
    const bool mattes = metric == MI_METRIC_MATTES;
    if (!mattes) bins = 0;  // no histogram
    *out = nullptr;
    if (fixed->ctx != ctx || moving->ctx != ctx || (fixed_mask && fixed_mask->ctx != ctx))
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "images belong to another context");
    if (mattes && bins < 2 * PADDING + 1)
        return set_error(ctx, MI_ERR_TOO_FEW_HISTOGRAM_BINS,
                         "need at least " + std::to_string(2 * PADDING + 1) + " histogram bins, got " +
                             std::to_string(bins));
    if (mattes && bins > MI_MAX_BINS)
        return set_error(ctx, MI_ERR_TOO_MANY_HISTOGRAM_BINS,
                         "the shared-memory histogram holds at most " + std::to_string(MI_MAX_BINS) + " bins");
    if (fixed_mask)
        for (int d = 0; d < 3; ++d)
            if (fixed_mask->geo.size[d] != fixed->geo.size[d])
                return set_error(ctx, MI_ERR_MASK_SIZE_MISMATCH, "fixed mask size differs from the fixed image");
    const int64_t nvox = fixed->n, mvox = moving->n;
    if (nvox >= ((int64_t)1 << 31) || mvox >= ((int64_t)1 << 32))
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT,
                         "volume too large: the fixed grid must hold fewer than 2^31 voxels and the moving "
                         "volume fewer than 2^32");
    double m_i2p[9], m_p2i[9], f_i2p[9];
    index_to_physical(moving->geo, m_i2p);
    if (!invert3(m_i2p, m_p2i)) return set_error(ctx, MI_ERR_SINGULAR_DIRECTION, "moving direction is singular");
    index_to_physical(fixed->geo, f_i2p);
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));

    mi_metric* m = new (std::nothrow) mi_metric();
    if (!m) return MI_ERR_OUT_OF_MEMORY;
    m->ctx = ctx;
    m->metric_kind = metric;
    m->fgeo = fixed->geo;
    m->mgeo = moving->geo;
    m->bins = bins;
    cudaStream_t st = ctx->stream;
    uint16_t* mbits = nullptr;  // BF16 storage: the rounded volume's bits, for the texture
    auto fail = [&](mi_status s) {
        cudaStreamSynchronize(st);
        cudaFree(mbits);
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
    if (storage == MI_STORAGE_BF16) {
        // the metric sees the volume rounded to BF16 everywhere: the range, the exact
        // fallback's copy (the widened values) and the texture (the bits)
        TRY_CUDA(cudaMalloc(&mbits, (size_t)mvox * 2));
        k_round_bf16<<<grid_for(mvox, 256, ctx->num_sms * 8), 256, 0, st>>>(m->moving, mvox, mbits);
        TRY_CUDA(cudaGetLastError());
    }
    if (moving_mask) {
        TRY_CUDA(cudaMalloc(&m->mmask, (size_t)mvox));
        TRY_CUDA(cudaMemcpyAsync(m->mmask, moving_mask, (size_t)mvox, cudaMemcpyHostToDevice, st));
    }
    mi_status s = build_samples(ctx, m, fixed_mask, sampling, nvox, mattes);
    if (s != MI_OK) return fail(s);

    // Histogram geometry from the sampled fixed values and the masked moving volume
    // (metric.rs:633-640, :913-924; MattesGeometry::new, mattes.rs:152-186).
    // Mean squares and correlation have no histogram and refuse no constant image.
    double fmin = 0.0, fmax = 0.0, mmin = 0.0, mmax = 0.0;
    double vmax = 0.0;  // the largest |voxel| of the whole moving volume (the fast path's bounds)
    mi_metric_info& info = m->info;
    info.bins = bins;
    info.n_samples = m->n_samples;
    if (mattes) {
        bool anyf, anym;
        s = minmax(ctx, m->fixed, m->samples, nullptr, m->n_samples, &fmin, &fmax, &anyf);
        if (s != MI_OK) return fail(s);
        s = minmax(ctx, m->moving, nullptr, m->mmask, mvox, &mmin, &mmax, &anym);
        if (s != MI_OK) return fail(s);
        double gmin = mmin, gmax = mmax;
        if (m->mmask) {
            // a corner may be any voxel, masked or not
            bool anyg;
            s = minmax(ctx, m->moving, nullptr, nullptr, mvox, &gmin, &gmax, &anyg);
            if (s != MI_OK) return fail(s);
        }
        vmax = std::max(std::fabs(gmin), std::fabs(gmax));
        if (fmax - fmin <= DBL_EPSILON) return fail(set_error(ctx, MI_ERR_CONSTANT_FIXED, "constant intensity: fixed"));
        if (mmax - mmin <= DBL_EPSILON) return fail(set_error(ctx, MI_ERR_CONSTANT_MOVING, "constant intensity: moving"));
        const double denom = (double)(bins - 2 * PADDING);
        info.fixed_min = fmin;
        info.fixed_max = fmax;
        info.moving_min = mmin;
        info.moving_max = mmax;
        info.fixed_bin_size = (fmax - fmin) / denom;
        info.moving_bin_size = (mmax - mmin) / denom;
        info.fixed_normalized_min = fmin / info.fixed_bin_size - (double)PADDING;
        info.moving_normalized_min = mmin / info.moving_bin_size - (double)PADDING;
    }

    SamplerParams& P = m->base;
    std::memset(&P, 0, sizeof(P));
    P.fsize0 = fixed->geo.size[0];
    P.fsize1 = fixed->geo.size[1];
    P.fsize2 = fixed->geo.size[2];
    P.div0 = make_fastdiv((uint32_t)P.fsize0);
    P.div1 = make_fastdiv((uint32_t)P.fsize1);
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
    for (int d = 0; d < 3; ++d) P.msz[d] = (int)moving->geo.size[d];
    P.ms1 = (uint32_t)P.mstride1;
    P.ms2 = (uint32_t)P.mstride2;
    {
        // the moving volume behind a point-sampling, clamp-to-edge, unnormalised-coordinate
        // texture (the fast path's corner fetch): a 2-D layered array, one layer per z
        // slice, whose cell corners come in two gathers, when the volume fits the
        // layered limits; else a block-linear 3-D array read by eight point fetches
        const bool b16 = storage == MI_STORAGE_BF16;
        const cudaChannelFormatDesc fmt = b16 ? cudaCreateChannelDesc<unsigned short>() : cudaCreateChannelDesc<float>();
        const size_t esize = b16 ? 2 : 4;
        const cudaExtent ext = make_cudaExtent((size_t)moving->geo.size[0], (size_t)moving->geo.size[1],
                                               (size_t)moving->geo.size[2]);
        int lw = 0, lh = 0, ll = 0;
        TRY_CUDA(cudaDeviceGetAttribute(&lw, cudaDevAttrMaxTexture2DLayeredWidth, ctx->device));
        TRY_CUDA(cudaDeviceGetAttribute(&lh, cudaDevAttrMaxTexture2DLayeredHeight, ctx->device));
        TRY_CUDA(cudaDeviceGetAttribute(&ll, cudaDevAttrMaxTexture2DLayeredLayers, ctx->device));
        const bool layered = moving->geo.size[0] <= lw && moving->geo.size[1] <= lh && moving->geo.size[2] <= ll &&
                             MOVING_LAYERED && texture == MI_TEXTURE_AUTO && mattes;
        TRY_CUDA(cudaMalloc3DArray(&m->marray, &fmt, ext, layered ? cudaArrayLayered : 0));
        P.mlayered = layered ? 1 : 0;
        cudaMemcpy3DParms cp = {};
        cp.srcPtr = make_cudaPitchedPtr(b16 ? (void*)mbits : (void*)m->moving, (size_t)moving->geo.size[0] * esize,
                                        (size_t)moving->geo.size[0], (size_t)moving->geo.size[1]);
        cp.dstArray = m->marray;
        cp.extent = ext;
        cp.kind = cudaMemcpyDeviceToDevice;
        const cudaError_t ce = cudaMemcpy3DAsync(&cp, st);
        if (mbits) {
            cudaStreamSynchronize(st);
            cudaFree(mbits);
            mbits = nullptr;
        }
        TRY_CUDA(ce);
        P.mbf16 = b16 ? 1 : 0;
        cudaResourceDesc res = {};
        res.resType = cudaResourceTypeArray;
        res.res.array.array = m->marray;
        cudaTextureDesc td = {};
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModePoint;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        TRY_CUDA(cudaCreateTextureObject(&m->mtex, &res, &td, nullptr));
        P.mtex = m->mtex;
    }
    P.bins = bins;
    P.fixed_bin_size = info.fixed_bin_size;
    P.moving_bin_size = info.moving_bin_size;
    P.inv_moving_bin_size = mattes ? 1.0 / info.moving_bin_size : 0.0;
    P.fixed_nmin = info.fixed_normalized_min;
    P.moving_nmin = info.moving_normalized_min;
    P.moving_min = mmin;
    P.moving_max = mmax;
    P.inv_bin_f = (float)P.inv_moving_bin_size;
    P.nmin_f = (float)P.moving_nmin;
    P.bin_hi_f = (float)(bins - PADDING - 1);
    P.vmax = vmax;
    P.brick_bl = mattes ? m->brick_bl : 0;
    // x_ref: the fixed grid's physical centre; x − x_ref = M_f·idx + (o_f − x_ref)
    const double mid[3] = {0.5 * (double)(P.fsize0 - 1), 0.5 * (double)(P.fsize1 - 1), 0.5 * (double)(P.fsize2 - 1)};
    for (int r = 0; r < 3; ++r) {
        P.xref[r] = P.forigin[r] + f_i2p[r * 3] * mid[0] + f_i2p[r * 3 + 1] * mid[1] + f_i2p[r * 3 + 2] * mid[2];
        P.xmid[r] = (float)mid[r];
    }

    if (!mattes) {
        s = moments_setup(m);
        if (s != MI_OK) return fail(s);
        TRY_CUDA(cudaStreamSynchronize(st));
        *out = m;
        return MI_OK;
    }

    // The exact fixed bin of every sample (a pure function of the fixed value).
    TRY_CUDA(cudaMalloc(&m->fbin, pad4(m->n_samples)));
    k_fixed_bins<<<grid_for(m->n_samples, 256, ctx->num_sms * 8), 256, 0, st>>>(P, m->fixed, m->samples,
                                                                              m->n_samples, m->fbin);
    TRY_CUDA(cudaGetLastError());
    // The brick layout of the samples for the staged-tile histogram pass (tile.cuh).
    s = build_brick_layout(ctx, m);
    if (s != MI_OK) return fail(s);
    s = tile_setup(ctx, m);
    if (s != MI_OK) return fail(s);

    // Workspace and launch shapes.
    Workspace& ws = m->ws;
    const int B = bins;
    // dynamic shared-memory limits only ever raised (a metric with fewer bins must not
    // lower them under another metric's launches)
#define TRY_STATUS(expr)                 \
    do {                                 \
        mi_status _s = (expr);           \
        if (_s != MI_OK) return fail(_s); \
    } while (0)
    TRY_STATUS(raise_smem_limit(ctx, (const void*)k_hist<true>, hist_kernel_smem(B)));
    TRY_STATUS(raise_smem_limit(ctx, (const void*)k_hist<false>, hist_kernel_smem(B)));
    TRY_STATUS(raise_smem_limit(ctx, (const void*)k_deriv, stream_smem(B)));
    TRY_STATUS(raise_smem_limit(ctx, (const void*)k_eval<true>, eval_smem(B)));
    TRY_STATUS(raise_smem_limit(ctx, (const void*)k_eval<false>, eval_smem(B)));
#undef TRY_STATUS
    int occ_h = 0, occ_d = 0, occ_e1 = 0, occ_e0 = 0, coop = 0;
    TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_h, k_hist<true>, HIST_BLOCK, hist_kernel_smem(B)));
    TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_d, k_deriv, DERIV_BLOCK, stream_smem(B)));
    TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_e1, k_eval<true>, HIST_BLOCK, eval_smem(B)));
    TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_e0, k_eval<false>, HIST_BLOCK, eval_smem(B)));
    TRY_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, ctx->device));
    // The fused form needs every CTA resident (a cooperative launch).
    const int resident = ctx->num_sms * std::min(occ_e1, occ_e0);
    // The split form is the default: the fused kernel's device time is the same, and
    // a cooperative launch waits for the stream to drain, which adds its latency to
    // every synchronous evaluation.
    ws.can_fuse = coop != 0 && resident >= 1;
    ws.fused = false;
    ws.grid_eval = ws.can_fuse ? grid_for(m->n_samples, HIST_BLOCK, resident) : 0;
    ws.grid_hist = hist_grid(ctx, m->n_samples, occ_h, B);
    ws.grid_deriv = grid_for((int64_t)pad4(m->n_samples) / 4, DERIV_BLOCK, ctx->num_sms * std::max(occ_d, 1));
    ws.block_hist = HIST_BLOCK;
    ws.block_deriv = DERIV_BLOCK;
    // Fixed-point scales of the histogram taps. A thread takes at most per_thread
    // samples, and a copy of the CTA histogram is fed by HIST_BLOCK/copies threads, so
    // it sees at most copy_max samples; each adds at most one tap to a bin (coarse
    // taps ≤ 2/3, fine taps < 2^-FINE_T). Every counter must stay below 2^32 and every
    // rounded tap below 2^22 (the magic-add rounding): k ≤ 22, kf ≤ FINE_T + 22. The global
    // u64 bin, in units of 2^-kf, takes at most n_samples·(2/3)·2^kf.
    {
        // both forms' histogram grids (the form can be switched after creation)
        const int64_t hgrid = ws.can_fuse ? std::min(ws.grid_hist, ws.grid_eval) : ws.grid_hist;
        // (and the staged-tile pass's bound, where it can run)
        const int64_t per_thread = std::max((m->n_samples + hgrid * HIST_BLOCK - 1) / (hgrid * HIST_BLOCK),
                                            m->tile_capable ? m->tile_per_thread : (int64_t)0);
        const double lim = 4294967295.0 * 0.98;
        const double coarse_max = (double)std::max<int64_t>(per_thread * (HIST_BLOCK / hist_copies(B)), 1);
        const double fine_max = (double)std::max<int64_t>(per_thread * (HIST_BLOCK / hist_fine_copies(B)), 1);
        int k = 22;
        while (k > 0 && std::ldexp(1.0, k) * (2.0 / 3.0) * coarse_max + coarse_max >= lim) --k;
        int kf = FINE_T + 22;
        while (kf > k && (std::ldexp(1.0, kf - FINE_T) * fine_max + fine_max >= lim ||
                          std::ldexp(1.0, kf) * (double)(m->n_samples + 1) >= 0x1p63))
            --kf;
        ws.hist_scale_log2 = k;
        ws.hist_scale = (float)std::ldexp(1.0, k);
        ws.fine_scale_log2 = kf;
    }
    {
        // padded to whole groups of four samples; padding records keep moving bin 0
        const size_t ns = pad4(m->n_samples);
        TRY_CUDA(cudaMalloc(&ws.rec_bins, ns * sizeof(uint16_t)));
        TRY_CUDA(cudaMemsetAsync(ws.rec_bins, 0, ns * sizeof(uint16_t), st));
        TRY_CUDA(cudaMalloc(&ws.rec_f, ns * sizeof(float)));
        TRY_CUDA(cudaMalloc(&ws.rec_g, 3 * ns * sizeof(float)));
    }
    // joint B², fixed counts B, then the joint part's B column sums
    TRY_CUDA(cudaMalloc(&ws.hist, ghist_bytes(B)));
    TRY_CUDA(cudaMemsetAsync(ws.hist, 0, ghist_bytes(B), st));
    // partials serve both forms: the split form's k_deriv grid and, should the form
    // be switched, the fused grid
    {
        const int pgrid = std::max(ws.grid_deriv, std::max(ws.grid_eval,
            grid_for((int64_t)pad4(m->n_samples) / 4, DERIV_BLOCK, ctx->num_sms * std::max(occ_d, 1))));
        ws.grid_split_hist = ws.grid_hist;
        ws.grid_split_deriv = grid_for((int64_t)pad4(m->n_samples) / 4, DERIV_BLOCK, ctx->num_sms * std::max(occ_d, 1));
        TRY_CUDA(cudaMalloc(&ws.partials, (size_t)pgrid * NMOM * 8));
    }
    TRY_CUDA(cudaMalloc(&ws.vsum, (size_t)value_slices(B) * 8));
    {
        // a grid-stride walk gives a CTA at most ceil(n / (grid·block))·block samples
        auto cap = [&](int grid) -> uint32_t {
            if (grid < 1) return 0u;
            const int64_t per = ((int64_t)m->n_samples + (int64_t)grid * HIST_BLOCK - 1) / ((int64_t)grid * HIST_BLOCK);
            return (uint32_t)(per * HIST_BLOCK);
        };
        ws.exq_cap_hist = cap(ws.grid_hist);
        ws.exq_cap_eval = cap(ws.grid_eval);
        const size_t len = std::max((size_t)ws.grid_hist * ws.exq_cap_hist, (size_t)ws.grid_eval * ws.exq_cap_eval);
        TRY_CUDA(cudaMalloc(&ws.exq, std::max<size_t>(len, 1) * sizeof(uint32_t)));
    }
    TRY_CUDA(cudaMalloc(&ws.result, RESULT_DOUBLES * 8));
    TRY_CUDA(cudaMalloc(&ws.done_counter, 4 * sizeof(unsigned int)));
    TRY_CUDA(cudaMemsetAsync(ws.done_counter, 0, 4 * sizeof(unsigned int), st));
    TRY_CUDA(cudaMemsetAsync(ws.result, 0, RESULT_DOUBLES * 8, st));
    TRY_CUDA(cudaHostAlloc(&ws.host_result, RESULT_DOUBLES * 8, cudaHostAllocMapped));
    std::memset(ws.host_result, 0, RESULT_DOUBLES * 8);  // no stale sequence number
    TRY_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&ws.host_result_dev), ws.host_result, 0));
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

mi_status mi_metric_sample_order(mi_metric* m, uint32_t* out, int64_t n) {
    if (!m || (!out && m->n_samples > 0)) return MI_ERR_INVALID_ARGUMENT;
    mi_context* ctx = m->ctx;
    if (n < m->n_samples)
        return mi::set_error(ctx, MI_ERR_INVALID_ARGUMENT, "output array shorter than the sample count");
    if (!m->samples) {
        for (int64_t i = 0; i < m->n_samples; ++i) out[i] = (uint32_t)i;
        return MI_OK;
    }
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    MI_CHECK_CUDA(ctx, cudaMemcpyAsync(out, m->samples, (size_t)m->n_samples * 4, cudaMemcpyDeviceToHost,
                                       ctx->stream));
    MI_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
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
                                         const double* fixed_params, int nfixed, double* value, double* derivative,
                                         int64_t* valid) {
    if (!m || !params || !value || !derivative) return MI_ERR_INVALID_ARGUMENT;
    mi::AffineForm f;
    mi_status s = mi::transform_form(kind, params, nparams, fixed_params, nfixed, &f);
    if (s != MI_OK) return mi::set_error(m->ctx, s, "bad transform kind or parameter count");
    // pack C_e contiguously with stride 3·P, the layout evaluate() takes
    double jc[3 * 3 * MI_MAX_PARAMS];
    for (int e = 0; e < 3; ++e)
        for (int i = 0; i < 3 * f.nparams; ++i) jc[e * 3 * f.nparams + i] = f.jacc[e][i];
    return mi::evaluate(m, f.stage, 1, f.jac0, jc, f.nparams, true, value, derivative, valid);
}

mi_status mi_metric_value_and_derivative_stages(mi_metric* m, const double* stages, int nstage, const double* jac0,
                                                const double* jac_c, int nparams, double* value, double* derivative,
                                                int64_t* valid) {
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
    ws.timing = enable < 0 ? 0 : (enable > 2 ? 2 : enable);
    return MI_OK;
}

mi_status mi_metric_set_fused(mi_metric* m, int fused) {
    if (!m) return MI_ERR_INVALID_ARGUMENT;
    if (m->metric_kind != MI_METRIC_MATTES)
        return mi::set_error(m->ctx, MI_ERR_INVALID_ARGUMENT, "the launch form is a Mattes-metric setting");
    mi::Workspace& ws = m->ws;
    if (fused && !ws.can_fuse)
        return mi::set_error(m->ctx, MI_ERR_INVALID_ARGUMENT, "a cooperative launch is not available here");
    ws.fused = fused != 0;
    ws.grid_hist = ws.fused ? ws.grid_eval : ws.grid_split_hist;
    ws.grid_deriv = ws.fused ? ws.grid_eval : ws.grid_split_deriv;
    return MI_OK;
}

mi_status mi_metric_get_fused(const mi_metric* m, int* fused) {
    if (!m || !fused) return MI_ERR_INVALID_ARGUMENT;
    *fused = m->ws.fused ? 1 : 0;
    return MI_OK;
}

mi_status mi_metric_set_tile_staging(mi_metric* m, int on) {
    if (!m) return MI_ERR_INVALID_ARGUMENT;
    if (m->metric_kind != MI_METRIC_MATTES)
        return mi::set_error(m->ctx, MI_ERR_INVALID_ARGUMENT, "staged tiles are a Mattes-metric setting");
    if (on && !m->tile_capable)
        return mi::set_error(m->ctx, MI_ERR_INVALID_ARGUMENT,
                             "staged tiles need the moving volume's x size to be a multiple of 4 and a driver "
                             "with cuTensorMapEncodeTiled");
    m->ws.staging = on ? 1 : 0;
    return MI_OK;
}

mi_status mi_metric_get_tile_staging(const mi_metric* m, int* on, int64_t* tiled_evals) {
    if (!m) return MI_ERR_INVALID_ARGUMENT;
    if (on) *on = m->ws.staging;
    if (tiled_evals) *tiled_evals = m->ws.tiled_evals;
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

mi_status mi_transform_form(int kind, const double* params, int nparams, const double* fixed_params, int nfixed,
                            double* stage12, double* jac0, double* jac_c) {
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
                                     int32_t* fixed_bin, int32_t* moving_bin, int64_t* flat, int8_t* exact, int64_t n) {
    using namespace mi;
    if (!m) return MI_ERR_INVALID_ARGUMENT;
    mi_context* ctx = m->ctx;
    if (m->metric_kind != MI_METRIC_MATTES)
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "per-sample Parzen decisions exist for the Mattes metric only");
    if (n < m->n_samples) return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "output arrays shorter than the sample count");
    if (nstage < 1 || nstage > MI_MAX_STAGES)
        return set_error(ctx, MI_ERR_POINT_MAP_STAGE_COUNT,
                         "the device replays 1 to " + std::to_string(MI_MAX_STAGES) + " point-map stages");
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    SamplerParams P;
    mi_status s = fill_params(m, stages, nstage, P);
    if (s != MI_OK) return s;
    const int64_t ns = m->n_samples;
    const size_t cap = (size_t)std::max<int64_t>(ns, 1);
    int8_t *d_st = nullptr, *d_ex = nullptr;
    int32_t *d_fb = nullptr, *d_mb = nullptr;
    int64_t* d_fl = nullptr;
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaMalloc(&d_st, cap);
    if (e == cudaSuccess) e = cudaMalloc(&d_ex, cap);
    if (e == cudaSuccess) e = cudaMalloc(&d_fb, cap * 4);
    if (e == cudaSuccess) e = cudaMalloc(&d_mb, cap * 4);
    if (e == cudaSuccess) e = cudaMalloc(&d_fl, cap * 8);
    if (e == cudaSuccess) {
        const int block = 256;
        k_decisions<<<grid_for(ns, block, ctx->num_sms * 8), block, 0, st>>>(P, m->moving, m->mmask, m->samples, m->fbin,
                                                                             ns, d_st, d_fb, d_mb, d_fl, d_ex);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && status) e = cudaMemcpyAsync(status, d_st, (size_t)ns, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && exact) e = cudaMemcpyAsync(exact, d_ex, (size_t)ns, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && fixed_bin) e = cudaMemcpyAsync(fixed_bin, d_fb, (size_t)ns * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && moving_bin) e = cudaMemcpyAsync(moving_bin, d_mb, (size_t)ns * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && flat) e = cudaMemcpyAsync(flat, d_fl, (size_t)ns * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_st);
    cudaFree(d_ex);
    cudaFree(d_fb);
    cudaFree(d_mb);
    cudaFree(d_fl);
    if (e != cudaSuccess) return cuda_status(ctx, e, "mi_metric_sample_decisions");
    return MI_OK;
}

}  // extern "C"
