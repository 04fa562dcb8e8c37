// Mattes mutual information on the device: metric set-up and the per-evaluation
// kernels.
//
// One evaluation (DeviceMattesMetric::evaluate, registration/device.rs:767-800) is two
// launches and one 8·(2+P)-byte copy back:
//   k_hist   pass 1: sampler (value and gradient) → Parzen joint histogram, per CTA
//            in shared memory as u32 fixed point (native shared atomics), flushed
//            into a global u64 histogram. Integer adds are exact, so the histogram does
//            not depend on the order. Each sample also leaves a 17-byte record
//            (moving bin, Parzen fraction, moving gradient) for pass 2. The last CTA
//            to finish runs the tail (registration/mattes.rs:273-328): normalisation,
//            marginals, −MI and the pRatio·nFactor table, and re-zeroes the global
//            histogram for the next evaluation.
//   k_deriv  pass 2: streams the records → 12 moments A[d] = Σ w g_d,
//            B[d][e] = Σ w g_d (x_e − x_ref,e), w = Σ_taps B₃′·pRatio (the form of the
//            reference's mattes_deriv, cuda/ops/mattes.rs:319-381), FP32 per thread and
//            FP64 from the warp reduction on, in a fixed shuffle/tree order into per-CTA
//            partials; the last CTA folds the partials in CTA order and contracts them
//            with the transform's Jacobian form (registration/cuda.rs:505-524).
// Every reduction order is a function of the launch shape alone, so repeated
// evaluations are bit-identical. No kernel waits on another CTA.

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

// Launch shape of the histogram pass: HIST_ILP samples per thread in flight (their
// corner gathers issued together), and a register cap that keeps HIST_MIN_BLOCKS
// CTAs of HIST_BLOCK threads resident per SM.
#ifndef MI_HIST_ILP
#define MI_HIST_ILP 2
#endif
#ifndef MI_HIST_MIN_BLOCKS
#define MI_HIST_MIN_BLOCKS 4
#endif
// Histogram copies per CTA (coarse and fine parts) and the fine part's threshold
// 2^-MI_HIST_FINE_T (see k_hist).
#ifndef MI_HIST_COPIES
#define MI_HIST_COPIES 4
#endif
#ifndef MI_HIST_FINE_COPIES
#define MI_HIST_FINE_COPIES 2
#endif
#ifndef MI_HIST_FINE_T
#define MI_HIST_FINE_T 10
#endif
constexpr int HIST_BLOCK = 256;
constexpr int HIST_MIN_BLOCKS = MI_HIST_MIN_BLOCKS;
constexpr int HIST_ILP = MI_HIST_ILP;
constexpr int DERIV_BLOCK = 256;
constexpr int NMOM = 12;

struct JacobianForm {
    int nparams;
    double jac0[3 * MI_MAX_PARAMS];
    double jacc[3][3 * MI_MAX_PARAMS];
};

// One histogram copy: B² joint + B fixed-marginal u32 counters, padded so copies
// start 4 banks apart.
__host__ __device__ inline int hist_copy_stride(int B) { return ((B * B + B + 31) & ~31) + 4; }
// Copies that fit in 48 KB (a power of two, 1–MI_HIST_COPIES).
int hist_copies(int B) {
    int c = MI_HIST_COPIES;
    while (c > 1 && (size_t)c * hist_copy_stride(B) * sizeof(unsigned int) > 48 * 1024) c >>= 1;
    return c;
}
// The fine histogram (B² u32 counters per copy) that takes the small outer taps.
__host__ __device__ inline int hist_fine_stride(int B) { return ((B * B + 31) & ~31) + 4; }
// Fine copies: up to MI_HIST_FINE_COPIES, fewer if the two parts together pass
// 52 KB (four 256-thread CTAs resident per SM at 32 bins).
int hist_fine_copies(int B) {
    const size_t coarse = (size_t)hist_copies(B) * hist_copy_stride(B) * sizeof(unsigned int);
    int c = MI_HIST_FINE_COPIES;
    while (c > 1 && coarse + (size_t)c * hist_fine_stride(B) * sizeof(unsigned int) > 52 * 1024) c >>= 1;
    return c;
}
size_t hist_smem(int B) {
    return ((size_t)hist_copies(B) * hist_copy_stride(B) + (size_t)hist_fine_copies(B) * hist_fine_stride(B)) *
           sizeof(unsigned int);
}
// Shared memory of the tail (see TailSmem).
constexpr int TAIL_BLOCK = 256;
__host__ __device__ inline int tail_groups(int B) { return TAIL_BLOCK / B; }
__host__ __device__ inline size_t tail_smem(int B) {
    return ((size_t)B * B + B + (size_t)tail_groups(B) * B + B) * 8 + ((2 * (size_t)B + 7) & ~(size_t)7);
}
size_t deriv_smem(int B) { return 32 * (size_t)NMOM * sizeof(double) + tail_smem(B) + (size_t)B * B * sizeof(float); }
// The fused kernel reuses one dynamic allocation for its phases. The derivative
// pass's layout: moment reduction scratch (32·NMOM doubles), the tail's state
// (tail_smem), then the pRatio table (B² floats).
size_t eval_smem(int B) { return std::max(hist_smem(B), std::max(deriv_smem(B), tail_smem(B))); }

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

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// Device buffers and per-launch constants shared by the evaluation kernels.
//   sync[0] done counter of the final phase, sync[2] grid-barrier counter of the
//   fused kernel.
//   result: value, valid, derivative[MI_MAX_PARAMS], then the error word.
struct EvalArgs {
    const float* moving;
    const uint8_t* mmask;
    const uint32_t* samples;
    const uint8_t* fbin;
    uint32_t n, npad;
    float hist_scale, fine_scale;
    int fine_shift, copies, fine_copies;
    double hist_inv;
    unsigned long long* ghist;
    uint16_t* rec_bins;  // per sample: moving bin | fixed bin << 8 (0 = not valid)
    float* rec_f;
    float* rec_g;
    double* partials;
    double* vsum;  // value slice sums (value_slices(B))
    unsigned int* sync;
    double* result;
};
constexpr int RESULT_ERR = 2 + MI_MAX_PARAMS;  // result slot holding the error word
constexpr int RESULT_DOUBLES = RESULT_ERR + 2;
__device__ __forceinline__ unsigned int* error_word(const EvalArgs& a) {
    return reinterpret_cast<unsigned int*>(a.result + RESULT_ERR);
}

// ---------------------------------------------------------------------------
// Pass 1: joint histogram (+ per-sample records for pass 2). The CTA histogram is
// u32 fixed point in two parts, both exact integer sums:
//   coarse: the two inner taps (always ≥ 1/6) and outer taps ≥ 2^-FINE_T, added as
//           round(w·2^k) (hist_scale = 2^k);
//   fine:   outer taps below 2^-FINE_T (a cubic B-spline's end taps, f³/6 and
//           (1−f)³/6, near a bin edge), added as round(w·2^kf) with kf > k
//           (fine_scale = 2^kf, fine_shift = kf − k).
// A sparse bin whose mass is made of end taps is where pRatio = log p is steep: a
// 2^-k quantum there moves the derivative by far more than FP32 rounding does, so
// those taps get the fine quantum. k and kf are chosen per launch so that no copy's
// counter can pass 2^32; the flush adds (coarse << fine_shift) + fine into the u64
// global histogram, whose unit is 2^-kf.
// ---------------------------------------------------------------------------
constexpr int FINE_T = MI_HIST_FINE_T;
constexpr float FINE_LIMIT = 1.0f / (float)(1u << FINE_T);

template <bool RECORD>
__device__ __forceinline__ void hist_phase(const SamplerParams& P, const EvalArgs& a, unsigned int* sh) {
    const int B = P.bins;
    const int nb = B * B + B;
    const int copies = a.copies, fine_copies = a.fine_copies;
    const int cstride = hist_copy_stride(B);
    const int fstride = hist_fine_stride(B);
    unsigned int* sh_fine = sh + copies * cstride;
    for (int i = threadIdx.x; i < copies * cstride + fine_copies * fstride; i += blockDim.x) sh[i] = 0u;
    __syncthreads();
    unsigned int* sh_joint = sh;
    unsigned int* sh_fixed = sh + B * B;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t n = a.n, npad = a.npad;
    const float* __restrict__ moving = a.moving;
    const uint8_t* __restrict__ mmask = a.mmask;
    const uint32_t* __restrict__ samples = a.samples;
    const uint8_t* __restrict__ fbin = a.fbin;
    const float hist_scale = a.hist_scale, fine_scale = a.fine_scale;
    // Two samples per iteration: both samples' corner gathers are issued (prep) before
    // either is finished, so each thread keeps two gathers in flight.
    // The CTA keeps `copies` interleaved copies of the histogram and lane l adds into
    // copy l mod copies: neighbouring lanes, whose sorted samples usually share a bin
    // pair, then add to different addresses instead of replaying on one. The copies
    // are summed at the flush (integer adds: the order does not matter).
    const int lane = threadIdx.x & 31;
    unsigned int* my_joint = sh_joint + (lane & (copies - 1)) * cstride;
    unsigned int* my_fixed = sh_fixed + (lane & (copies - 1)) * cstride;
    unsigned int* my_fine = sh_fine + (lane & (fine_copies - 1)) * fstride;
    auto account = [&](const Prep& p, uint32_t s, bool real) {
        if (!real) return;
        Sample o;
        o.exact = false;
        const int st = finish<RECORD>(P, p, moving, o);
        if (st != SAMPLE_VALID) {
            if (RECORD) a.rec_bins[s] = 0;
            return;
        }
        const int fi = __ldg(fbin + s);
        float w[4];
        bspline3_taps(o.f, w);
        const int off = fi * B + (o.mi - 1);
        unsigned int* row = my_joint + off;
        unsigned int* frow = my_fine + off;
        // round(w·scale) by the 1.5·2^23 magic add (w·scale < 2^22 for both parts):
        // one FMA, no conversion
        atomicAdd(row + 1, __float_as_uint(fmaf(w[1], hist_scale, 12582912.0f)) - 0x4B400000u);
        atomicAdd(row + 2, __float_as_uint(fmaf(w[2], hist_scale, 12582912.0f)) - 0x4B400000u);
#pragma unroll
        for (int t = 0; t < 4; t += 3) {
            const bool fine = w[t] < FINE_LIMIT;
            atomicAdd((fine ? frow : row) + t,
                      __float_as_uint(fmaf(w[t], fine ? fine_scale : hist_scale, 12582912.0f)) - 0x4B400000u);
        }
        atomicAdd(my_fixed + fi, 1u);
        if (RECORD) {
            a.rec_bins[s] = (uint16_t)(o.mi | (fi << 8));
            a.rec_f[s] = o.f;
            a.rec_g[s] = o.g[0];
            a.rec_g[(size_t)npad + s] = o.g[1];
            a.rec_g[2 * (size_t)npad + s] = o.g[2];
        }
    };
    // whole warps iterate together: the loop bound is the warp's first sample
    const uint32_t wbase = blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
    if (HIST_ILP == 2) {
        for (uint32_t b = wbase; b < n; b += 2 * stride) {
            const uint32_t s = b + lane, s2 = s + stride;
            const bool one = s < n, two = s2 < n;
            const uint32_t fa = one ? (samples ? __ldg(samples + s) : s) : 0u;
            const uint32_t fb = two ? (samples ? __ldg(samples + s2) : s2) : fa;
            Prep pa, pb;
            prep<RECORD>(P, fa, moving, mmask, pa);
            prep<RECORD>(P, fb, moving, mmask, pb);
            account(pa, s, one);
            account(pb, s2, two);
        }
    } else {
        for (uint32_t b = wbase; b < n; b += stride) {
            const uint32_t s = b + lane;
            const bool one = s < n;
            Prep pa;
            prep<RECORD>(P, one ? (samples ? __ldg(samples + s) : s) : 0u, moving, mmask, pa);
            account(pa, s, one);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        unsigned long long v = 0ull;
        for (int c = 0; c < copies; ++c) v += sh[c * cstride + i];
        if (i < B * B) {
            unsigned long long f = 0ull;
            for (int c = 0; c < fine_copies; ++c) f += sh_fine[c * fstride + i];
            v = (v << a.fine_shift) + f;
        }
        if (v) atomicAdd(&a.ghist[i], v);
    }
}

// ---------------------------------------------------------------------------
// The tail (registration/mattes.rs:273-328) over the finished global histogram. The
// marginals are sums of the integer histogram, so every CTA forms them exactly (any
// order, same bits):
//   total = Σ joint, col[m] = Σ_f joint[f][m], valid = Σ_f count[f].
// With p = joint/total the reference's quantities are
//   joint_sum = total·2^-kf, jp = joint/total, mm = col/total, fm = count/joint_sum,
//   pRatio = ln(jp/mm) = ln(joint/col), −MI = −Σ jp·(pRatio − ln fm),
// the ratio inside the logarithm formed from the exact integers; nFactor =
// 1/(moving bin size·valid); degenerate (value DBL_MAX, zero derivative) when there
// is no valid sample or Σ joint < ε (mattes.rs:590-609).
// ---------------------------------------------------------------------------
// The tail's shared-memory state, carved from `base` (tail_smem(B) bytes): a copy of
// the global histogram (B² joint + B counts, u64), per-group column partials, the
// column sums and fixed counts, and the column/row flags mm > ε, fm > ε.
struct TailSmem {
    unsigned long long* hist;  // B*B + B
    unsigned long long* part;  // tail_groups(B) * B
    unsigned long long* col;   // B
    uint8_t* okm;              // B
    uint8_t* okf;              // B
};
__device__ __forceinline__ TailSmem tail_layout(int B, unsigned char* base) {
    TailSmem t;
    t.hist = reinterpret_cast<unsigned long long*>(base);
    t.part = t.hist + B * B + B;
    t.col = t.part + tail_groups(B) * B;
    t.okm = reinterpret_cast<uint8_t*>(t.col + B);
    t.okf = t.okm + B;
    return t;
}

// Per-CTA tail state: the integer marginals, the normalisers and the degenerate flag.
struct TailCtx {
    unsigned long long total, valid;
    double dt;         // total, as a double
    double joint_sum;  // total·2^-kf
    double n_factor;   // 1/(moving bin size·valid)
    bool degenerate;
};

// Every CTA copies the histogram into shared memory with coalesced loads and forms
// the marginals from the copy: column m's sum in tail_groups(B) row groups, then over
// the groups; counts are read in place. Integer sums, so any order gives the same
// bits.
__device__ TailCtx tail_prepare(int B, double moving_bin_size, const EvalArgs& a, const TailSmem& ts) {
    const int B2 = B * B, nb = B2 + B;
    const unsigned long long* __restrict__ gh = a.ghist;
    for (int i0 = threadIdx.x; i0 < nb; i0 += 4 * blockDim.x) {
        unsigned long long v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = i0 + u * blockDim.x;
            v[u] = i < nb ? __ldcg(gh + i) : 0ull;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = i0 + u * blockDim.x;
            if (i < nb) ts.hist[i] = v[u];
        }
    }
    __syncthreads();
    const int G = tail_groups(B);
    if ((int)threadIdx.x < G * B) {
        const int m = threadIdx.x % B, g = threadIdx.x / B;
        unsigned long long v = 0ull;
        for (int f = g; f < B; f += G) v += ts.hist[f * B + m];
        ts.part[g * B + m] = v;
    }
    __syncthreads();
    if ((int)threadIdx.x < B) {
        unsigned long long v = 0ull;
        for (int g = 0; g < G; ++g) v += ts.part[g * B + threadIdx.x];
        ts.col[threadIdx.x] = v;
    }
    __syncthreads();
    const unsigned long long* cnt = ts.hist + B2;
    const int lane = threadIdx.x & 31;
    TailCtx t;
    t.total = 0ull;
    t.valid = 0ull;
    for (int m = lane; m < B; m += 32) {
        t.total += ts.col[m];
        t.valid += cnt[m];
    }
    t.total = warp_sum_u64(t.total);
    t.valid = warp_sum_u64(t.valid);
    t.dt = (double)t.total;
    t.joint_sum = t.dt * a.hist_inv;
    t.degenerate = t.valid == 0ull || t.joint_sum < DBL_EPSILON;
    t.n_factor = t.degenerate ? 0.0 : 1.0 / (moving_bin_size * (double)t.valid);
    if ((int)threadIdx.x < B) {
        ts.okm[threadIdx.x] = (double)ts.col[threadIdx.x] / t.dt > DBL_EPSILON;
        ts.okf[threadIdx.x] = (double)cnt[threadIdx.x] / t.joint_sum > DBL_EPSILON;
    }
    __syncthreads();
    return t;
}

// pRatio·nFactor of every bin into pr (shared memory, FP32): 0 where the reference
// skips the bin, else ln(joint/col)·nFactor with the ratio formed in FP64 and the
// logarithm taken in FP32 (the table is FP32).
__device__ void pr_table(int B, const TailCtx& t, const TailSmem& ts, float* pr) {
    const int B2 = B * B;
    const float nf = (float)t.n_factor;
    for (int i = threadIdx.x; i < B2; i += blockDim.x) {
        const int f = i / B, m = i - f * B;
        const unsigned long long jv = ts.hist[i];
        float r = 0.0f;
        if (ts.okf[f] && ts.okm[m] && jv && (double)jv / t.dt > DBL_EPSILON)
            r = logf((float)((double)jv / (double)ts.col[m])) * nf;
        pr[i] = r;
    }
}

// −MI is summed in value slices of 32 bins, one warp each (lane l takes bin
// 32·s + l, then a fixed xor tree), and the slice sums are folded in slice order
// (fold_value). Whichever warp of whichever kernel computes a slice, it gets the
// same bits, so every launch form reports the same value.
__host__ __device__ inline int value_slices(int B) { return (B * B + 31) / 32; }

__device__ double value_slice(int B, const TailCtx& t, const TailSmem& ts, int slice) {
    const int lane = threadIdx.x & 31;
    const int i = slice * 32 + lane;
    double term = 0.0;
    if (i < B * B) {
        const unsigned long long jv = ts.hist[i];
        const int f = i / B, m = i - f * B;
        const double jp = (double)jv / t.dt;
        const double mm = (double)ts.col[m] / t.dt;
        const double fm = (double)ts.hist[B * B + f] / t.joint_sum;
        if (fm > DBL_EPSILON && mm > DBL_EPSILON && jp > DBL_EPSILON)
            term = jp * (log((double)jv / (double)ts.col[m]) - log(fm));
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) term += __shfl_xor_sync(0xffffffffu, term, off);
    return term;
}

// This CTA's share of the value slices (global warp w takes slices w, w + W, …),
// their sums stored in a.vsum.
__device__ void value_slices_share(int B, const EvalArgs& a, const TailCtx& t, const TailSmem& ts) {
    const int lane = threadIdx.x & 31;
    const int nw = blockDim.x >> 5;
    const int ns = value_slices(B);
    for (int s = blockIdx.x * nw + (threadIdx.x >> 5); s < ns; s += gridDim.x * nw) {
        const double v = value_slice(B, t, ts, s);
        if (lane == 0) a.vsum[s] = v;
    }
}

// One warp: value and valid into result (lane 0), from the slice sums.
__device__ void fold_value(int B, const EvalArgs& a, const TailCtx& t) {
    const int lane = threadIdx.x & 31;
    const int ns = value_slices(B);
    double v = 0.0;
    for (int s = lane; s < ns; s += 32) v += __ldcg(a.vsum + s);
#pragma unroll
    for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if (lane == 0) {
        a.result[0] = t.degenerate ? DBL_MAX : -v;
        a.result[1] = (double)t.valid;
    }
}

// ---------------------------------------------------------------------------
// Pass 2: derivative moments streamed from the pass-1 records, FP32 per thread,
// FP64 from the warp reduction on; the last CTA folds the CTA partials in CTA order
// and contracts them with the transform's Jacobian form.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void accumulate_moments(const SamplerParams& P, const float* pr, int B, int mi, int fi,
                                                   float f, float g0, float g1, float g2, uint32_t flat,
                                                   float* acc) {
    uint32_t i, j, k;
    grid_index(P, flat, i, j, k);
    const float fi_ = (float)i, fj = (float)j, fk = (float)k;
    float dx[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
        dx[d] = fmaf(P.xA[d * 3 + 2], fk, fmaf(P.xA[d * 3 + 1], fj, fmaf(P.xA[d * 3 + 0], fi_, P.xb[d])));
    float dw[4];
    bspline3_deriv_taps(f, dw);
    const float* row = pr + fi * B + (mi - 1);
    const float w = fmaf(dw[3], row[3], fmaf(dw[2], row[2], fmaf(dw[1], row[1], dw[0] * row[0])));
    const float wg[3] = {w * g0, w * g1, w * g2};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        acc[d] += wg[d];
        acc[3 + d * 3 + 0] = fmaf(wg[d], dx[0], acc[3 + d * 3 + 0]);
        acc[3 + d * 3 + 1] = fmaf(wg[d], dx[1], acc[3 + d * 3 + 1]);
        acc[3 + d * 3 + 2] = fmaf(wg[d], dx[2], acc[3 + d * 3 + 2]);
    }
}

// The moments of this CTA's share of the samples, stored into partials[slot][CTA].
// The CTA first forms the tail itself (tail_prepare, pr_table) and its share of the
// value slices; the first group of records is requested before that so its loads
// overlap the tail. Records are read four samples
// per thread with 8- and 16-byte vector loads (every record array is padded to a
// multiple of four samples; padding records carry bins 0 and are skipped). Returns
// the tail state.
__device__ TailCtx deriv_phase(const SamplerParams& P, const EvalArgs& a, double* dsh) {
    const int B = P.bins;
    double* red = dsh;  // 32 * NMOM
    unsigned char* tbase = reinterpret_cast<unsigned char*>(dsh + 32 * NMOM);
    const TailSmem ts = tail_layout(B, tbase);
    float* pr = reinterpret_cast<float*>(tbase + tail_smem(B));  // B*B
    float acc[NMOM];
#pragma unroll
    for (int i = 0; i < NMOM; ++i) acc[i] = 0.0f;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t npad = a.npad;
    const uint32_t ngroups = npad >> 2;
    const uint2* b4p = reinterpret_cast<const uint2*>(a.rec_bins);
    const float4* f4p = reinterpret_cast<const float4*>(a.rec_f);
    const float4* gx4p = reinterpret_cast<const float4*>(a.rec_g);
    const float4* gy4p = reinterpret_cast<const float4*>(a.rec_g + npad);
    const float4* gz4p = reinterpret_cast<const float4*>(a.rec_g + 2 * (size_t)npad);
    const uint4* s4p = reinterpret_cast<const uint4*>(a.samples);
    // the next group's records are loaded before the current group is accumulated
    struct Group {
        uint2 b;
        float4 f, gx, gy, gz;
        uint4 fl;
    };
    auto load = [&](uint32_t q, Group& g) {
        g.b = __ldcg(b4p + q);
        g.f = __ldcg(f4p + q);
        g.gx = __ldcg(gx4p + q);
        g.gy = __ldcg(gy4p + q);
        g.gz = __ldcg(gz4p + q);
        g.fl = a.samples ? __ldg(s4p + q) : make_uint4(4 * q, 4 * q + 1, 4 * q + 2, 4 * q + 3);
    };
    auto one = [&](uint32_t bins, float f, float gx, float gy, float gz, uint32_t flat) {
        if (bins & 0xffu) accumulate_moments(P, pr, B, bins & 0xffu, bins >> 8, f, gx, gy, gz, flat, acc);
    };
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    Group cur;
    if (q < ngroups) load(q, cur);
    const TailCtx t = tail_prepare(B, P.moving_bin_size, a, ts);
    if (!t.degenerate) {
        pr_table(B, t, ts, pr);
        value_slices_share(B, a, t, ts);
    }
    __syncthreads();
    if (!t.degenerate) {
        while (q < ngroups) {
            const uint32_t qn = q + stride;
            Group nxt;
            if (qn < ngroups) load(qn, nxt);
            one(cur.b.x & 0xffffu, cur.f.x, cur.gx.x, cur.gy.x, cur.gz.x, cur.fl.x);
            one(cur.b.x >> 16, cur.f.y, cur.gx.y, cur.gy.y, cur.gz.y, cur.fl.y);
            one(cur.b.y & 0xffffu, cur.f.z, cur.gx.z, cur.gy.z, cur.gz.z, cur.fl.z);
            one(cur.b.y >> 16, cur.f.w, cur.gx.w, cur.gy.w, cur.gz.w, cur.fl.w);
            cur = nxt;
            q = qn;
        }
    }
    // CTA reduction in a fixed order: shuffles within a warp, then over warps.
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double accd[NMOM];
#pragma unroll
    for (int i = 0; i < NMOM; ++i) {
        double v = (double)acc[i];
#pragma unroll
        for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        accd[i] = v;
    }
    if (lane == 0)
        for (int i = 0; i < NMOM; ++i) red[warp * NMOM + i] = accd[i];
    __syncthreads();
    // partials are stored slot-major, [slot][CTA], so the fold reads them coalesced
    if (threadIdx.x < NMOM) {
        double v = 0.0;
        for (int w = 0; w < nw; ++w) v += red[w * NMOM + threadIdx.x];
        a.partials[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = v;
    }
    return t;
}

// Run by the last CTA to finish the derivative phase: fold every CTA's partials in
// a fixed order (lane l of a slot sums CTAs l, l+21, … eight loads at a time; the 21
// lane sums of a slot are then added in lane order) and contract with the Jacobian
// form: ∂/∂p_k = Σ_d J(x_ref)[d][k]·A_d + Σ_{d,e} C_e[d][k]·B[d][e],
// J(x_ref) = J(0) + Σ_e x_ref,e·C_e.
__device__ void deriv_fold(const SamplerParams& P, const JacobianForm& J, const EvalArgs& a, bool degenerate) {
    constexpr int FOLD = 21;
    __shared__ double fold[FOLD * NMOM];
    __shared__ double mom[NMOM];
    if (threadIdx.x < FOLD * NMOM) {
        const int slot = threadIdx.x / FOLD, ln = threadIdx.x % FOLD;
        const double* src = a.partials + (int64_t)slot * gridDim.x;
        double v = 0.0;
        unsigned int b = ln;
        for (; b + 7 * FOLD < gridDim.x; b += 8 * FOLD) {
            double t[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) t[u] = __ldcg(src + b + u * FOLD);
#pragma unroll
            for (int u = 0; u < 8; ++u) v += t[u];
        }
        for (; b < gridDim.x; b += FOLD) v += __ldcg(src + b);
        fold[slot * FOLD + ln] = v;
    }
    __syncthreads();
    if (threadIdx.x < NMOM) {
        double v = 0.0;
        for (int l = 0; l < FOLD; ++l) v += fold[threadIdx.x * FOLD + l];
        mom[threadIdx.x] = v;
    }
    __syncthreads();
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
        a.result[2 + k] = dk;
    }
}

// Arrival at the end of a kernel: returns true in the last CTA to arrive (after
// which every other CTA's global writes are visible to it).
__device__ __forceinline__ bool last_to_arrive(unsigned int* counter) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (last) __threadfence();
    return last;
}

__device__ __forceinline__ unsigned int load_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier of the fused kernel (a cooperative launch, so every CTA is
// resident). Arrivals count up across the kernel: barrier k waits for k·gridDim.x.
// The wait is bounded: after BARRIER_SPINS polls the CTA raises the error word and
// every CTA that sees it leaves, so a launch that lost a CTA ends instead of hanging.
constexpr unsigned int BARRIER_SPINS = 1u << 22;
__device__ __forceinline__ bool grid_barrier(const EvalArgs& a, unsigned int k) {
    __shared__ int ok;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int* count = a.sync + 2;
        unsigned int* err = error_word(a);
        const unsigned int target = k * gridDim.x;
        atomicAdd(count, 1u);
        int good = 1;
        unsigned int spins = 0;
        while (load_acquire(count) < target) {
            if (load_acquire(err) != 0u || ++spins > BARRIER_SPINS) {
                good = 0;
                break;
            }
            __nanosleep(64);
        }
        if (!good) atomicOr(err, 1u);
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// ---------------------------------------------------------------------------
// Kernels. The fused evaluation is one cooperative launch:
//   histogram → grid barrier → every CTA forms the tail (CTA 0 writes value and
//   valid) and its share of the derivative moments → the last CTA to finish folds
//   the moments, writes the derivative, re-zeroes the global histogram and resets
//   the counters. The value-only form runs the tail in CTA 0 alone.
// The split form (k_hist, then k_deriv or k_tail) does the same work with a kernel
// boundary in place of the barrier.
// ---------------------------------------------------------------------------
template <bool DERIV>
__global__ void __launch_bounds__(HIST_BLOCK, HIST_MIN_BLOCKS)
k_eval(SamplerParams P, JacobianForm J, EvalArgs a) {
    extern __shared__ __align__(16) unsigned char esh[];
    unsigned int* sh = reinterpret_cast<unsigned int*>(esh);
    double* dsh = reinterpret_cast<double*>(esh);
    const int B = P.bins;
    hist_phase<DERIV>(P, a, sh);
    if (!grid_barrier(a, 1)) return;
    TailCtx t;
    if (DERIV) {
        t = deriv_phase(P, a, dsh);
    } else {
        const TailSmem ts = tail_layout(B, esh);
        t = tail_prepare(B, P.moving_bin_size, a, ts);
        if (!t.degenerate) value_slices_share(B, a, t, ts);
    }
    if (!last_to_arrive(a.sync)) return;
    // every CTA has left the barrier and is done with the histogram
    if (DERIV) deriv_fold(P, J, a, t.degenerate);
    if (threadIdx.x < 32) fold_value(B, a, t);
    if (threadIdx.x == 0) {
        a.sync[0] = 0u;
        a.sync[2] = 0u;
    }
    for (int i = threadIdx.x; i < B * B + B; i += blockDim.x) a.ghist[i] = 0ull;
}

template <bool RECORD>
__global__ void __launch_bounds__(HIST_BLOCK, HIST_MIN_BLOCKS)
k_hist(SamplerParams P, EvalArgs a) {
    extern __shared__ unsigned int sh[];
    hist_phase<RECORD>(P, a, sh);
}

// Value-only tail of the split form: one CTA.
__global__ void __launch_bounds__(TAIL_BLOCK)
k_tail(int B, double moving_bin_size, EvalArgs a) {
    extern __shared__ __align__(16) unsigned char tsh[];
    const TailSmem ts = tail_layout(B, tsh);
    const TailCtx t = tail_prepare(B, moving_bin_size, a, ts);
    if (!t.degenerate) value_slices_share(B, a, t, ts);
    __syncthreads();
    if (threadIdx.x < 32) fold_value(B, a, t);
    for (int i = threadIdx.x; i < B * B + B; i += blockDim.x) a.ghist[i] = 0ull;
}

// Tail and derivative pass of the split form.
__global__ void __launch_bounds__(DERIV_BLOCK)
k_deriv(SamplerParams P, JacobianForm J, EvalArgs a) {
    extern __shared__ double dsh[];
    const TailCtx t = deriv_phase(P, a, dsh);
    if (!last_to_arrive(a.sync)) return;
    deriv_fold(P, J, a, t.degenerate);
    if (threadIdx.x < 32) fold_value(P.bins, a, t);
    if (threadIdx.x == 0) a.sync[0] = 0u;
    for (int i = threadIdx.x; i < P.bins * P.bins + P.bins; i += blockDim.x) a.ghist[i] = 0ull;
}

// Per-sample decisions of the same sampler the kernels use, for the exactness tests.
__global__ void k_decisions(SamplerParams P, const float* __restrict__ moving,
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

void free_metric(mi_metric* m) {
    if (!m) return;
    if (m->mtex) cudaDestroyTextureObject(m->mtex);
    if (m->marray) cudaFreeArray(m->marray);
    cudaFree(m->fixed);
    cudaFree(m->moving);
    cudaFree(m->mmask);
    cudaFree(m->samples);
    cudaFree(m->fbin);
    cudaFree(m->ws.hist);
    cudaFree(m->ws.partials);
    cudaFree(m->ws.vsum);
    cudaFree(m->ws.result);
    cudaFree(m->ws.done_counter);
    cudaFree(m->ws.rec_bins);
    cudaFree(m->ws.rec_f);
    cudaFree(m->ws.rec_g);
    if (m->ws.host_result) cudaFreeHost(m->ws.host_result);
    for (int i = 0; i < 5; ++i)
        if (m->ws.ev[i]) cudaEventDestroy(m->ws.ev[i]);
    delete m;
}

// Build the sample list: the strategy's draw, gated by the fixed mask, sorted
// ascending. The histogram is a sum of exact integers and so does not depend on the
// order; sorting only buys locality.
mi_status build_samples(mi_context* ctx, mi_metric* m, const mi_image* fixed_mask, const mi_sampling* smp,
                        int64_t nvox) {
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
    if (nkept > 1) {
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

void mat3_mul(const double* a, const double* b, double* out) {
    double t[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) t[r * 3 + c] = a[r * 3] * b[c] + a[r * 3 + 1] * b[3 + c] + a[r * 3 + 2] * b[6 + c];
    std::memcpy(out, t, sizeof(t));
}

void mat3_vec(const double* a, const double* v, double* out) {
    double t[3];
    for (int r = 0; r < 3; ++r) t[r] = a[r * 3] * v[0] + a[r * 3 + 1] * v[1] + a[r * 3 + 2] * v[2];
    std::memcpy(out, t, sizeof(t));
}

// Per-evaluation sampler constants: the stages, the composite map grid index →
// continuous index, and a bound on how far that map can be from the exact chain.
mi_status fill_params(mi_metric* m, const double* stages, int nstage, SamplerParams& P) {
    P = m->base;
    P.nstage = nstage;
    for (int s = 0; s < nstage; ++s)
        for (int i = 0; i < 12; ++i) P.stage[s][i] = stages[s * 12 + i];
    // T(x) = MT·x + tT, the stages folded (for the fast path only; the exact chain
    // replays them one by one)
    double MT[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, tT[3] = {0, 0, 0};
    for (int s = 0; s < nstage; ++s) {
        const double* S = P.stage[s];
        double nm[9], nt[3];
        mat3_mul(S, MT, nm);
        mat3_vec(S, tT, nt);
        for (int d = 0; d < 3; ++d) nt[d] += S[9 + d];
        std::memcpy(MT, nm, sizeof(nm));
        std::memcpy(tT, nt, sizeof(nt));
    }
    double MTf[9], A[9], tmp[3], b[3];
    mat3_mul(MT, P.fi2p, MTf);
    mat3_mul(P.mp2i, MTf, A);
    mat3_vec(MT, P.forigin, tmp);
    for (int d = 0; d < 3; ++d) tmp[d] += tT[d] - P.morigin[d];
    mat3_vec(P.mp2i, tmp, b);
    for (int i = 0; i < 9; ++i) P.cA[i] = A[i];
    for (int d = 0; d < 3; ++d) P.cb[d] = b[d];
    // Magnitude bound of every intermediate of the exact chain, in moving voxels,
    // over the fixed grid's corners; the chain's rounding is ≲ 20·2^-53 of it and
    // cerr allows 2^-40 (≈ 400× margin).
    double cmax = 0.0;
    for (int corner = 0; corner < 8; ++corner) {
        const double idx[3] = {(corner & 1) ? (double)(P.fsize0 - 1) : 0.0,
                               (corner & 2) ? (double)(P.fsize1 - 1) : 0.0,
                               (corner & 4) ? (double)(P.fsize2 - 1) : 0.0};
        double mag[3];
        for (int r = 0; r < 3; ++r)
            mag[r] = std::fabs(P.forigin[r]) + std::fabs(P.fi2p[r * 3]) * idx[0] +
                     std::fabs(P.fi2p[r * 3 + 1]) * idx[1] + std::fabs(P.fi2p[r * 3 + 2]) * idx[2];
        for (int s = 0; s < nstage; ++s) {
            const double* S = P.stage[s];
            double nmag[3];
            for (int r = 0; r < 3; ++r)
                nmag[r] = std::fabs(S[r * 3]) * mag[0] + std::fabs(S[r * 3 + 1]) * mag[1] +
                          std::fabs(S[r * 3 + 2]) * mag[2] + std::fabs(S[9 + r]);
            std::memcpy(mag, nmag, sizeof(mag));
        }
        for (int r = 0; r < 3; ++r) mag[r] += std::fabs(P.morigin[r]);
        for (int r = 0; r < 3; ++r) {
            const double cm = std::fabs(P.mp2i[r * 3]) * mag[0] + std::fabs(P.mp2i[r * 3 + 1]) * mag[1] +
                              std::fabs(P.mp2i[r * 3 + 2]) * mag[2];
            cmax = std::max(cmax, cm);
        }
    }
    if (!std::isfinite(cmax)) return set_error(m->ctx, MI_ERR_INVALID_ARGUMENT, "non-finite point map");
    P.cerr = std::ldexp(1.0, -40) * (1.0 + cmax) * (double)(1 + nstage);
    P.ilo = -0.5 + 2.0 * P.cerr;
    P.olo = -0.5 - 2.0 * P.cerr;
    for (int d = 0; d < 3; ++d) {
        P.ihi[d] = P.mhi[d] - 2.0 * P.cerr;
        P.ohi[d] = P.mhi[d] + 2.0 * P.cerr;
    }
    P.bin_hi = (double)(P.bins - PADDING - 1);
    return MI_OK;
}

}  // namespace

mi_status evaluate(mi_metric* m, const double* stages, int nstage, const double* jac0, const double* jacc,
                   int nparams, bool want_derivative, double* value, double* derivative, int64_t* valid) {
    mi_context* ctx = m->ctx;
    if (nstage < 0 || nstage > MI_MAX_STAGES)
        return set_error(ctx, MI_ERR_POINT_MAP_STAGE_COUNT,
                         "the device replays at most " + std::to_string(MI_MAX_STAGES) + " point-map stages");
    if (nstage > 0 && !stages) return MI_ERR_INVALID_ARGUMENT;
    if (want_derivative && (nparams < 1 || nparams > MI_MAX_PARAMS || !jac0 || !jacc || !derivative))
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "bad Jacobian form");
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    SamplerParams P;
    mi_status s = fill_params(m, stages, nstage, P);
    if (s != MI_OK) return s;
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
    a.rec_bins = want_derivative ? ws.rec_bins : nullptr;
    a.rec_f = want_derivative ? ws.rec_f : nullptr;
    a.rec_g = want_derivative ? ws.rec_g : nullptr;
    a.partials = ws.partials;
    a.vsum = ws.vsum;
    a.sync = ws.done_counter;
    a.result = ws.result;
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
        if (want_derivative)
            k_hist<true><<<ws.grid_hist, HIST_BLOCK, hist_smem(B), st>>>(P, a);
        else
            k_hist<false><<<ws.grid_hist, HIST_BLOCK, hist_smem(B), st>>>(P, a);
        if (per_kernel) MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[1], st));
        if (want_derivative)
            k_deriv<<<ws.grid_deriv, DERIV_BLOCK, deriv_smem(B), st>>>(P, J, a);
        else
            k_tail<<<1, TAIL_BLOCK, tail_smem(B), st>>>(B, P.moving_bin_size, a);
        if (per_kernel) {
            MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[2], st));
            MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[3], st));
        }
    }
    MI_CHECK_CUDA(ctx, cudaGetLastError());
    MI_CHECK_CUDA(ctx, cudaMemcpyAsync(ws.host_result, ws.result, RESULT_DOUBLES * sizeof(double),
                                       cudaMemcpyDeviceToHost, st));
    if (timing) MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[4], st));
    MI_CHECK_CUDA(ctx, cudaStreamSynchronize(st));
    unsigned int err = 0;
    std::memcpy(&err, ws.host_result + RESULT_ERR, sizeof(err));
    if (err) {
        // a barrier gave up: clear the counters, the error word and the histogram
        MI_CHECK_CUDA(ctx, cudaMemsetAsync(ws.done_counter, 0, 4 * sizeof(unsigned int), st));
        MI_CHECK_CUDA(ctx, cudaMemsetAsync(ws.result, 0, RESULT_DOUBLES * sizeof(double), st));
        MI_CHECK_CUDA(ctx, cudaMemsetAsync(ws.hist, 0, (size_t)(B * B + B) * 8, st));
        MI_CHECK_CUDA(ctx, cudaStreamSynchronize(st));
        return set_error(ctx, MI_ERR_TIMEOUT, "a grid barrier of the fused evaluation timed out");
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
    for (int i = 0; i < 9; ++i) {
        P.mp2i[i] = m_p2i[i];
        P.mp2if[i] = (float)m_p2i[i];
    }
    P.has_mmask = moving_mask ? 1 : 0;
    for (int d = 0; d < 3; ++d) P.msz[d] = (int)moving->geo.size[d];
    P.ms1 = (uint32_t)P.mstride1;
    P.ms2 = (uint32_t)P.mstride2;
    {
        // the moving volume as a block-linear 3-D array behind a point-sampling,
        // clamp-to-edge, unnormalised-coordinate texture (the fast path's corner fetch)
        const cudaChannelFormatDesc fmt = cudaCreateChannelDesc<float>();
        const cudaExtent ext = make_cudaExtent((size_t)moving->geo.size[0], (size_t)moving->geo.size[1],
                                               (size_t)moving->geo.size[2]);
        TRY_CUDA(cudaMalloc3DArray(&m->marray, &fmt, ext));
        cudaMemcpy3DParms cp = {};
        cp.srcPtr = make_cudaPitchedPtr(m->moving, (size_t)moving->geo.size[0] * sizeof(float),
                                        (size_t)moving->geo.size[0], (size_t)moving->geo.size[1]);
        cp.dstArray = m->marray;
        cp.extent = ext;
        cp.kind = cudaMemcpyDeviceToDevice;
        TRY_CUDA(cudaMemcpy3DAsync(&cp, st));
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
    P.inv_moving_bin_size = 1.0 / info.moving_bin_size;
    P.fixed_nmin = info.fixed_normalized_min;
    P.moving_nmin = info.moving_normalized_min;
    P.moving_min = mmin;
    P.moving_max = mmax;
    // x_ref: the fixed grid's physical centre; x − x_ref = M_f·idx + (o_f − x_ref)
    const double mid[3] = {0.5 * (double)(P.fsize0 - 1), 0.5 * (double)(P.fsize1 - 1), 0.5 * (double)(P.fsize2 - 1)};
    for (int r = 0; r < 3; ++r) {
        P.xref[r] = P.forigin[r] + f_i2p[r * 3] * mid[0] + f_i2p[r * 3 + 1] * mid[1] + f_i2p[r * 3 + 2] * mid[2];
        P.xb[r] = (float)(P.forigin[r] - P.xref[r]);
        for (int c = 0; c < 3; ++c) P.xA[r * 3 + c] = (float)f_i2p[r * 3 + c];
    }

    // The exact fixed bin of every sample (a pure function of the fixed value).
    TRY_CUDA(cudaMalloc(&m->fbin, pad4(m->n_samples)));
    k_fixed_bins<<<grid_for(m->n_samples, 256, ctx->num_sms * 8), 256, 0, st>>>(P, m->fixed, m->samples,
                                                                              m->n_samples, m->fbin);
    TRY_CUDA(cudaGetLastError());

    // Workspace and launch shapes.
    Workspace& ws = m->ws;
    const int B = bins;
    TRY_CUDA(cudaFuncSetAttribute(k_hist<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hist_smem(B)));
    TRY_CUDA(cudaFuncSetAttribute(k_hist<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hist_smem(B)));
    TRY_CUDA(cudaFuncSetAttribute(k_deriv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)deriv_smem(B)));
    TRY_CUDA(cudaFuncSetAttribute(k_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tail_smem(B)));
    TRY_CUDA(cudaFuncSetAttribute(k_eval<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)eval_smem(B)));
    TRY_CUDA(cudaFuncSetAttribute(k_eval<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)eval_smem(B)));
    int occ_h = 0, occ_d = 0, occ_e1 = 0, occ_e0 = 0, coop = 0;
    TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_h, k_hist<true>, HIST_BLOCK, hist_smem(B)));
    TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_d, k_deriv, DERIV_BLOCK, deriv_smem(B)));
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
    ws.grid_hist = grid_for(m->n_samples, HIST_BLOCK, ctx->num_sms * std::max(occ_h, 1));
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
        const int64_t per_thread = (m->n_samples + hgrid * HIST_BLOCK - 1) / (hgrid * HIST_BLOCK);
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
    TRY_CUDA(cudaMalloc(&ws.hist, (size_t)(B * B + B) * 8));
    TRY_CUDA(cudaMemsetAsync(ws.hist, 0, (size_t)(B * B + B) * 8, st));
    // partials serve both forms: the split form's k_deriv grid and, should the form
    // be switched, the fused grid
    {
        const int pgrid = std::max(ws.grid_deriv, std::max(ws.grid_eval,
            grid_for((int64_t)pad4(m->n_samples) / 4, DERIV_BLOCK, ctx->num_sms * std::max(occ_d, 1))));
        ws.grid_split_hist = grid_for(m->n_samples, HIST_BLOCK, ctx->num_sms * std::max(occ_h, 1));
        ws.grid_split_deriv = grid_for((int64_t)pad4(m->n_samples) / 4, DERIV_BLOCK, ctx->num_sms * std::max(occ_d, 1));
        TRY_CUDA(cudaMalloc(&ws.partials, (size_t)pgrid * NMOM * 8));
    }
    TRY_CUDA(cudaMalloc(&ws.vsum, (size_t)value_slices(B) * 8));
    TRY_CUDA(cudaMalloc(&ws.result, RESULT_DOUBLES * 8));
    TRY_CUDA(cudaMalloc(&ws.done_counter, 4 * sizeof(unsigned int)));
    TRY_CUDA(cudaMemsetAsync(ws.done_counter, 0, 4 * sizeof(unsigned int), st));
    TRY_CUDA(cudaMemsetAsync(ws.result, 0, RESULT_DOUBLES * 8, st));
    TRY_CUDA(cudaMallocHost(&ws.host_result, RESULT_DOUBLES * 8));
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
    if (n < m->n_samples) return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "output arrays shorter than the sample count");
    if (nstage < 0 || nstage > MI_MAX_STAGES) return set_error(ctx, MI_ERR_POINT_MAP_STAGE_COUNT, "too many stages");
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
