// Device phases of a Mattes evaluation, shared by the single-metric kernels
// (mattes.cu) and the batched registration kernels (batch.cu): the histogram pass,
// the tail, the derivative moments and their fold. Each phase takes the range of
// samples (or four-sample groups) it walks and how the threads stride over it, so
// the same code runs over a whole metric (grid stride) or over one chunk of one pair
// (block stride).
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>

#include "internal.h"
#include "sampler.cuh"

namespace mi {
namespace {

namespace cg = cooperative_groups;

// Launch shapes: resident CTAs per SM the histogram and derivative kernels' register
// budgets are sized for.
#ifndef MI_DERIV_MIN_BLOCKS
#define MI_DERIV_MIN_BLOCKS 2
#endif
#ifndef MI_HIST_MIN_BLOCKS
#define MI_HIST_MIN_BLOCKS 2
#endif
// 1: the histogram pass's main loop issues the next sample's corner gathers before it
// finishes the current one; 0: one sample at a time.
#ifndef MI_HIST_PIPELINE
#define MI_HIST_PIPELINE 0
#endif
constexpr bool HIST_PIPELINE = MI_HIST_PIPELINE != 0;
// 1: the derivative pass requests the next group of records before accumulating the
// current one; 0: one group at a time.
#ifndef MI_DERIV_PREFETCH
#define MI_DERIV_PREFETCH 1
#endif
constexpr bool DERIV_PREFETCH = MI_DERIV_PREFETCH != 0;
// Replicas of the split form's global histogram (see EvalArgs::reps).
#ifndef MI_GHIST_REPS
#define MI_GHIST_REPS 1
#endif
constexpr int GHIST_REPS = MI_GHIST_REPS;
// Thread-block cluster size of the split form's histogram pass (its CTAs sum their
// histograms over distributed shared memory before the global flush); 1: no cluster.
#ifndef MI_HIST_CLUSTER
#define MI_HIST_CLUSTER 1
#endif
constexpr int HIST_CLUSTER = MI_HIST_CLUSTER;
// Samples whose cell the fast path cannot settle (SAMPLE_EXACT): 1 queues them and runs
// the whole exact chain after the histogram phase's main loop, 0 runs it inside the loop
// (out of line, see MI_EXACT_NOINLINE). Inside measured faster: a few exact samples per
// CTA, drained after the loop, held back the CTA's flush by their dependent loads. The
// exact value part on the corners already fetched (SAMPLE_EXACT_CELL) runs in the loop.
#ifndef MI_EXACT_DEFERRED
#define MI_EXACT_DEFERRED 0
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
// Order of a materialised sample list: 0 sorts by voxel index (x-fastest rows);
// b > 0 sorts into bricks of 2^b voxels per axis, so that a warp's samples, and the
// moving cells they map to, are spatially close. 8³ bricks measured k_hist 40.9 µs
// against 43.0 for row order on the 256³ workload (4³ and 16³ within 0.2 µs of 8³).
#ifndef MI_SAMPLE_BRICK_LOG2
#define MI_SAMPLE_BRICK_LOG2 3
#endif
constexpr int SAMPLE_BRICK_LOG2 = MI_SAMPLE_BRICK_LOG2;
// The moving volume's texture: 1 stores it 2-D layered (one layer per z slice, a cell's
// corners in two gathers) wherever the volume fits the layered limits, 0 always 3-D
// (eight point fetches).
#ifndef MI_MOVING_LAYERED
#define MI_MOVING_LAYERED 1
#endif
constexpr bool MOVING_LAYERED = MI_MOVING_LAYERED != 0;
// Threads per histogram CTA: 512 (two resident per SM) measured 0.8 µs per
// evaluation faster than 256 (four per SM) on the 256³ workload: half as many CTAs
// zero, flush and retire their histograms.
#ifndef MI_HIST_BLOCK
#define MI_HIST_BLOCK 512
#endif
constexpr int HIST_BLOCK = MI_HIST_BLOCK;
constexpr int HIST_MIN_BLOCKS = MI_HIST_MIN_BLOCKS;
// Threads per derivative CTA (at least TAIL_BLOCK: the tail's column sums use
// TAIL_BLOCK threads).
#ifndef MI_DERIV_BLOCK
#define MI_DERIV_BLOCK 256
#endif
constexpr int DERIV_BLOCK = MI_DERIV_BLOCK;
constexpr int DERIV_MIN_BLOCKS = MI_DERIV_MIN_BLOCKS;
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
// 52 KB (so that even four CTAs fit in an SM's shared memory at 32 bins).
int hist_fine_copies(int B) {
    const size_t coarse = (size_t)hist_copies(B) * hist_copy_stride(B) * sizeof(unsigned int);
    int c = MI_HIST_FINE_COPIES;
    while (c > 1 && coarse + (size_t)c * hist_fine_stride(B) * sizeof(unsigned int) > 52 * 1024) c >>= 1;
    return c;
}
// The copies, then B u64 column sums of the CTA's histogram (used when the launch
// flushes column marginals, EvalArgs::gcols).
__host__ __device__ inline size_t hist_region_bytes(int B, int copies, int fine_copies) {
    return ((size_t)copies * hist_copy_stride(B) + (size_t)fine_copies * hist_fine_stride(B)) * sizeof(unsigned int) +
           (size_t)B * sizeof(unsigned long long);
}
size_t hist_smem(int B) { return hist_region_bytes(B, hist_copies(B), hist_fine_copies(B)); }
// Shared memory of the tail (see TailSmem).
constexpr int TAIL_BLOCK = 256;
__host__ __device__ inline int tail_groups(int B) { return TAIL_BLOCK / B; }
__host__ __device__ inline size_t tail_smem(int B) {
    return ((size_t)B * B + B + (size_t)tail_groups(B) * B + B) * 8 + ((2 * (size_t)B + 7) & ~(size_t)7) + 8 +
           (size_t)2 * B * 8;
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
//   sync[0] done counter of the final phase, sync[1] arrival counter of the split
//   form's histogram pass, sync[2] grid-barrier counter of the fused kernel.
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
    unsigned long long* gcols = nullptr;  // B column sums of the joint part, flushed with it (or null)
    // The global histogram (joint, counts, column sums) in `reps` replicas, rep_stride
    // u64 apart: CTA b flushes into replica b mod reps, which spreads the flush's
    // atomics over more addresses; the split form's tail sums the replicas. 1 elsewhere.
    int reps = 1;
    uint32_t rep_stride = 0;
    uint16_t* rec_bins;  // per sample: moving bin | fixed bin << 8 (0 = not valid)
    float* rec_f;
    float* rec_g;
    double* partials;
    double* vsum;  // value slice sums (value_slices(B))
    uint32_t* exq = nullptr;  // per-CTA queues of samples handed to the exact chain (exq_cap each)
    uint32_t exq_cap = 0;
    unsigned int* sync;
    double* result;
    // mapped pinned mirror of result (or null): the split form's last kernel writes value,
    // valid, derivative and a zero error word there as well, so the host reads them
    // once the stream completes (the kernel's completion makes the stores visible) with
    // no device-to-host copy
    double* result_host = nullptr;
    // the evaluation's sequence number, written into result_host's last slot after a
    // system-scope fence once everything else is there (the host may poll it)
    unsigned long long seq = 0;
    // the brick layout (brick.cuh) of the staged-tile histogram pass: a code per padded
    // sample, the run (brick) of every chunk of 32, each run's packed brick coordinates
    // and the walk-order position of its first sample
    const uint32_t* codes = nullptr;
    const uint32_t* chunk_run = nullptr;
    const uint32_t* run_brick = nullptr;
    const uint32_t* run_start = nullptr;
    uint32_t nchunks = 0;
};
constexpr int RESULT_ERR = 2 + MI_MAX_PARAMS;  // result slot holding the error word
constexpr int RESULT_DOUBLES = RESULT_ERR + 2;
__device__ __forceinline__ unsigned int* error_word(const EvalArgs& a) {
    return reinterpret_cast<unsigned int*>(a.result + RESULT_ERR);
}

// The error word a histogram pass with staged tiles raises (sync[3], a wait that timed
// out), as the result's error slot, and cleared for the next evaluation. Run by the one
// thread that writes the value.
__device__ __forceinline__ double carry_error(const EvalArgs& a) {
    const unsigned int e = *reinterpret_cast<volatile unsigned int*>(a.sync + 3);
    if (e) a.sync[3] = 0u;
    return e ? __longlong_as_double((long long)e) : 0.0;
}

// SplitMix64's finaliser (Steele, Lea and Flood, OOPSLA 2014): a bijection of 64-bit
// words whose every output bit depends on every input bit.
__host__ __device__ inline unsigned long long publish_mix(unsigned long long h) {
    h *= 0xbf58476d1ce4e5b9ull;
    h ^= h >> 27;
    h *= 0x94d049bb133111ebull;
    h ^= h >> 31;
    return h;
}

// One published word's share of the tag: the word salted with its slot, then mixed.
__host__ __device__ inline unsigned long long publish_word(int slot, unsigned long long w) {
    return publish_mix(w ^ ((unsigned long long)(slot + 1) * 0x9e3779b97f4a7c15ull));
}

// The tag of a published result: the mixed sequence number XOR every published word's
// share (value, valid count, the np derivative components, the error word). A result
// whose words have not all arrived differs from the tag by the XOR of the late words'
// old and new shares, which is not zero but by a 2^-64 chance; a previous evaluation's
// tag carries another sequence number.
__host__ __device__ inline unsigned long long publish_tag(unsigned long long seq, const volatile unsigned long long* w,
                                                          int np) {
    unsigned long long h = publish_mix(seq);
    for (int i = 0; i < 2 + np; ++i) h ^= publish_word(i, w[i]);
    return h ^ publish_word(RESULT_ERR, w[RESULT_ERR]);
}

// The CTA's copy of the words it publishes (value, valid, derivative and, at
// RESULT_ERR, the error word), written beside the mirror's so the tag is formed from
// shared memory.
__device__ __forceinline__ double* published_words() {
    __shared__ double pub[RESULT_ERR + 1];
    return pub;
}

// Run by the whole last CTA after it has written the result into the mirror and its
// words into published_words: warp 0 writes, into the mirror's last slot, a tag that
// hashes the evaluation's sequence number with every published word (publish_tag; one
// lane per word, then an xor tree). The mirror's words may reach the host in any order
// and no system-scope fence orders them (it cost 1.8 µs of every evaluation): the host
// takes the result once the tag matches the words it reads, which a partly arrived
// result does not.
__device__ __forceinline__ void publish_seq(const EvalArgs& a, int np) {
    if (!a.result_host) return;
    __syncthreads();
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        const double* w = published_words();
        const int slot = lane < 2 + np ? lane : RESULT_ERR;
        unsigned long long h =
            lane <= 2 + np ? publish_word(slot, (unsigned long long)__double_as_longlong(w[slot])) : 0ull;
#pragma unroll
        for (int off = 16; off; off >>= 1) h ^= __shfl_xor_sync(0xffffffffu, h, off);
        if (lane == 0)
            *reinterpret_cast<volatile unsigned long long*>(a.result_host + RESULT_ERR + 1) = h ^ publish_mix(a.seq);
    }
}

// Programmatic dependent launch: the histogram pass lets the launch that follows it
// (launched with programmatic stream serialisation) be scheduled as its CTAs retire;
// that launch waits here for the histogram pass to complete, with its writes
// visible, before it reads any of them. Without the attribute the wait returns at
// once.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

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

// The samples a phase walks: [begin, end), this warp starting at begin + warp_first,
// all threads striding by `stride`.
struct SampleRange {
    uint32_t begin, end, warp_first, stride;
};
__device__ __forceinline__ SampleRange grid_samples(uint32_t n) {
    return SampleRange{0u, n, blockIdx.x * blockDim.x + (threadIdx.x & ~31u), gridDim.x * blockDim.x};
}

// The samples a histogram phase hands to the exact chain: this CTA's queue in global
// memory (sample indices, room for every sample the phase can see), drained after the
// phase's main loop. Null: the exact chain runs in the loop.
struct ExactQueue {
    uint32_t* base;
    uint32_t cap;
};

template <bool RECORD, bool CLUSTER_FLUSH = false>
__device__ __forceinline__ void hist_phase(const SamplerParams& P, const EvalArgs& a, unsigned int* sh,
                                           const SampleRange r, const ExactQueue exq = ExactQueue{nullptr, 0u}) {
    __shared__ unsigned int exq_count;
    const int B = P.bins;
    const int nb = B * B + B;
    const int copies = a.copies, fine_copies = a.fine_copies;
    const int cstride = hist_copy_stride(B);
    const int fstride = hist_fine_stride(B);
    unsigned int* sh_fine = sh + copies * cstride;
    for (int i = threadIdx.x; i < copies * cstride + fine_copies * fstride; i += blockDim.x) sh[i] = 0u;
    // the CTA's column sums follow the copies (copies·cstride + fine_copies·fstride is a
    // multiple of four words, so they are 16-byte aligned)
    unsigned long long* colacc = reinterpret_cast<unsigned long long*>(sh + copies * cstride + fine_copies * fstride);
    if (a.gcols)
        for (int i = threadIdx.x; i < B; i += blockDim.x) colacc[i] = 0ull;
    if (threadIdx.x == 0) exq_count = 0u;
    __syncthreads();
    unsigned int* sh_joint = sh;
    unsigned int* sh_fixed = sh + B * B;
    const uint32_t stride = r.stride;
    const uint32_t n = r.end, npad = a.npad;
    const float* __restrict__ moving = a.moving;
    const uint8_t* __restrict__ mmask = a.mmask;
    const uint32_t* __restrict__ samples = a.samples;
    const uint8_t* __restrict__ fbin = a.fbin;
    const float hist_scale = a.hist_scale, fine_scale = a.fine_scale;
    // The CTA keeps `copies` interleaved copies of the histogram and lane l adds into
    // copy l mod copies: neighbouring lanes, whose sorted samples usually share a bin
    // pair, then add to different addresses instead of replaying on one. The copies
    // are summed at the flush (integer adds: the order does not matter).
    const int lane = threadIdx.x & 31;
    unsigned int* my_joint = sh_joint + (lane & (copies - 1)) * cstride;
    unsigned int* my_fixed = sh_fixed + (lane & (copies - 1)) * cstride;
    unsigned int* my_fine = sh_fine + (lane & (fine_copies - 1)) * fstride;
    auto account = [&](int st, const Sample& o, uint32_t s, int fi) {
        if (st != SAMPLE_VALID) {
            if (RECORD) a.rec_bins[s] = 0;
            return;
        }
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
    // Whole warps iterate together (the loop bound is the warp's first sample).
    const uint32_t wbase = r.begin + r.warp_first;
    // A sample the fast path cannot decide goes to the exact chain: queued (or, without
    // a queue, run here, out of line: the whole chain, or only its value part on the
    // corners already fetched when just a range or Parzen decision was uncertain).
    auto settle = [&](int st, const Prep& p, uint32_t s, int fi) {
        Sample o;
        if (st == SAMPLE_VALID) st = finish_fast<RECORD>(P, p, o);
        if (st == SAMPLE_EXACT_CELL) {
            Sample e;
            st = sample_exact_cell<RECORD>(P, p.flat, p.v, e);
            account(st, e, s, fi);
        } else if (st == SAMPLE_EXACT) {
            if (exq.base) {
                exq.base[atomicAdd(&exq_count, 1u)] = s;
            } else {
                Sample e;
                st = sample_exact<RECORD>(P, p.flat, moving, mmask, e);
                account(st, e, s, fi);
            }
        } else {
            account(st, o, s, fi);
        }
    };
    if (HIST_PIPELINE) {
        // Software-pipelined: the next sample's corner gathers are issued before this
        // sample is finished, so each thread keeps two samples' gathers in flight while
        // only one sample's finish is live. The index two samples ahead and the next
        // fixed bin are requested a step earlier still.
        constexpr int NONE = -1;
        uint32_t s = wbase + lane;
        const uint32_t s1 = s + stride;
        uint32_t flat_next = s1 < n ? (samples ? __ldg(samples + s1) : s1) : 0u;
        Prep pc;
        int stc = NONE, fic = 0;
        if (s < n) {
            stc = prep_fast<RECORD>(P, samples ? __ldg(samples + s) : s, mmask, pc);
            fic = (int)__ldg(fbin + s);
        }
        for (uint32_t b = wbase; b < n; b += stride) {
            const uint32_t sn = s + stride, sn2 = sn + stride;
            const uint32_t flat_next2 = sn2 < n ? (samples ? __ldg(samples + sn2) : sn2) : 0u;
            Prep pn;
            int stn = NONE, fin = 0;
            if (sn < n) {
                fin = (int)__ldg(fbin + sn);
                stn = prep_fast<RECORD>(P, flat_next, mmask, pn);
            }
            if (stc != NONE) settle(stc, pc, s, fic);
            pc = pn;
            stc = stn;
            fic = fin;
            s = sn;
            flat_next = flat_next2;
        }
    } else {
        // The next sample's index and this sample's fixed bin are requested at the top of
        // the iteration, so their loads overlap this sample's corner gathers instead of
        // adding two memory round trips per sample.
        uint32_t s = wbase + lane;
        uint32_t flat = s < n ? (samples ? __ldg(samples + s) : s) : 0u;
        for (uint32_t b = wbase; b < n; b += stride) {
            const bool one = s < n;
            const int fi = one ? (int)__ldg(fbin + s) : 0;
            const uint32_t sn = s + stride;
            const uint32_t flat_next = sn < n ? (samples ? __ldg(samples + sn) : sn) : 0u;
            if (one) {
                Prep p;
                settle(prep_fast<RECORD>(P, flat, mmask, p), p, s, fi);
            }
            s = sn;
            flat = flat_next;
        }
    }
    if (exq.base) {
        // the queued samples through the exact chain, spread over the CTA
        __syncthreads();
        const unsigned int nq = exq_count;
        for (unsigned int q = threadIdx.x; q < nq; q += blockDim.x) {
            const uint32_t sq = __ldcg(exq.base + q);
            Sample e;
            const int st = sample_exact<RECORD>(P, samples ? __ldg(samples + sq) : sq, moving, mmask, e);
            account(st, e, sq, (int)__ldg(fbin + sq));
        }
    }
    __syncthreads();
    // this CTA's replica of the global histogram
    const size_t rep_off = (size_t)(blockIdx.x % (unsigned)a.reps) * a.rep_stride;
    unsigned long long* rep_hist = a.ghist + rep_off;
    unsigned long long* rep_cols = a.gcols ? a.gcols + rep_off : nullptr;
    if (CLUSTER_FLUSH) {
        // The CTAs of a thread-block cluster sum their histograms over distributed
        // shared memory: CTA rank r takes every bin i ≡ r (mod cluster size), reads
        // that bin's copies in every CTA of the cluster and adds the cluster's sum into
        // the global histogram once, so the global atomics are one cluster's worth, not
        // one CTA's. Integer sums: the order does not matter.
        cg::cluster_group cl = cg::this_cluster();
        const unsigned int nr = cl.num_blocks(), rank = cl.block_rank();
        cl.sync();  // every CTA's histogram is final
        for (int i = (int)(rank * blockDim.x + threadIdx.x); i < nb; i += (int)(nr * blockDim.x)) {
            unsigned long long v = 0ull, f = 0ull;
            for (unsigned int q = 0; q < nr; ++q) {
                const unsigned int* rs = cl.map_shared_rank(sh, q);
                for (int c = 0; c < copies; ++c) v += rs[c * cstride + i];
                if (i < B * B)
                    for (int c = 0; c < fine_copies; ++c) f += rs[copies * cstride + c * fstride + i];
            }
            if (i < B * B) {
                v = (v << a.fine_shift) + f;
                if (a.gcols && v) atomicAdd(&colacc[i % B], v);
            }
            if (v) atomicAdd(&rep_hist[i], v);
        }
        __syncthreads();
        if (a.gcols)
            for (int m = threadIdx.x; m < B; m += blockDim.x)
                if (colacc[m]) atomicAdd(&rep_cols[m], colacc[m]);
        cl.sync();  // no CTA leaves while another still reads its shared memory
        return;
    }
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        unsigned long long v = 0ull;
        for (int c = 0; c < copies; ++c) v += sh[c * cstride + i];
        if (i < B * B) {
            unsigned long long f = 0ull;
            for (int c = 0; c < fine_copies; ++c) f += sh_fine[c * fstride + i];
            v = (v << a.fine_shift) + f;
            if (a.gcols && v) atomicAdd(&colacc[i % B], v);
        }
        if (v) atomicAdd(&rep_hist[i], v);
    }
    if (a.gcols) {
        // column marginals of the joint part, exact integer sums like the bins
        __syncthreads();
        for (int m = threadIdx.x; m < B; m += blockDim.x)
            if (colacc[m]) atomicAdd(&rep_cols[m], colacc[m]);
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
    unsigned long long* jmin;  // 1: the least joint count whose joint probability exceeds ε
    double* lcol;              // B: ln(column sum)
    double* lfm;               // B: ln(fixed marginal)
};
__device__ __forceinline__ TailSmem tail_layout(int B, unsigned char* base) {
    TailSmem t;
    t.hist = reinterpret_cast<unsigned long long*>(base);
    t.part = t.hist + B * B + B;
    t.col = t.part + tail_groups(B) * B;
    t.okm = reinterpret_cast<uint8_t*>(t.col + B);
    t.okf = t.okm + B;
    t.jmin = reinterpret_cast<unsigned long long*>(t.okm + ((2 * B + 7) & ~7));
    t.lcol = reinterpret_cast<double*>(t.jmin + 1);
    t.lfm = t.lcol + B;
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
// The fetch: the histogram (and, when the launch flushed them, the column sums) into
// shared memory.
__device__ void tail_fetch(int B, const EvalArgs& a, const TailSmem& ts) {
    const int B2 = B * B, nb = B2 + B;
    const int nl = a.gcols ? nb + B : nb;  // the column sums follow the counts
    const unsigned long long* __restrict__ gh = a.ghist;
    const unsigned long long* __restrict__ gc = a.gcols;
    for (int i0 = threadIdx.x; i0 < nl; i0 += 8 * blockDim.x) {
        unsigned long long v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * blockDim.x;
            v[u] = i < nb ? __ldcg(gh + i) : (i < nl ? __ldcg(gc + (i - nb)) : 0ull);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * blockDim.x;
            if (i < nb)
                ts.hist[i] = v[u];
            else if (i < nl)
                ts.col[i - nb] = v[u];
        }
    }
    __syncthreads();
}

// The integer marginals' totals and the normalisers, computed by every warp from the
// column sums and fixed counts (integer sums: any order, same bits).
__device__ __forceinline__ TailCtx tail_scalars(int B, const unsigned long long* col, const unsigned long long* cnt,
                                                double hist_inv, double moving_bin_size) {
    const int lane = threadIdx.x & 31;
    TailCtx t;
    t.total = 0ull;
    t.valid = 0ull;
    for (int m = lane; m < B; m += 32) {
        t.total += col[m];
        t.valid += cnt[m];
    }
    t.total = warp_sum_u64(t.total);
    t.valid = warp_sum_u64(t.valid);
    t.dt = (double)t.total;
    t.joint_sum = t.dt * hist_inv;
    t.degenerate = t.valid == 0ull || t.joint_sum < DBL_EPSILON;
    t.n_factor = t.degenerate ? 0.0 : 1.0 / (moving_bin_size * (double)t.valid);
    return t;
}

// Column m and row m's per-margin quantities: the ε flags of the moving and fixed
// marginals (mm = col/total, fm = count/joint_sum; mattes.rs:305-320) and their
// logarithms ln(col) and ln(fm) in FP64, so that a bin's term needs one logarithm.
__device__ __forceinline__ void margin_terms(int m, const unsigned long long* col, const unsigned long long* cnt,
                                             const TailCtx& t, uint8_t* okm, uint8_t* okf, double* lcol,
                                             double* lfm) {
    const double fm = (double)cnt[m] / t.joint_sum;
    okm[m] = (double)col[m] / t.dt > DBL_EPSILON;
    okf[m] = fm > DBL_EPSILON;
    lcol[m] = log((double)col[m]);
    lfm[m] = log(fm);
}

// jp = jv/total > ε is monotone in the integer jv: its least jv, found once starting
// next to ε·total, so the table tests an integer instead of dividing.
__device__ __forceinline__ unsigned long long least_joint(double dt) {
    unsigned long long c = (unsigned long long)(DBL_EPSILON * dt);
    for (int it = 0; it < 64 && c > 0ull && (double)(c - 1ull) / dt > DBL_EPSILON; ++it) --c;
    for (int it = 0; it < 64 && !((double)c / dt > DBL_EPSILON); ++it) ++c;
    return c > 0ull ? c : 1ull;
}

// The least integer c ≥ 1 with (double)c / d > ε, for the whole calling warp (every lane
// calls it, every lane gets it): the test is monotone in c, so lanes 0..7 try eight
// candidates around ε·d at once, and the serial search (least_joint) runs only when the
// boundary is not among them.
__device__ __forceinline__ unsigned long long least_passing(double d) {
    const int lane = threadIdx.x & 31;
    const long long c0 = (long long)(DBL_EPSILON * d);
    const long long cand = c0 - 3 + lane;
    const bool pass = lane < 8 && cand >= 1 && (double)cand / d > DBL_EPSILON;
    const unsigned int hit = __ballot_sync(0xffffffffu, pass) & 0xffu;
    const int k = hit ? __ffs(hit) - 1 : 8;
    return k >= 1 && k < 8 ? (unsigned long long)(c0 - 3 + k) : least_joint(d);
}

// The rest of the tail on the fetched histogram.
__device__ TailCtx tail_finish(int B, double moving_bin_size, const EvalArgs& a, const TailSmem& ts) {
    const int B2 = B * B;
    if (!a.gcols) {
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
    }
    const unsigned long long* cnt = ts.hist + B2;
    const TailCtx t = tail_scalars(B, ts.col, cnt, a.hist_inv, moving_bin_size);
    if ((int)threadIdx.x < B) margin_terms(threadIdx.x, ts.col, cnt, t, ts.okm, ts.okf, ts.lcol, ts.lfm);
    if (threadIdx.x == blockDim.x - 1) *ts.jmin = least_joint(t.dt);
    __syncthreads();
    return t;
}

__device__ TailCtx tail_prepare(int B, double moving_bin_size, const EvalArgs& a, const TailSmem& ts) {
    tail_fetch(B, a, ts);
    return tail_finish(B, moving_bin_size, a, ts);
}

// A bin's pRatio·nFactor (mattes.rs:305-320): ln(jp/mm)·nFactor = ln(jv/col)·nFactor,
// 0 where the reference skips the bin. The table the derivative pass reads is FP32, and
// so is this entry: the logarithm of the ratio of the two exact integer counts, taken
// with the fast reciprocal and logf (a few units of 2^-24). Forming it in FP64 cost every
// derivative CTA 4 µs of FP64 logarithms on the 32-bin workload; in FP32 the table
// differs from the FP64 one by ≤ 4·10⁻⁷ of its largest entry, which moves the
// derivative by far less than the FP32 per-sample arithmetic already does. The value's
// logarithms stay FP64 (value_term).
__device__ __forceinline__ float pr_entry(bool take, unsigned long long jv, unsigned long long col, float nf) {
    return take ? logf(__fdividef((float)jv, (float)col)) * nf : 0.0f;
}

// pRatio·nFactor of every bin into pr (shared memory). The entry's (row, column)
// advance with the thread's stride, so no per-entry division.
__device__ void pr_table(int B, const TailCtx& t, const TailSmem& ts, float* pr) {
    const int B2 = B * B;
    const unsigned long long jmin = *ts.jmin;
    int f = (int)threadIdx.x / B, m = (int)threadIdx.x - f * B;
    const int df = (int)blockDim.x / B, dm = (int)blockDim.x - df * B;
    const float nf = (float)t.n_factor;
    for (int i = threadIdx.x; i < B2; i += blockDim.x) {
        const unsigned long long jv = ts.hist[i];
        pr[i] = pr_entry(ts.okf[f] && ts.okm[m] && jv >= jmin, jv, ts.col[m], nf);
        f += df;
        m += dm;
        if (m >= B) {
            m -= B;
            ++f;
        }
    }
}

// −MI is summed in value slices of 32 bins, one warp each (lane l takes bin
// 32·s + l, then a fixed xor tree), and the slice sums are folded in slice order
// (fold_value). Whichever warp of whichever kernel computes a slice, it gets the
// same bits, so every launch form reports the same value.
__host__ __device__ inline int value_slices(int B) { return (B * B + 31) / 32; }

// One bin's term of −MI's sum, jp·(ln(jp/mm) − ln fm) with jp/mm = jv/col, formed in
// FP64 as (jv/total)·(ln jv − ln col − ln fm) from the margins' logarithms; 0 where the
// reference skips the bin (jp, mm or fm not above ε: `ok` holds the two marginal
// flags, jv ≥ jmin is jp > ε).
__device__ __forceinline__ double value_term(unsigned long long jv, bool take, double ljv, double lcol, double lfm,
                                             const TailCtx& t) {
    return take ? ((double)jv / t.dt) * ((ljv - lcol) - lfm) : 0.0;
}

__device__ __forceinline__ double slice_sum(double term) {
#pragma unroll
    for (int off = 16; off; off >>= 1) term += __shfl_xor_sync(0xffffffffu, term, off);
    return term;
}

__device__ double value_slice(int B, const TailCtx& t, const TailSmem& ts, int slice) {
    const int lane = threadIdx.x & 31;
    const int i = slice * 32 + lane;
    double term = 0.0;
    if (i < B * B) {
        const int f = i / B, m = i - f * B;
        const unsigned long long jv = ts.hist[i];
        const bool take = ts.okf[f] && ts.okm[m] && jv >= *ts.jmin;
        term = value_term(jv, take, take ? log((double)jv) : 0.0, ts.lcol[m], ts.lfm[f], t);
    }
    return slice_sum(term);
}

// This CTA's share of the value slices: with the CTAs numbered 0..units−1 (this one
// `unit`), warp w of CTA u takes slices w·units + u, then W further on (W = all
// warps), so a launch of many CTAs gives at most one slice to a warp and the slices
// land on different CTAs; the sums go to a.vsum.
__device__ void value_slices_share(int B, const EvalArgs& a, const TailCtx& t, const TailSmem& ts, int unit,
                                   int units) {
    const int lane = threadIdx.x & 31;
    const int nw = blockDim.x >> 5;
    const int ns = value_slices(B);
    for (int s = (threadIdx.x >> 5) * units + unit; s < ns; s += units * nw) {
        const double v = value_slice(B, t, ts, s);
        if (lane == 0) a.vsum[s] = v;
    }
}

// One warp: −MI from the slice sums in slice order (lane-strided, then a fixed xor
// tree).
__device__ __forceinline__ double fold_slices(const double* vs, int ns, bool global) {
    const int lane = threadIdx.x & 31;
    double v = 0.0;
    for (int s = lane; s < ns; s += 32) v += global ? __ldcg(vs + s) : vs[s];
#pragma unroll
    for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}


// One warp: value and valid into result (lane 0), from the slice sums.
__device__ void fold_value(int B, const EvalArgs& a, const TailCtx& t) {
    const int lane = threadIdx.x & 31;
    const double v = fold_slices(a.vsum, value_slices(B), true);
    if (lane == 0) {
        const double r0 = t.degenerate ? DBL_MAX : -v, r1 = (double)t.valid;
        a.result[0] = r0;
        a.result[1] = r1;
        if (a.result_host) {
            const double e = carry_error(a);  // a staged-tile wait that timed out
            a.result_host[0] = r0;
            a.result_host[1] = r1;
            a.result_host[RESULT_ERR] = e;
            published_words()[0] = r0;
            published_words()[1] = r1;
            published_words()[RESULT_ERR] = e;
        }
    }
}

// ---------------------------------------------------------------------------
// The value-only evaluation's tail, once: run by the whole CTA of the histogram pass
// that flushes last (no other CTA waits for it). It reads the finished global
// histogram from L2 once, writes value and valid into a.result and (when `mirror`)
// into the mapped mirror with the sequence number, and clears the global histogram,
// its column sums and the arrival counter for the next evaluation. Every quantity is
// formed by the same functions as the other tails (tail_scalars, margin_terms,
// least_joint, value_term, slice_sum, fold_slices), so the value has the same bits in
// every launch form.
// ---------------------------------------------------------------------------
__host__ __device__ inline size_t tail_once_smem(int B) {
    return (size_t)4 * B * 8 + (size_t)value_slices(B) * 8 + (((size_t)2 * B + 7) & ~(size_t)7) + 8;
}

__device__ __forceinline__ void tail_once(int B, double moving_bin_size, const EvalArgs& a, unsigned char* base, bool mirror) {
    const int B2 = B * B;
    const int ns = value_slices(B);
    unsigned long long* col = reinterpret_cast<unsigned long long*>(base);
    unsigned long long* cnt = col + B;
    double* lcol = reinterpret_cast<double*>(cnt + B);
    double* lfm = lcol + B;
    double* vs = lfm + B;
    uint8_t* okm = reinterpret_cast<uint8_t*>(vs + ns);
    uint8_t* okf = okm + B;
    unsigned long long* jmin_s = reinterpret_cast<unsigned long long*>(okm + ((2 * B + 7) & ~7));
    const int lane = threadIdx.x & 31;
    const int wfirst = (int)threadIdx.x - lane;
    const int bd = (int)blockDim.x;
    // The bins go in whole warps, eight per thread per round: bin i = i0 + u·bd + lane,
    // so the warp's 32 lanes hold value slice (i0 + u·bd)/32. The first round's bins
    // are requested together with the column sums and fixed counts.
    constexpr int R = 2;
    unsigned long long jv[R];
    // each bin, count and column sum is the sum of its replicas (integers: any order)
    const int reps = a.reps;
    const size_t rs = a.rep_stride;
    auto load_round = [&](int i0) {
#pragma unroll
        for (int u = 0; u < R; ++u) {
            const int i = i0 + u * bd + lane;
            unsigned long long v = 0ull;
            if (i < B2)
                for (int r = 0; r < reps; ++r) v += __ldcg(a.ghist + r * rs + i);
            jv[u] = v;
        }
    };
    load_round(wfirst);
    for (int i = threadIdx.x; i < B; i += bd) {
        unsigned long long c = 0ull, k = 0ull;
        for (int r = 0; r < reps; ++r) {
            c += __ldcg(a.gcols + r * rs + i);
            k += __ldcg(a.ghist + r * rs + B2 + i);
        }
        col[i] = c;
        cnt[i] = k;
    }
    __syncthreads();
    const TailCtx t = tail_scalars(B, col, cnt, a.hist_inv, moving_bin_size);
    if ((int)threadIdx.x < B) margin_terms(threadIdx.x, col, cnt, t, okm, okf, lcol, lfm);
    if (threadIdx.x == blockDim.x - 1) *jmin_s = least_joint(t.dt);
    __syncthreads();
    const unsigned long long jmin = *jmin_s;
    for (int i0 = wfirst; i0 < ns * 32; i0 += R * bd) {
        if (i0 != wfirst) load_round(i0);
#pragma unroll
        for (int u = 0; u < R; ++u) {
            const int iw = i0 + u * bd;  // warp-uniform: the slice's first bin
            if (iw < ns * 32) {
                const int i = iw + lane;
                double term = 0.0;
                if (i < B2 && !t.degenerate) {
                    const int f = i / B, m = i - f * B;
                    const bool take = okf[f] && okm[m] && jv[u] >= jmin;
                    term = value_term(jv[u], take, take ? log((double)jv[u]) : 0.0, lcol[m], lfm[f], t);
                }
                term = slice_sum(term);
                if (lane == 0) vs[iw >> 5] = term;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const double v = fold_slices(vs, ns, false);
        if (lane == 0) {
            const double r0 = t.degenerate ? DBL_MAX : -v, r1 = (double)t.valid;
            a.result[0] = r0;
            a.result[1] = r1;
            if (mirror && a.result_host) {
                const double e = carry_error(a);
                a.result_host[0] = r0;
                a.result_host[1] = r1;
                a.result_host[RESULT_ERR] = e;
                published_words()[0] = r0;
                published_words()[1] = r1;
                published_words()[RESULT_ERR] = e;
            }
        }
    }
    for (int r = 0; r < reps; ++r) {
        for (int i = threadIdx.x; i < B2 + B; i += bd) a.ghist[r * rs + i] = 0ull;
        for (int i = threadIdx.x; i < B; i += bd) a.gcols[r * rs + i] = 0ull;
    }
    if (threadIdx.x == 0) a.sync[1] = 0u;
    if (mirror) publish_seq(a, 0);
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
    // the sample's offset from the fixed grid's centre in index units, exact in FP32
    const float dx[3] = {__fsub_rn((float)i, P.xmid[0]), __fsub_rn((float)j, P.xmid[1]),
                         __fsub_rn((float)k, P.xmid[2])};
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
// The four-sample groups a derivative phase walks: [begin, end), this thread starting
// at begin + first, striding by `stride`; where its moments go (partials slot s at
// part[s·part_stride]); and its share of the value slices (unit of units).
struct GroupWork {
    uint32_t begin, end, first, stride;
    double* part;
    int64_t part_stride;
    int unit, units;
};
__device__ __forceinline__ GroupWork grid_groups(const EvalArgs& a) {
    return GroupWork{0u, a.npad >> 2, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x,
                     a.partials + blockIdx.x, (int64_t)gridDim.x, (int)blockIdx.x, (int)gridDim.x};
}

// The CTA's moments, reduced in a fixed order (shuffles within a warp, then over
// warps in FP64), stored into partials slot-major, [slot][CTA], so the fold reads
// them coalesced.
__device__ __forceinline__ void store_moments(const float* acc, double* red, double* part, int64_t part_stride) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    // reduce-scatter over the warp: the 12 moments (padded to 16 slots) are halved at
    // each xor step (a lane keeps the half its step bit selects and adds its partner's
    // copy of it), so after four steps lane pair (2s, 2s + 1) holds slot s summed over
    // 16 lanes and the fifth step adds the pair: 16 shuffles instead of 60
    double x[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = i < NMOM ? (double)acc[i] : 0.0;
    int slot = 0;
#pragma unroll
    for (int h = 8, off = 16; h >= 1; h >>= 1, off >>= 1) {
        const bool hi = (lane & off) != 0;
#pragma unroll
        for (int j = 0; j < h; ++j) {
            const double keep = hi ? x[j + h] : x[j];
            const double give = hi ? x[j] : x[j + h];
            x[j] = keep + __shfl_xor_sync(0xffffffffu, give, off);
        }
        slot += hi ? h : 0;
    }
    x[0] += __shfl_xor_sync(0xffffffffu, x[0], 1);
    if ((lane & 1) == 0 && slot < NMOM) red[warp * NMOM + slot] = x[0];
    __syncthreads();
    if (threadIdx.x < NMOM) {
        double v = 0.0;
        for (int k = 0; k < nw; ++k) v += red[k * NMOM + threadIdx.x];
        part[(int64_t)threadIdx.x * part_stride] = v;
    }
}

// The record stream of a derivative phase: this thread's four-sample groups, the
// next group's loads issued before the current group is accumulated; `cur` holds the
// first group, already requested by the caller.
struct RecordGroup {
    uint2 b;
    float4 f, gx, gy, gz;
    uint4 fl;
};
__device__ __forceinline__ void load_group(const EvalArgs& a, uint32_t q, RecordGroup& g) {
    const uint32_t npad = a.npad;
    g.b = __ldcg(reinterpret_cast<const uint2*>(a.rec_bins) + q);
    g.f = __ldcg(reinterpret_cast<const float4*>(a.rec_f) + q);
    g.gx = __ldcg(reinterpret_cast<const float4*>(a.rec_g) + q);
    g.gy = __ldcg(reinterpret_cast<const float4*>(a.rec_g + npad) + q);
    g.gz = __ldcg(reinterpret_cast<const float4*>(a.rec_g + 2 * (size_t)npad) + q);
    g.fl = a.samples ? __ldg(reinterpret_cast<const uint4*>(a.samples) + q)
                     : make_uint4(4 * q, 4 * q + 1, 4 * q + 2, 4 * q + 3);
}

__device__ __forceinline__ void stream_records(const SamplerParams& P, const EvalArgs& a, const float* pr, uint32_t q,
                                               uint32_t ngroups, uint32_t stride, RecordGroup cur, float* acc) {
    const int B = P.bins;
    auto one = [&](uint32_t bins, float f, float gx, float gy, float gz, uint32_t flat) {
        if (bins & 0xffu) accumulate_moments(P, pr, B, bins & 0xffu, bins >> 8, f, gx, gy, gz, flat, acc);
    };
    if (!DERIV_PREFETCH) {
        // one group at a time (more resident CTAs carry the latency)
        while (q < ngroups) {
            one(cur.b.x & 0xffffu, cur.f.x, cur.gx.x, cur.gy.x, cur.gz.x, cur.fl.x);
            one(cur.b.x >> 16, cur.f.y, cur.gx.y, cur.gy.y, cur.gz.y, cur.fl.y);
            one(cur.b.y & 0xffffu, cur.f.z, cur.gx.z, cur.gy.z, cur.gz.z, cur.fl.z);
            one(cur.b.y >> 16, cur.f.w, cur.gx.w, cur.gy.w, cur.gz.w, cur.fl.w);
            q += stride;
            if (q < ngroups) load_group(a, q, cur);
        }
        return;
    }
    while (q < ngroups) {
        const uint32_t qn = q + stride;
        RecordGroup nxt;
        if (qn < ngroups) load_group(a, qn, nxt);
        one(cur.b.x & 0xffffu, cur.f.x, cur.gx.x, cur.gy.x, cur.gz.x, cur.fl.x);
        one(cur.b.x >> 16, cur.f.y, cur.gx.y, cur.gy.y, cur.gz.y, cur.fl.y);
        one(cur.b.y & 0xffffu, cur.f.z, cur.gx.z, cur.gy.z, cur.gz.z, cur.fl.z);
        one(cur.b.y >> 16, cur.f.w, cur.gx.w, cur.gy.w, cur.gz.w, cur.fl.w);
        cur = nxt;
        q = qn;
    }
}

// The record source of a derivative phase: how a four-sample group is requested and
// streamed. GridRecords reads the grid-index layout (sample list of flat indices);
// the brick layout's source is BrickRecords (brick.cuh).
struct GridRecords {
    using Group = RecordGroup;
    static __device__ __forceinline__ void load(const EvalArgs& a, uint32_t q, Group& g) { load_group(a, q, g); }
    static __device__ __forceinline__ void stream(const SamplerParams& P, const EvalArgs& a, const float* pr,
                                                  uint32_t q, uint32_t ngroups, uint32_t stride, Group cur,
                                                  float* acc) {
        stream_records(P, a, pr, q, ngroups, stride, cur, acc);
    }
};

template <class Src = GridRecords>
__device__ TailCtx deriv_phase(const SamplerParams& P, const EvalArgs& a, double* dsh, const GroupWork w) {
    const int B = P.bins;
    double* red = dsh;  // 32 * NMOM
    unsigned char* tbase = reinterpret_cast<unsigned char*>(dsh + 32 * NMOM);
    const TailSmem ts = tail_layout(B, tbase);
    float* pr = reinterpret_cast<float*>(tbase + tail_smem(B));  // B*B
    float acc[NMOM];
#pragma unroll
    for (int i = 0; i < NMOM; ++i) acc[i] = 0.0f;
    const uint32_t q = w.begin + w.first;
    typename Src::Group cur;
    // the histogram's loads go out first (every CTA waits on them); the first record
    // group's loads then overlap the rest of the tail
    tail_fetch(B, a, ts);
    if (q < w.end) Src::load(a, q, cur);
    const TailCtx t = tail_finish(B, P.moving_bin_size, a, ts);
    if (!t.degenerate) pr_table(B, t, ts, pr);
    __syncthreads();
    // a warp with a value slice sums it before its share of the records
    if (!t.degenerate) value_slices_share(B, a, t, ts, w.unit, w.units);
    if (!t.degenerate) Src::stream(P, a, pr, q, w.end, w.stride, cur, acc);
    store_moments(acc, red, w.part, w.part_stride);
    return t;
}

// The split form's derivative pass with its own tail. Every CTA forms the pRatio·nFactor
// table itself from the integer histogram, in one round of requests: this thread's
// bins, the column sums and fixed counts, and the first group of its records all go out
// together; the marginals' totals and the least passing joint and fixed counts follow
// in every warp (tail_scalars, least_passing), then each thread's bins' entries
// (pr_entry). The value's 32-bin
// slices are summed where they fall: the warp holding slice u in CTA u (u < the CTA
// count; the rest in CTA u mod count) forms its terms from the same logarithms
// (value_term, slice_sum) into a.vsum, and the last CTA folds them (fold_slices), so
// the value has the bits of every other form. No CTA waits for another before its
// record stream, and the histogram pass ends at its flush.
__host__ __device__ inline size_t stream_smem(int B) {
    return 32 * (size_t)NMOM * sizeof(double) + (size_t)B * B * sizeof(float) + (size_t)2 * B * 8;
}

// Returns the tail state (for the last CTA's fold).
template <class Src = GridRecords>
__device__ TailCtx stream_phase(const SamplerParams& P, const EvalArgs& a, double* dsh, const GroupWork w) {
    const int B = P.bins, B2 = B * B;
    double* red = dsh;
    float* pr = reinterpret_cast<float*>(dsh + 32 * NMOM);
    unsigned long long* col = reinterpret_cast<unsigned long long*>(pr + B2);
    unsigned long long* cnt = col + B;
    const int lane = threadIdx.x & 31;
    const int bd = (int)blockDim.x;
    const int wfirst = (int)threadIdx.x - lane;
    const int ns = value_slices(B);
    float acc[NMOM];
#pragma unroll
    for (int i = 0; i < NMOM; ++i) acc[i] = 0.0f;
    const uint32_t q = w.begin + w.first;
    // one round of requests: the first R·bd bins (bin i0 + u·bd + lane for warp base
    // i0), the margins, the first record group
    constexpr int R = 4;
    unsigned long long jv[R];
    auto load_round = [&](int i0) {
#pragma unroll
        for (int u = 0; u < R; ++u) {
            const int i = i0 + u * bd + lane;
            jv[u] = i < B2 ? __ldcg(a.ghist + i) : 0ull;
        }
    };
    load_round(wfirst);
    for (int i = threadIdx.x; i < B; i += bd) {
        col[i] = __ldcg(a.gcols + i);
        cnt[i] = __ldcg(a.ghist + B2 + i);
    }
    typename Src::Group cur;
    if (q < w.end) Src::load(a, q, cur);
    __syncthreads();
    // The pRatio table needs the ε tests of the joint counts and the margins, not the
    // margins' logarithms (those feed only the value, whose slices are summed after this
    // CTA's records). Each test (count/total > ε for a joint count or column sum,
    // count/joint_sum > ε for a fixed count; mattes.rs:305-320) is monotone in the
    // integer count, so each warp finds the two least passing counts itself
    // (least_passing) and the tests become integer compares: the table follows the
    // fetch with no further barrier.
    const TailCtx t = tail_scalars(B, col, cnt, a.hist_inv, P.moving_bin_size);
    const unsigned long long jmin = least_passing(t.dt);
    const unsigned long long fmin = least_passing(t.joint_sum);
    const float nf = (float)t.n_factor;
    {
        // this thread's bins i = wfirst + lane + k·bd (k = 0, 1, …), row f and column m
        // advanced with i
        const int df = bd / B, dm = bd - df * B;
        int f = (wfirst + lane) / B, m = wfirst + lane - f * B;
        for (int i0 = wfirst; i0 < ns * 32; i0 += R * bd) {
            if (i0 != wfirst) load_round(i0);
#pragma unroll
            for (int u = 0; u < R; ++u) {
                const int i = i0 + u * bd + lane;
                if (i < B2) {
                    const bool take = !t.degenerate && cnt[f] >= fmin && col[m] >= jmin && jv[u] >= jmin;
                    pr[i] = pr_entry(take, jv[u], col[m], nf);
                }
                f += df;
                m += dm;
                if (m >= B) {
                    m -= B;
                    ++f;
                }
            }
        }
    }
    __syncthreads();
    if (!t.degenerate) Src::stream(P, a, pr, q, w.end, w.stride, cur, acc);
    // the value slices that fall to this CTA (slices unit + units·(u + k·warps) to warp
    // u), each bin's term from the logarithms the other forms take (margin_terms,
    // value_term)
    if (!t.degenerate) {
        const int nwarp = bd >> 5;
        for (int sl = (int)(threadIdx.x >> 5) * (int)w.units + (int)w.unit; sl < ns;
             sl += nwarp * (int)w.units) {
            const int i = sl * 32 + lane;
            double term = 0.0;
            if (i < B2) {
                const int f = i / B, m = i - f * B;
                const unsigned long long v = __ldcg(a.ghist + i);
                if (cnt[f] >= fmin && col[m] >= jmin && v >= jmin) {
                    const double lcol = log((double)col[m]);
                    const double lfm = log((double)cnt[f] / t.joint_sum);
                    term = value_term(v, true, log((double)v), lcol, lfm, t);
                }
            }
            term = slice_sum(term);
            if (lane == 0) a.vsum[sl] = term;
        }
    }
    store_moments(acc, red, w.part, w.part_stride);
    return t;
}

// Run by the last CTA to finish the derivative phase: fold the `count` partials of
// each slot ([slot][count]) in a fixed order (lane l of a slot sums entries l, l+18,
// …, in batches of twenty loads issued together, so up to 360 partials per slot take
// one round trip; the 18 lane sums of a slot are then added by one warp in a fixed xor
// tree) and
// contract with the Jacobian form: ∂/∂p_k = Σ_d J(x_ref)[d][k]·A_d + Σ_{d,e} C_e[d][k]·B[d][e],
// J(x_ref) = J(0) + Σ_e x_ref,e·C_e, through one linear map of the slot sums formed
// while the partials load. The fold takes the first 216 threads; with
// WITH_VALUE the CTA's last warp (a CTA of more than 216 threads) folds the value
// slices (fold_value) meanwhile.
template <bool WITH_VALUE = false>
__device__ void deriv_fold(const SamplerParams& P, const JacobianForm& J, const EvalArgs& a, const TailCtx& tc,
                           const double* partials, unsigned int count) {
    constexpr int FOLD = 18, BATCH = 20;
    const bool degenerate = tc.degenerate;
    const int np = J.nparams;
    __shared__ double fold[FOLD * NMOM];
    __shared__ double sums[NMOM];
    __shared__ double wmap[MI_MAX_PARAMS * NMOM];
    if (threadIdx.x < FOLD * NMOM) {
        const int slot = threadIdx.x / FOLD, ln = threadIdx.x % FOLD;
        const double* src = partials + (int64_t)slot * count;
        // the first batch of loads goes out before W is formed, the rest after
        double t[BATCH];
#pragma unroll
        for (int u = 0; u < BATCH; ++u) t[u] = ln + u * FOLD < count ? __ldcg(src + ln + u * FOLD) : 0.0;
        if ((int)threadIdx.x < np * NMOM) {
            // While the loads are in flight: the derivative is linear in the 12 slot sums,
            // ∂_k = Σ_t W[k][t]·sums[t]; W composes the gradient's index→physical map (M,
            // moving physical→index, registration/metric.rs:848-861), the position's
            // x − x_ref = M_f·(idx − mid) (M_f fixed index→physical) and the Jacobian form
            // J(x) = J(0) + Σ_e x_e·C_e at x_ref:
            //   W[k][j] = Σ_d J(x_ref)[d][k]·M[j][d],
            //   W[k][3 + 3j + m] = Σ_{d,e} C_e[d][k]·M[j][d]·M_f[e][m].
            const int k = threadIdx.x / NMOM, col = threadIdx.x % NMOM;
            double w = 0.0;
            if (col < 3) {
                for (int d = 0; d < 3; ++d) {
                    double jr = J.jac0[d * np + k];
                    for (int e = 0; e < 3; ++e) jr += P.xref[e] * J.jacc[e][d * np + k];
                    w += jr * P.mp2i[col * 3 + d];
                }
            } else {
                const int j = (col - 3) / 3, m = (col - 3) % 3;
                for (int d = 0; d < 3; ++d)
                    for (int e = 0; e < 3; ++e) w += J.jacc[e][d * np + k] * (P.mp2i[j * 3 + d] * P.fi2p[e * 3 + m]);
            }
            wmap[threadIdx.x] = w;
        }
        double v = 0.0;
#pragma unroll
        for (int u = 0; u < BATCH; ++u) v += t[u];
        for (unsigned int b = ln + BATCH * FOLD; b < count; b += BATCH * FOLD) {
#pragma unroll
            for (int u = 0; u < BATCH; ++u) t[u] = b + u * FOLD < count ? __ldcg(src + b + u * FOLD) : 0.0;
#pragma unroll
            for (int u = 0; u < BATCH; ++u) v += t[u];
        }
        fold[slot * FOLD + ln] = v;
    } else if (WITH_VALUE && threadIdx.x >= blockDim.x - 32) {
        fold_value(P.bins, a, tc);
    }
    __syncthreads();
    {
        // each slot's FOLD lane sums, added by one warp in a fixed xor tree
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        for (int slot = warp; slot < NMOM; slot += nw) {
            double v = lane < FOLD ? fold[slot * FOLD + lane] : 0.0;
            v = slice_sum(v);
            if (lane == 0) sums[slot] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x < np) {
        const int k = threadIdx.x;
        double dk = 0.0;
        if (!degenerate) {
#pragma unroll
            for (int t = 0; t < NMOM; ++t) dk += wmap[k * NMOM + t] * sums[t];
        }
        a.result[2 + k] = dk;
        if (a.result_host) {
            a.result_host[2 + k] = dk;
            published_words()[2 + k] = dk;
        }
    }
}

// Arrival at the end of a kernel: returns true in the last CTA to arrive (after
// which every other CTA's global writes are visible to it). The CTA's writes are
// ordered before its arrival by the barrier and one thread's device-scope fence (the
// fence is cumulative over what the barrier ordered before it), as in a grid-wide
// barrier's arrival.
__device__ __forceinline__ bool last_to_arrive(unsigned int* counter) {
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const bool l = atomicAdd(counter, 1u) == gridDim.x - 1;
        if (l) __threadfence();
        last = l;
    }
    __syncthreads();
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

}  // namespace
}  // namespace mi
