// The brick path of the Mattes sampler: the single-metric evaluation's samples are
// grouped by brick of the fixed grid (2^bl voxels per axis), and each brick's samples
// are padded to whole chunks of 32, one sample per lane. Per sample the list holds one
// 32-bit code: its offset δ inside the brick (bl bits per axis) and its exact fixed
// Parzen bin above them; a padding lane holds BRICK_PAD.
//
// Per evaluation and brick, the composite map from fixed grid index to moving
// continuous index is evaluated once at the brick's origin (brick_base); per sample
// c = c(origin) + cA·δ by three FP64 FMAs per axis, within 2·cerr of the exact chain.
// The decisions are the grid-index fast path's (sampler.cuh prep_fast, finish_fast):
// a fraction within the bound of a cell face, an inside test or a mask rounding that
// could flip, a range or Parzen decision within its bound, goes to the exact FP64
// chain; a brick whose whole image lies inside the moving buffer by more than the
// bound skips the per-sample inside test. So validity, both bins and the gradient's
// cell are the reference's for every sample; only the continuous weights carry FP32
// rounding. What the layout saves is the per-sample grid-index division, the fixed-bin
// load (the bin travels in the code) and the per-sample inside test.
#pragma once

#include <cstdint>

#include "eval_device.cuh"
#include "sampler.cuh"

namespace mi {
namespace {

constexpr uint32_t BRICK_PAD = 0xFFFFFFFFu;
constexpr int BRICK_CHUNK = 32;
// 1: the histogram pass requests the next chunk's corners before finishing the current
// chunk's sample (two samples' gathers in flight per thread); 0: one at a time.
#ifndef MI_BRICK_PIPELINE
#define MI_BRICK_PIPELINE 0
#endif
constexpr bool BRICK_PIPELINE = MI_BRICK_PIPELINE != 0;

// A CTA's per-brick constants, formed once per evaluation into shared memory.
struct BrickBase {
    double co[3];     // c at the brick's origin (the composite map's FMA form)
    int inside;       // the whole brick maps inside the moving buffer
    uint32_t packed;  // the brick's coordinates (bx | by << 10 | bz << 20)
};
static_assert(sizeof(BrickBase) == 32, "two 16-byte loads per chunk");

__device__ __forceinline__ void brick_origin(const SamplerParams& P, uint32_t packed, uint32_t& i0, uint32_t& j0,
                                             uint32_t& k0) {
    const int bl = P.brick_bl;
    i0 = (packed & 1023u) << bl;
    j0 = ((packed >> 10) & 1023u) << bl;
    k0 = (packed >> 20) << bl;
}

// The brick's constants: c at its origin from the composite map (prep_fast's FMA
// form) and the inside flag from the brick's extent (lo_ext/hi_ext carry the margin).
__device__ __forceinline__ BrickBase brick_base(const SamplerParams& P, uint32_t packed) {
    uint32_t i0, j0, k0;
    brick_origin(P, packed, i0, j0, k0);
    const double o0 = (double)i0, o1 = (double)j0, o2 = (double)k0;
    BrickBase b;
    bool inside = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double co = fma(P.cA[d * 3 + 2], o2, fma(P.cA[d * 3 + 1], o1, fma(P.cA[d * 3 + 0], o0, P.cb[d])));
        b.co[d] = co;
        inside = inside && co + P.lo_ext[d] >= -0.5 && co + P.hi_ext[d] < P.mhi[d];
    }
    b.inside = inside ? 1 : 0;
    b.packed = packed;
    return b;
}

// First stage: the continuous index, the face, inside and mask decisions, the corner
// requests. SAMPLE_VALID (corners requested), SAMPLE_OUTSIDE or SAMPLE_EXACT.
template <bool MASK>
__device__ __forceinline__ int brick_prep(const SamplerParams& P, const BrickBase& b, uint32_t code,
                                          const uint8_t* __restrict__ mmask, Prep& p) {
    const int bl = P.brick_bl;
    const uint32_t msk = (1u << bl) - 1u;
    const double dx = (double)(code & msk), dy = (double)((code >> bl) & msk), dz = (double)((code >> (2 * bl)) & msk);
    double c[3], fl[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        c[d] = fma(P.cA[d * 3 + 2], dz, fma(P.cA[d * 3 + 1], dy, fma(P.cA[d * 3 + 0], dx, b.co[d])));
        fl[d] = floor(c[d]);
        p.fr[d] = (float)(c[d] - fl[d]);
    }
    // a fraction within 2·cerr of a face may belong to the next cell (the interpolant's
    // gradient jumps there)
    const float flo = fminf(fminf(p.fr[0], p.fr[1]), p.fr[2]);
    const float fhi = fmaxf(fmaxf(p.fr[0], p.fr[1]), p.fr[2]);
    if (!(flo > P.face_lo && fhi < P.face_hi)) return SAMPLE_EXACT;
    if (!b.inside) {
        bool uncertain = false;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (!(c[d] >= P.ilo && c[d] < P.ihi[d])) {
                if (c[d] < P.olo || c[d] >= P.ohi[d]) return SAMPLE_OUTSIDE;
                uncertain = true;
            }
        }
        if (uncertain) return SAMPLE_EXACT;
    }
    if (MASK) {
        // the mask voxel floor(c + 0.5) (registration/metric.rs:817-833), certain when
        // c + 0.5 is farther than 2·cerr from an integer
        const double ce = 2.0 * P.cerr;
        uint32_t mflat = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double h = c[d] + 0.5;
            const double r = floor(h);
            if (floor(h - ce) != floor(h + ce)) return SAMPLE_EXACT;
            if (!(r >= 0.0 && r < (double)P.msz[d])) return SAMPLE_OUTSIDE;
            const uint32_t ri = (uint32_t)r;
            mflat += d == 0 ? ri : (d == 1 ? ri * P.ms1 : ri * P.ms2);
        }
        if (!__ldg(mmask + mflat)) return SAMPLE_OUTSIDE;
    }
    fetch_corners(P, fl, p.v);
    return SAMPLE_VALID;
}

// A sample's grid index from its brick and code.
__device__ __forceinline__ void brick_ijk(const SamplerParams& P, uint32_t packed, uint32_t code, uint32_t& i,
                                          uint32_t& j, uint32_t& k) {
    const int bl = P.brick_bl;
    const uint32_t msk = (1u << bl) - 1u;
    brick_origin(P, packed, i, j, k);
    i += code & msk;
    j += (code >> bl) & msk;
    k += (code >> (2 * bl)) & msk;
}

// The whole brick sampler for one sample (fast path, exact chain where it cannot
// decide); o.exact reports which path decided.
template <bool GRAD>
__device__ __forceinline__ int brick_sample(const SamplerParams& P, const BrickBase& b, uint32_t code,
                                            const float* __restrict__ moving, const uint8_t* __restrict__ mmask,
                                            Sample& o) {
    Prep p;
    o.exact = false;
    int st = P.has_mmask ? brick_prep<true>(P, b, code, mmask, p) : brick_prep<false>(P, b, code, mmask, p);
    if (st == SAMPLE_VALID) st = finish_fast<GRAD>(P, p, o);
    if (st == SAMPLE_EXACT) {
        uint32_t i, j, k;
        brick_ijk(P, b.packed, code, i, j, k);
        Sample e;
        st = sample_exact_ijk<GRAD>(P, i, j, k, moving, mmask, e);
        o = e;
        o.exact = true;
    }
    return st;
}

// The chunk groups of a histogram launch: group g holds chunks g·W … g·W + W − 1 (W =
// warps per CTA, one chunk per warp), and CTA c walks the contiguous groups
// [⌊c·n/grid⌋, ⌊(c + 1)·n/grid⌋) of the n groups, so neighbouring bricks, whose moving
// footprints overlap, run on the same SM (dealing the groups out round-robin balanced
// the CTAs but measured slower: 194 against 176 µs for the 256³ whole grid, as every
// CTA then sweeps the whole volume through its caches). The CTA's brick table holds,
// group after group, the runs each group touches (tab_runs[tab_off[cta] …]), and
// chunk_entry[c] is the table entry of chunk c's brick; both are built at set-up for
// the launch's grid.
__device__ __forceinline__ void brick_groups(uint32_t ngroups, uint32_t& g0, uint32_t& g1) {
    // CTA c: groups [⌊c·n/grid⌋, ⌊(c+1)·n/grid⌋), the counts differing by at most one
    g0 = (uint32_t)(((uint64_t)blockIdx.x * ngroups) / gridDim.x);
    g1 = (uint32_t)(((uint64_t)(blockIdx.x + 1) * ngroups) / gridDim.x);
}
__device__ __forceinline__ void brick_table(const SamplerParams& P, const EvalArgs& a, BrickBase* tab) {
    const uint32_t e0 = __ldg(a.tab_off + blockIdx.x), e1 = __ldg(a.tab_off + blockIdx.x + 1);
    for (uint32_t t = threadIdx.x; t < e1 - e0; t += blockDim.x)
        tab[t] = brick_base(P, __ldg(a.run_brick + __ldg(a.tab_runs + e0 + t)));
}

// The CTA histogram of a brick-layout histogram pass (hist_phase's parts: coarse and
// fine u32 fixed-point copies, lane-interleaved, and the joint part's column sums),
// zeroed by brick_hist_zero and added into the global u64 histogram by
// brick_hist_flush; brick_account adds one sample's taps and writes its record.
struct BrickHist {
    unsigned int* joint;  // this lane's coarse copy
    unsigned int* fixed;  // this lane's fixed-count copy
    unsigned int* fine;   // this lane's fine copy
};
__device__ __forceinline__ void brick_hist_zero(const EvalArgs& a, unsigned int* sh, int B) {
    const int cstride = hist_copy_stride(B), fstride = hist_fine_stride(B);
    for (int i = threadIdx.x; i < a.copies * cstride + a.fine_copies * fstride; i += blockDim.x) sh[i] = 0u;
    unsigned long long* colacc =
        reinterpret_cast<unsigned long long*>(sh + a.copies * cstride + a.fine_copies * fstride);
    if (a.gcols)
        for (int i = threadIdx.x; i < B; i += blockDim.x) colacc[i] = 0ull;
}
__device__ __forceinline__ BrickHist brick_hist_lane(const EvalArgs& a, unsigned int* sh, int B) {
    const int cstride = hist_copy_stride(B), fstride = hist_fine_stride(B);
    const int lane = threadIdx.x & 31;
    BrickHist h;
    h.joint = sh + (lane & (a.copies - 1)) * cstride;
    h.fixed = sh + B * B + (lane & (a.copies - 1)) * cstride;
    h.fine = sh + a.copies * cstride + (lane & (a.fine_copies - 1)) * fstride;
    return h;
}
template <bool RECORD>
__device__ __forceinline__ void brick_account(const EvalArgs& a, const BrickHist& h, int B, int st, const Sample& o,
                                              uint32_t s, int fi) {
    if (st != SAMPLE_VALID) {
        if (RECORD) a.rec_bins[s] = 0;
        return;
    }
    float w[4];
    bspline3_taps(o.f, w);
    const int off = fi * B + (o.mi - 1);
    unsigned int* row = h.joint + off;
    unsigned int* frow = h.fine + off;
    // round(w·scale) by the 1.5·2^23 magic add (w·scale < 2^22 for both parts)
    atomicAdd(row + 1, __float_as_uint(fmaf(w[1], a.hist_scale, 12582912.0f)) - 0x4B400000u);
    atomicAdd(row + 2, __float_as_uint(fmaf(w[2], a.hist_scale, 12582912.0f)) - 0x4B400000u);
#pragma unroll
    for (int t = 0; t < 4; t += 3) {
        const bool fine = w[t] < FINE_LIMIT;
        atomicAdd((fine ? frow : row) + t,
                  __float_as_uint(fmaf(w[t], fine ? a.fine_scale : a.hist_scale, 12582912.0f)) - 0x4B400000u);
    }
    atomicAdd(h.fixed + fi, 1u);
    if (RECORD) {
        a.rec_bins[s] = (uint16_t)(o.mi | (fi << 8));
        a.rec4[s] = make_float4(o.g[0], o.g[1], o.g[2], o.f);
    }
}
// After the CTA's last sample (the caller synchronises the CTA first).
__device__ __forceinline__ void brick_hist_flush(const EvalArgs& a, unsigned int* sh, int B) {
    const int nb = B * B + B;
    const int copies = a.copies, fine_copies = a.fine_copies;
    const int cstride = hist_copy_stride(B), fstride = hist_fine_stride(B);
    const unsigned int* sh_fine = sh + copies * cstride;
    unsigned long long* colacc = reinterpret_cast<unsigned long long*>(sh + copies * cstride + fine_copies * fstride);
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        unsigned long long v = 0ull;
        for (int cc = 0; cc < copies; ++cc) v += sh[cc * cstride + i];
        if (i < B * B) {
            unsigned long long f = 0ull;
            for (int cc = 0; cc < fine_copies; ++cc) f += sh_fine[cc * fstride + i];
            v = (v << a.fine_shift) + f;
            if (a.gcols && v) atomicAdd(&colacc[i % B], v);
        }
        if (v) atomicAdd(&a.ghist[i], v);
    }
    if (a.gcols) {
        __syncthreads();
        for (int m = threadIdx.x; m < B; m += blockDim.x)
            if (colacc[m]) atomicAdd(&a.gcols[m], colacc[m]);
    }
}

// A sample the fast path could not take to the end: finish_fast, then the exact chain
// (out of line) where a decision is open; accounted either way. The exact chain's result
// lives in its own object so that the fast path's stays in registers.
template <bool RECORD>
__device__ __forceinline__ void brick_settle(const SamplerParams& P, const EvalArgs& a, const BrickHist& h, int st,
                                             const Prep& p, uint32_t code, uint32_t packed, uint32_t s) {
    const int fi = (int)(code >> (3 * P.brick_bl));
    Sample o;
    if (st == SAMPLE_VALID) st = finish_fast<RECORD>(P, p, o);
    if (st == SAMPLE_EXACT) {
        uint32_t i, j, k;
        brick_ijk(P, packed, code, i, j, k);
        Sample e;
        st = sample_exact_ijk<RECORD>(P, i, j, k, a.moving, a.mmask, e);
        brick_account<RECORD>(a, h, P.bins, st, e, s, fi);
    } else {
        brick_account<RECORD>(a, h, P.bins, st, o, s, fi);
    }
}

// Pass 1 over the brick layout: the CTA's chunk groups (brick_table), one sample per
// lane, the corners through the moving volume's texture.
template <bool RECORD>
__device__ __forceinline__ void brick_hist_phase(const SamplerParams& P, const EvalArgs& a, unsigned int* sh,
                                                 BrickBase* tab) {
    const int B = P.bins;
    brick_hist_zero(a, sh, B);
    brick_table(P, a, tab);
    __syncthreads();
    const uint8_t* __restrict__ mmask = a.mmask;
    const uint32_t* __restrict__ codes = a.codes;
    const int lane = threadIdx.x & 31;
    const BrickHist h = brick_hist_lane(a, sh, B);
    // this warp's chunk of each of the CTA's groups; the next group's code, run and table
    // entry are requested a group ahead
    const uint32_t nw = blockDim.x >> 5, warp = threadIdx.x >> 5;
    const uint32_t nchunks = a.nchunks;
    const uint32_t ngroups = (nchunks + nw - 1) / nw;
    const uint32_t* __restrict__ centry = a.chunk_entry;
    uint32_t g0, g1;
    brick_groups(ngroups, g0, g1);
    auto fetch = [&](uint32_t g, uint32_t& code, uint32_t& entry) {
        const uint32_t c = g * nw + warp;
        code = BRICK_PAD;
        entry = 0u;
        if (g < g1 && c < nchunks) {
            code = __ldg(codes + (size_t)c * BRICK_CHUNK + lane);
            entry = __ldg(centry + c);
        }
    };
    uint32_t g = g0;
    uint32_t code, entry;
    fetch(g, code, entry);
    if (BRICK_PIPELINE) {
        // Software-pipelined: the next group's corner gathers are requested before this
        // group's sample is finished, so a thread keeps two samples' gathers in flight.
        constexpr int NONE = -1;
        Prep pc;
        int stc = NONE;
        uint32_t pkc = 0u, codec = code;
        if (code != BRICK_PAD) {
            const BrickBase b = tab[entry];
            pkc = b.packed;
            stc = P.has_mmask ? brick_prep<true>(P, b, code, mmask, pc) : brick_prep<false>(P, b, code, mmask, pc);
        }
        uint32_t code_n, entry_n;
        fetch(g + 1, code_n, entry_n);
        for (; g < g1; ++g) {
            uint32_t code_n2, entry_n2;
            fetch(g + 2, code_n2, entry_n2);
            Prep pn;
            int stn = NONE;
            uint32_t pkn = 0u;
            if (code_n != BRICK_PAD) {
                const BrickBase b = tab[entry_n];
                pkn = b.packed;
                stn = P.has_mmask ? brick_prep<true>(P, b, code_n, mmask, pn)
                                  : brick_prep<false>(P, b, code_n, mmask, pn);
            }
            if (stc != NONE) brick_settle<RECORD>(P, a, h, stc, pc, codec, pkc, (g * nw + warp) * BRICK_CHUNK + lane);
            pc = pn;
            stc = stn;
            pkc = pkn;
            codec = code_n;
            code_n = code_n2;
            entry_n = entry_n2;
        }
    } else {
        for (; g < g1; ++g) {
            uint32_t code_n, entry_n;
            fetch(g + 1, code_n, entry_n);
            if (code != BRICK_PAD) {
                const BrickBase b = tab[entry];
                Prep p;
                const int st =
                    P.has_mmask ? brick_prep<true>(P, b, code, mmask, p) : brick_prep<false>(P, b, code, mmask, p);
                brick_settle<RECORD>(P, a, h, st, p, code, b.packed, (g * nw + warp) * BRICK_CHUNK + lane);
            }
            code = code_n;
            entry = entry_n;
        }
    }
    __syncthreads();
    brick_hist_flush(a, sh, B);
}

// Pass 2's record groups over the brick layout: four consecutive padded samples (one
// chunk holds eight groups), their codes, and their chunk's x(brick origin) − x_ref.
struct BrickGroup {
    uint2 b;
    float4 r[4];  // per sample: gx, gy, gz, Parzen fraction
    uint4 code;
    float4 xb;
};
__device__ __forceinline__ void brick_load_group(const EvalArgs& a, uint32_t q, BrickGroup& g) {
    g.b = __ldcg(reinterpret_cast<const uint2*>(a.rec_bins) + q);
#pragma unroll
    for (int u = 0; u < 4; ++u) g.r[u] = __ldcg(a.rec4 + 4 * (size_t)q + u);
    g.code = __ldg(reinterpret_cast<const uint4*>(a.codes) + q);
    g.xb = __ldg(a.chunk_xbase + (q >> 3));
}

// One record's moments: w = Σ_taps B₃′·pRatio, A[d] += w g_d, B[d][e] += w g_d dx_e.
__device__ __forceinline__ void accumulate_record(const float* pr, int B, int mi, int fi, float f, float g0, float g1,
                                                  float g2, const float* dx, float* acc) {
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

__device__ __forceinline__ void brick_stream_records(const SamplerParams& P, const EvalArgs& a, const float* pr,
                                                     uint32_t q, uint32_t ngroups, uint32_t stride, BrickGroup cur,
                                                     float* acc) {
    const int B = P.bins;
    const int bl = P.brick_bl;
    const uint32_t msk = (1u << bl) - 1u;
    auto one = [&](uint32_t bins, const float4& r, uint32_t code, const float4& xb) {
        if (bins & 0xffu) {
            const float f = r.w, gx = r.x, gy = r.y, gz = r.z;
            const float dxi = (float)(code & msk), dyi = (float)((code >> bl) & msk),
                        dzi = (float)((code >> (2 * bl)) & msk);
            float dx[3];
            dx[0] = fmaf(P.xA[2], dzi, fmaf(P.xA[1], dyi, fmaf(P.xA[0], dxi, xb.x)));
            dx[1] = fmaf(P.xA[5], dzi, fmaf(P.xA[4], dyi, fmaf(P.xA[3], dxi, xb.y)));
            dx[2] = fmaf(P.xA[8], dzi, fmaf(P.xA[7], dyi, fmaf(P.xA[6], dxi, xb.z)));
            accumulate_record(pr, B, bins & 0xffu, bins >> 8, f, gx, gy, gz, dx, acc);
        }
    };
    while (q < ngroups) {
        const uint32_t qn = q + stride;
        BrickGroup nxt;
        if (qn < ngroups) brick_load_group(a, qn, nxt);
        one(cur.b.x & 0xffffu, cur.r[0], cur.code.x, cur.xb);
        one(cur.b.x >> 16, cur.r[1], cur.code.y, cur.xb);
        one(cur.b.y & 0xffffu, cur.r[2], cur.code.z, cur.xb);
        one(cur.b.y >> 16, cur.r[3], cur.code.w, cur.xb);
        cur = nxt;
        q = qn;
    }
}

struct BrickRecords {
    using Group = BrickGroup;
    static __device__ __forceinline__ void load(const EvalArgs& a, uint32_t q, Group& g) { brick_load_group(a, q, g); }
    static __device__ __forceinline__ void stream(const SamplerParams& P, const EvalArgs& a, const float* pr,
                                                  uint32_t q, uint32_t ngroups, uint32_t stride, Group cur,
                                                  float* acc) {
        brick_stream_records(P, a, pr, q, ngroups, stride, cur, acc);
    }
};

}  // namespace
}  // namespace mi
