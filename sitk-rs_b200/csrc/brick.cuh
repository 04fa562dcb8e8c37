// The brick layout of a Mattes metric's sample list, used by the histogram pass with
// TMA-staged moving tiles (tile.cuh). The walk order of the samples (build_samples) is
// brick-major: bricks of 2^bl fixed voxels per axis, then 8³ sub-bricks, then voxels.
// Each brick's run of samples is padded to whole chunks of 32, one sample per lane;
// per padded position the layout holds one 32-bit code: the sample's offset δ inside
// its brick (bl bits per axis) and its exact fixed Parzen bin above them, or BRICK_PAD.
// A chunk knows its run (chunk_run), a run its brick (run_brick, packed coordinates)
// and the walk-order position of its first sample (run_start), so a padded position p
// of run r is the walk-order sample run_start[r] + p − 32·run_chunk0[r].
#pragma once

#include <cstdint>

#include "eval_device.cuh"
#include "sampler.cuh"

namespace mi {
namespace {

constexpr uint32_t BRICK_PAD = 0xFFFFFFFFu;
constexpr int BRICK_CHUNK = 32;

// A brick's constants for one evaluation.
struct BrickBase {
    double co[3];     // c at the brick's origin (the composite map's FMA form)
    int inside;       // the whole brick maps inside the moving buffer
    uint32_t packed;  // the brick's coordinates (bx | by << 10 | bz << 20)
};

__device__ __forceinline__ void brick_origin(const SamplerParams& P, uint32_t packed, uint32_t& i0, uint32_t& j0,
                                             uint32_t& k0) {
    const int bl = P.brick_bl;
    i0 = (packed & 1023u) << bl;
    j0 = ((packed >> 10) & 1023u) << bl;
    k0 = (packed >> 20) << bl;
}

// c at the brick's origin from the composite map (prep_fast's FMA form) and whether the
// brick's whole extent (lo_ext/hi_ext, with the bound's margin) maps inside.
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

// A sample's flat fixed-grid index from its brick and code.
__device__ __forceinline__ uint32_t brick_flat(const SamplerParams& P, uint32_t packed, uint32_t code) {
    const int bl = P.brick_bl;
    const uint32_t msk = (1u << bl) - 1u;
    uint32_t i, j, k;
    brick_origin(P, packed, i, j, k);
    i += code & msk;
    j += (code >> bl) & msk;
    k += (code >> (2 * bl)) & msk;
    return i + (uint32_t)P.fsize0 * (j + (uint32_t)P.fsize1 * k);
}

// The CTA histogram of a histogram pass (hist_phase's parts: coarse and fine u32
// fixed-point copies, lane-interleaved, and the joint part's column sums), zeroed by
// brick_hist_zero and added into the global u64 histogram by brick_hist_flush;
// brick_account adds one sample's taps and writes its record, as hist_phase does.
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
        a.rec_f[s] = o.f;
        a.rec_g[s] = o.g[0];
        a.rec_g[(size_t)a.npad + s] = o.g[1];
        a.rec_g[2 * (size_t)a.npad + s] = o.g[2];
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

}  // namespace
}  // namespace mi
