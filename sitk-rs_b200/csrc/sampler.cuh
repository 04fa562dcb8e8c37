// The per-sample chain of the Mattes metric on the device: fixed-grid point →
// point-map stages → continuous index → moving mask / inside test → trilinear value
// (and gradient) → moving-range reject → Parzen bins.
//
// Two evaluations of the chain share this file.
//
// exact_index() and exact_value() compute every step that feeds a discrete decision
// (the inside test, the mask rounding, the range reject and the moving Parzen
// truncation) in FP64 with each multiply, add and divide rounded separately
// (__dmul_rn / __dadd_rn / __ddiv_rn, which nvcc never contracts into an FMA), in
// the reference host's operation order:
//   point      registration/scales.rs:259-271 (origin-seeded accumulation)
//   stages     core/matrix.rs:9-21 + transform/parametric.rs:549-553
//   index      registration/metric.rs:795-806 (origin subtracted first)
//   mask       registration/metric.rs:817-833, core/coord.rs:185-191 (floor(c+0.5))
//   inside     transform/interpolator.rs:29-34
//   trilinear  transform/interpolator.rs:103-152 (corner order, clamping, products)
//   bins       registration/mattes.rs:193-206, :464-478
// so its decisions are the host's exactly. The one liberty is the sign of an exact
// zero (a chain seeded with x rather than 0.0 + x), on which no decision depends.
//
// sample() is the fast path every kernel calls. It forms the continuous index with
// three FP64 FMAs per axis from the composite map (within cerr of the exact chain),
// interpolates in FP32, and carries a rigorous bound on how far each quantity can
// be from the exact chain's. Each decision is taken from the fast values only when
// the bound cannot straddle its threshold; otherwise the quantity is recomputed by
// the exact functions. The interpolant gradient is discontinuous across cell faces,
// so the gradient pass also recomputes c exactly whenever c lies within the bound of
// an integer. Either way the decisions and the gradient's cell equal the reference's;
// only the continuous weights (B-spline taps, gradient, fractions) carry FP32
// rounding, inside the metric's tolerance. The fixed bin is exact by construction:
// it is computed once per metric by exact arithmetic (fixed_bin()).
#pragma once

#include <cstdint>

#include "internal.h"

namespace mi {

constexpr int PADDING = 2;  // registration/mattes.rs:92


enum : int { SAMPLE_OUTSIDE = 0, SAMPLE_OUT_OF_RANGE = 1, SAMPLE_VALID = 2 };

struct Sample {
    float g[3];     // moving gradient in index space (GRAD); the physical gradient is Mᵀ·g
    float f;        // Parzen fraction: moving term − moving bin
    int mi;         // moving Parzen bin
    bool exact;     // a decision or the gradient's cell came from the exact chain
};

__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
    return (uint32_t)(((uint64_t)__umulhi(n, f.m) + n) >> f.s);
}

__device__ __forceinline__ void grid_index(const SamplerParams& P, uint32_t flat, uint32_t& i,
                                           uint32_t& j, uint32_t& k) {
    const uint32_t row = fdiv(flat, P.div0);
    i = flat - row * P.div0.d;
    k = fdiv(row, P.div1);
    j = row - k * P.div1.d;
}

__device__ __forceinline__ int parzen_bin(double term, int bins) {
    long long idx = (long long)term;  // truncation toward zero
    const long long lo = PADDING, hi = (long long)bins - PADDING - 1;
    idx = idx < lo ? lo : (idx > hi ? hi : idx);
    return (int)idx;
}

// The fixed bin of a fixed value (mattes.rs:193-206), exact.
__device__ __forceinline__ int fixed_bin(const SamplerParams& P, float fv) {
    return parzen_bin(__dsub_rn(__ddiv_rn((double)fv, P.fixed_bin_size), P.fixed_nmin), P.bins);
}

// The reference's continuous index, exact: fixed-grid point (origin-seeded), the
// stages one by one, then M·(p − origin) with the origin subtracted first.
__device__ __forceinline__ void exact_index(const SamplerParams& P, uint32_t i, uint32_t j, uint32_t k,
                                            double* c) {
    const double di = (double)i, dj = (double)j, dk = (double)k;
    double x[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        double acc = P.forigin[r];
        acc = __dadd_rn(acc, __dmul_rn(P.fi2p[r * 3 + 0], di));
        acc = __dadd_rn(acc, __dmul_rn(P.fi2p[r * 3 + 1], dj));
        acc = __dadd_rn(acc, __dmul_rn(P.fi2p[r * 3 + 2], dk));
        x[r] = acc;
    }
    double p0 = x[0], p1 = x[1], p2 = x[2];
    for (int st = 0; st < P.nstage; ++st) {
        const double* a = P.stage[st];
        double q[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double acc = __dmul_rn(a[d * 3 + 0], p0);
            acc = __dadd_rn(acc, __dmul_rn(a[d * 3 + 1], p1));
            acc = __dadd_rn(acc, __dmul_rn(a[d * 3 + 2], p2));
            q[d] = __dadd_rn(acc, a[9 + d]);
        }
        p0 = q[0];
        p1 = q[1];
        p2 = q[2];
    }
    const double e0 = __dsub_rn(p0, P.morigin[0]);
    const double e1 = __dsub_rn(p1, P.morigin[1]);
    const double e2 = __dsub_rn(p2, P.morigin[2]);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        double acc = __dmul_rn(P.mp2i[r * 3 + 0], e0);
        acc = __dadd_rn(acc, __dmul_rn(P.mp2i[r * 3 + 1], e1));
        acc = __dadd_rn(acc, __dmul_rn(P.mp2i[r * 3 + 2], e2));
        c[r] = acc;
    }
}

// The reference's trilinear value at an exact continuous index that has passed the
// inside test: weights w_d[0] = 1 − frac, w_d[1] = frac, the corner weight the host's
// running product ((w0·w1)·w2) (its leading 1.0· is exact), summed in corner order.
// The eight clamped corners it reads are left in v (corner t at bit offsets
// (t & 1, (t >> 1) & 1, t >> 2)), for a caller that also needs the gradient.
// The FP64 trilinear sum on the cell's corners v at the fractions fr (om = 1 − fr), in
// the reference's order.
__device__ __forceinline__ double exact_trilinear(const double* fr, const double* om, const float* v) {
    const double w00 = __dmul_rn(om[0], om[1]);
    const double w10 = __dmul_rn(fr[0], om[1]);
    const double w01 = __dmul_rn(om[0], fr[1]);
    const double w11 = __dmul_rn(fr[0], fr[1]);
    double mv = __dmul_rn(__dmul_rn(w00, om[2]), (double)v[0]);
    mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(w10, om[2]), (double)v[1]));
    mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(w01, om[2]), (double)v[2]));
    mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(w11, om[2]), (double)v[3]));
    mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(w00, fr[2]), (double)v[4]));
    mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(w10, fr[2]), (double)v[5]));
    mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(w01, fr[2]), (double)v[6]));
    mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(w11, fr[2]), (double)v[7]));
    return mv;
}

__device__ __forceinline__ double exact_value_corners(const SamplerParams& P, const double* c,
                                                      const float* __restrict__ moving, float* v) {
    double fr[3], om[3];
    int64_t b0[3], b1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double f = floor(c[d]);
        fr[d] = __dsub_rn(c[d], f);
        om[d] = __dsub_rn(1.0, fr[d]);
        const int64_t base = (int64_t)f;
        const int64_t hi = P.msize[d] - 1;
        b0[d] = base < 0 ? 0 : (base > hi ? hi : base);
        b1[d] = base + 1 < 0 ? 0 : (base + 1 > hi ? hi : base + 1);
    }
    const int64_t oy0 = b0[1] * P.mstride1, oy1 = b1[1] * P.mstride1;
    const int64_t oz0 = b0[2] * P.mstride2, oz1 = b1[2] * P.mstride2;
    v[0] = __ldg(moving + (b0[0] + oy0 + oz0));
    v[1] = __ldg(moving + (b1[0] + oy0 + oz0));
    v[2] = __ldg(moving + (b0[0] + oy1 + oz0));
    v[3] = __ldg(moving + (b1[0] + oy1 + oz0));
    v[4] = __ldg(moving + (b0[0] + oy0 + oz1));
    v[5] = __ldg(moving + (b1[0] + oy0 + oz1));
    v[6] = __ldg(moving + (b0[0] + oy1 + oz1));
    v[7] = __ldg(moving + (b1[0] + oy1 + oz1));
    return exact_trilinear(fr, om, v);
}

__device__ __forceinline__ double exact_value(const SamplerParams& P, const double* c,
                                              const float* __restrict__ moving) {
    float v[8];
    return exact_value_corners(P, c, moving, v);
}

// The sampler: fast path with exact fallback (see the file comment), in two stages
// so a kernel can keep several samples' gathers in flight.
//
// prep():
// 1. c from the composite map (3 FP64 FMAs per axis), within ce of the exact c.
// 2. If a geometric decision (mask rounding, inside test) could flip within ±ce, or —
//    for the gradient, which is discontinuous across cell faces — c is within ce of
//    an integer, c is recomputed exactly (exact_index) and ce becomes 0.
// 3. Geometric decisions on c; the mask byte and the eight corners are loaded.
// finish():
// 4. FP32 trilinear value (and gradient) on the cell of c, with a bound dv on its
//    distance from the reference's FP64 value.
// 5. Range reject and Parzen bin from the FP32 value when dv cannot flip them;
//    otherwise the reference's value is recomputed exactly (exact_value).
// The eight corners of the cell whose lowest corner is fl (floor of a continuous
// index that passed the inside test, so each fl[d] ∈ [−1, size − 1]), corner t at
// fl + (t & 1, (t >> 1) & 1, t >> 2), from the moving volume's texture (point
// sampling at voxel centres, clamp addressing = the clamp-to-edge of each corner).
// Layered form: tld4 on the 2-D layered texture returns the 2×2 texels of one z slice
// whose bilinear footprint covers (x, y), each clamped to the slice's edge, in the
// order (x0, y1), (x1, y1), (x1, y0), (x0, y0); at (x, y) = fl + 1 the footprint is
// exactly the cell's x0 = fl_x, y0 = fl_y. Two gathers (slices fl_z and fl_z + 1,
// clamped to the volume) replace eight point fetches.
__device__ __forceinline__ void gather_f32(cudaTextureObject_t t, int layer, float x, float y, float* g) {
    asm volatile("tld4.r.a2d.v4.f32.f32 {%0, %1, %2, %3}, [%4, {%5, %6, %7, %8}];"
                 : "=f"(g[0]), "=f"(g[1]), "=f"(g[2]), "=f"(g[3])
                 : "l"(t), "r"(layer), "f"(x), "f"(y), "f"(0.0f));
}
__device__ __forceinline__ void gather_u32(cudaTextureObject_t t, int layer, float x, float y, uint32_t* g) {
    asm volatile("tld4.r.a2d.v4.u32.f32 {%0, %1, %2, %3}, [%4, {%5, %6, %7, %8}];"
                 : "=r"(g[0]), "=r"(g[1]), "=r"(g[2]), "=r"(g[3])
                 : "l"(t), "r"(layer), "f"(x), "f"(y), "f"(0.0f));
}

__device__ __forceinline__ void fetch_corners(const SamplerParams& P, const double* fl, float* v) {
    if (P.mlayered) {
        const float x = (float)fl[0] + 1.0f, y = (float)fl[1] + 1.0f;
        const int z0 = (int)fl[2];
        const int l0 = z0 < 0 ? 0 : z0, l1 = z0 + 1 > P.msz[2] - 1 ? P.msz[2] - 1 : z0 + 1;
        if (P.mbf16) {
            uint32_t g0[4], g1[4];
            gather_u32(P.mtex, l0, x, y, g0);
            gather_u32(P.mtex, l1, x, y, g1);
            v[0] = __uint_as_float(g0[3] << 16);
            v[1] = __uint_as_float(g0[2] << 16);
            v[2] = __uint_as_float(g0[0] << 16);
            v[3] = __uint_as_float(g0[1] << 16);
            v[4] = __uint_as_float(g1[3] << 16);
            v[5] = __uint_as_float(g1[2] << 16);
            v[6] = __uint_as_float(g1[0] << 16);
            v[7] = __uint_as_float(g1[1] << 16);
        } else {
            float g0[4], g1[4];
            gather_f32(P.mtex, l0, x, y, g0);
            gather_f32(P.mtex, l1, x, y, g1);
            v[0] = g0[3];
            v[1] = g0[2];
            v[2] = g0[0];
            v[3] = g0[1];
            v[4] = g1[3];
            v[5] = g1[2];
            v[6] = g1[0];
            v[7] = g1[1];
        }
        return;
    }
    float cx[2], cy[2], cz[2];
    cx[0] = (float)fl[0] + 0.5f;
    cy[0] = (float)fl[1] + 0.5f;
    cz[0] = (float)fl[2] + 0.5f;
    cx[1] = cx[0] + 1.0f;
    cy[1] = cy[0] + 1.0f;
    cz[1] = cz[0] + 1.0f;
    if (P.mbf16) {
        // BF16 storage: the upper half of an f32, so the widening is exact
#pragma unroll
        for (int t = 0; t < 8; ++t)
            v[t] = __uint_as_float((uint32_t)tex3D<unsigned short>(P.mtex, cx[t & 1], cy[(t >> 1) & 1], cz[t >> 2])
                                   << 16);
    } else {
#pragma unroll
        for (int t = 0; t < 8; ++t) v[t] = tex3D<float>(P.mtex, cx[t & 1], cy[(t >> 1) & 1], cz[t >> 2]);
    }
}

struct Prep {
    uint32_t flat;
    float fr[3];
    float v[8];
};

// Outcome of a fast-path stage: a decision, or the sample handed to the exact chain —
// the whole chain (SAMPLE_EXACT, from prep_fast: the cell itself is uncertain), or only
// its value part on the cell the fast path fetched (SAMPLE_EXACT_CELL, from
// finish_fast: the cell, inside test and mask are certain, a range or Parzen decision
// is not).
enum : int { SAMPLE_EXACT = 3, SAMPLE_EXACT_CELL = 4 };

// prep_fast(): the fast path's first stage. c from the composite map (within cerr of
// the exact c). A sample whose inside test or mask rounding could flip within ±cerr,
// or whose c lies within cerr of an integer (the interpolant's gradient jumps across
// cell faces, so the cell must be the reference's), is handed to the exact chain
// (SAMPLE_EXACT); a sample surely outside the moving buffer, or on a masked voxel, is
// SAMPLE_OUTSIDE; otherwise the cell's fractions are kept and its eight corners
// requested (SAMPLE_VALID). The value-only and the value+derivative passes hand the
// same samples to the exact chain, so both form the same histogram bits.
template <bool GRAD, class Corners>
__device__ __forceinline__ int prep_fast_src(const SamplerParams& P, uint32_t flat, const uint8_t* __restrict__ mmask,
                                             Prep& p, Corners corners) {
    p.flat = flat;
    uint32_t i, j, k;
    grid_index(P, flat, i, j, k);
    double c[3];
    {
        const double di = (double)i, dj = (double)j, dk = (double)k;
#pragma unroll
        for (int r = 0; r < 3; ++r)
            c[r] = fma(P.cA[r * 3 + 2], dk, fma(P.cA[r * 3 + 1], dj, fma(P.cA[r * 3 + 0], di, P.cb[r])));
    }
    const double ce = P.cerr;
    bool uncertain = false;
    // inside test [−0.5, size − 0.5): the bounds ilo/ihi (surely inside) and olo/ohi
    // (surely outside) carry a margin of 2·ce
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (!(c[d] >= P.ilo && c[d] < P.ihi[d])) {
            if (c[d] < P.olo || c[d] >= P.ohi[d]) return SAMPLE_OUTSIDE;
            uncertain = true;
        }
    }
    if (P.has_mmask) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double h = c[d] + 0.5;
            if (floor(h - ce) != floor(h + ce)) uncertain = true;
        }
    }
    double fl[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        fl[d] = floor(c[d]);
        const double frd = c[d] - fl[d];
        if (frd <= ce || frd >= 1.0 - ce) uncertain = true;
        p.fr[d] = (float)frd;
    }
    if (uncertain) return SAMPLE_EXACT;
    if (P.has_mmask) {
        // decided on c (certain)
        uint32_t mflat = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double r = floor(c[d] + 0.5);
            if (!(r >= 0.0 && r < (double)P.msz[d])) return SAMPLE_OUTSIDE;
            const uint32_t ri = (uint32_t)r;
            mflat += d == 0 ? ri : (d == 1 ? ri * P.ms1 : ri * P.ms2);
        }
        if (!__ldg(mmask + mflat)) return SAMPLE_OUTSIDE;
    }
    // The eight corners of the cell of c. c passed the inside test, so floor(c) ∈
    // [−1, size − 1]; the texture's point sampling at voxel centres returns the stored
    // voxel unchanged and its clamp addressing is the reference's clamp-to-edge of each
    // corner index. (prep_fast_src takes another source of the same values.)
    corners(fl, p.v);
    return SAMPLE_VALID;
}

template <bool GRAD>
__device__ __forceinline__ int prep_fast(const SamplerParams& P, uint32_t flat, const uint8_t* __restrict__ mmask,
                                         Prep& p) {
    return prep_fast_src<GRAD>(P, flat, mmask, p, [&](const double* fl, float* v) { fetch_corners(P, fl, v); });
}

// The trilinear value at fractions fr of the cell with corners v (x-lerps, then y,
// then z) and, for GRAD, the exact gradient of the interpolant in index space.
template <bool GRAD>
__device__ __forceinline__ float trilinear(const float* v, const float* fr, float* gidx) {
    const float x00 = fmaf(fr[0], v[1] - v[0], v[0]);
    const float x10 = fmaf(fr[0], v[3] - v[2], v[2]);
    const float x01 = fmaf(fr[0], v[5] - v[4], v[4]);
    const float x11 = fmaf(fr[0], v[7] - v[6], v[6]);
    const float y0 = fmaf(fr[1], x10 - x00, x00);
    const float y1 = fmaf(fr[1], x11 - x01, x01);
    if (GRAD) {
        const float a0 = fmaf(fr[1], (v[3] - v[2]) - (v[1] - v[0]), v[1] - v[0]);
        const float a1 = fmaf(fr[1], (v[7] - v[6]) - (v[5] - v[4]), v[5] - v[4]);
        gidx[0] = fmaf(fr[2], a1 - a0, a0);
        gidx[1] = fmaf(fr[2], (x11 - x01) - (x10 - x00), x10 - x00);
        gidx[2] = y1 - y0;
    }
    return fmaf(fr[2], y1 - y0, y0);
}

// finish_fast(): the fast path's second stage. The FP32 trilinear value (and index-
// space gradient), then the range and Parzen decisions against the metric's global
// bounds (point_map_fill): |mv − v_ref| ≤ dv for every sample of the evaluation, so
//   mv < rlo_out or mv > rhi_out            surely out of range,
//   rlo_in ≤ mv ≤ rhi_in                    surely in range,
// the thresholds being the range ends ∓ the bound rounded outward to f32; and the
// Parzen term's floor is certain when floor(termf − dterm) = floor(termf + dterm)
// after the clamp to [2, bins − 3]. Anything else is SAMPLE_EXACT_CELL. Every operation is
// an explicitly rounded intrinsic, so every kernel that inlines this takes the same
// path for a sample.
template <bool GRAD>
__device__ __forceinline__ int finish_fast(const SamplerParams& P, const Prep& p, Sample& o) {
    const float mv = trilinear<GRAD>(p.v, p.fr, o.g);
    if (mv < P.rlo_out || mv > P.rhi_out) return SAMPLE_OUT_OF_RANGE;
    if (!(mv >= P.rlo_in && mv <= P.rhi_in)) return SAMPLE_EXACT_CELL;
    const float termf = __fmaf_rn(mv, P.inv_bin_f, -P.nmin_f);
    // truncation then clamp to [2, bins − 3] equals floor then clamp for every term
    // (anything below 2 clamps to 2)
    const float lo = fminf(fmaxf(floorf(__fsub_rn(termf, P.dterm)), (float)PADDING), P.bin_hi_f);
    const float hi = fminf(fmaxf(floorf(__fadd_rn(termf, P.dterm)), (float)PADDING), P.bin_hi_f);
    if (lo != hi) return SAMPLE_EXACT_CELL;
    o.mi = (int)lo;
    o.f = __fsub_rn(termf, lo);
    return SAMPLE_VALID;
}

// The exact chain for one sample, out of line (it is rare, and keeping it out of the
// callers' loops keeps their register footprint to the fast path's): the reference's
// continuous index, inside test, mask rounding, FP64 trilinear value and Parzen bin
// (every decision the host's), and, for GRAD, the FP32 index-space gradient of the
// interpolant on the eight corners the value read.
// The exact chain as a real call: the callers' loops then keep only the fast path's
// registers live, and the call's spills happen only for the rare samples that take it.
#ifndef MI_EXACT_NOINLINE
#define MI_EXACT_NOINLINE 1
#endif
#if MI_EXACT_NOINLINE
#define MI_EXACT_INLINE __noinline__
#else
#define MI_EXACT_INLINE __forceinline__
#endif
// The value part alone (sample_exact_cell: no loads) inline in its callers by default.
#ifndef MI_EXACT_CELL_NOINLINE
#define MI_EXACT_CELL_NOINLINE 0
#endif
#if MI_EXACT_CELL_NOINLINE
#define MI_EXACT_CELL_INLINE __noinline__
#else
#define MI_EXACT_CELL_INLINE __forceinline__
#endif
// The exact chain's decisions on the reference's value mvx at the exact index c of the
// cell with corners v: range reject, Parzen bin and fraction, and for GRAD the FP32
// index-space gradient of the interpolant.
template <bool GRAD>
__device__ __forceinline__ int exact_decide(const SamplerParams& P, const double* c, double mvx, const float* v,
                                            Sample& o) {
    if (mvx < P.moving_min || mvx > P.moving_max) return SAMPLE_OUT_OF_RANGE;
    if (GRAD) {
        float fr[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) fr[d] = (float)__dsub_rn(c[d], floor(c[d]));
        trilinear<true>(v, fr, o.g);
    }
    const double term = __dsub_rn(__ddiv_rn(mvx, P.moving_bin_size), P.moving_nmin);
    o.mi = parzen_bin(term, P.bins);
    o.f = (float)(term - (double)o.mi);
    return SAMPLE_VALID;
}

template <bool GRAD>
__device__ MI_EXACT_INLINE int sample_exact_ijk(const SamplerParams& P, uint32_t i, uint32_t j, uint32_t k,
                                             const float* __restrict__ moving, const uint8_t* __restrict__ mmask,
                                             Sample& o) {
    double c[3];
    exact_index(P, i, j, k, c);
#pragma unroll
    for (int d = 0; d < 3; ++d)
        if (!(c[d] >= -0.5 && c[d] < P.mhi[d])) return SAMPLE_OUTSIDE;
    if (P.has_mmask) {
        uint32_t mflat = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double r = floor(c[d] + 0.5);
            if (!(r >= 0.0 && r < (double)P.msz[d])) return SAMPLE_OUTSIDE;
            const uint32_t ri = (uint32_t)r;
            mflat += d == 0 ? ri : (d == 1 ? ri * P.ms1 : ri * P.ms2);
        }
        if (!__ldg(mmask + mflat)) return SAMPLE_OUTSIDE;
    }
    float v[8];
    const double mvx = exact_value_corners(P, c, moving, v);
    return exact_decide<GRAD>(P, c, mvx, v, o);
}

template <bool GRAD>
__device__ __forceinline__ int sample_exact(const SamplerParams& P, uint32_t flat, const float* __restrict__ moving,
                                            const uint8_t* __restrict__ mmask, Sample& o) {
    uint32_t i, j, k;
    grid_index(P, flat, i, j, k);
    return sample_exact_ijk<GRAD>(P, i, j, k, moving, mmask, o);
}

// The exact chain's value part for a sample whose cell the fast path settled
// (SAMPLE_EXACT_CELL): the fast c was at least cerr from every cell face, the inside
// test and the mask byte were certain, so the exact index lies in the same cell, passes
// the same tests, and the eight corners the fast path fetched (v, each the clamped voxel
// the reference reads) are the ones the reference's trilinear sum takes. Only the exact
// index, the FP64 sum and the decisions remain; no corner is read again.
template <bool GRAD>
__device__ MI_EXACT_CELL_INLINE int sample_exact_cell(const SamplerParams& P, uint32_t flat, const float* v, Sample& o) {
    uint32_t i, j, k;
    grid_index(P, flat, i, j, k);
    double c[3];
    exact_index(P, i, j, k, c);
    double fr[3], om[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        fr[d] = __dsub_rn(c[d], floor(c[d]));
        om[d] = __dsub_rn(1.0, fr[d]);
    }
    return exact_decide<GRAD>(P, c, exact_trilinear(fr, om, v), v, o);
}

// The whole sampler for one sample: the fast path, handing to the exact chain where it
// cannot decide. o.exact reports which path decided.
template <bool GRAD>
__device__ __forceinline__ int sample(const SamplerParams& P, uint32_t flat, const float* __restrict__ moving,
                                      const uint8_t* __restrict__ mmask, Sample& o) {
    Prep p;
    o.exact = false;
    int st = prep_fast<GRAD>(P, flat, mmask, p);
    if (st == SAMPLE_VALID) st = finish_fast<GRAD>(P, p, o);
    if (st == SAMPLE_EXACT || st == SAMPLE_EXACT_CELL) {
        Sample e;
        st = st == SAMPLE_EXACT ? sample_exact<GRAD>(P, flat, moving, mmask, e) : sample_exact_cell<GRAD>(P, flat, p.v, e);
        o = e;
        o.exact = true;
    }
    return st;
}

// The four Parzen taps of a sample. With f = term − mi ∈ [0, 1] the taps sit at
// u = m − term = −1−f, −f, 1−f, 2−f (m = mi−1 … mi+2), where the cubic B-spline
// B₃(u) and its derivative B₃′(u) (mattes.rs:96-124; ITK's BSplineKernelFunction<3>
// and BSplineDerivativeKernelFunction<3>) reduce to one polynomial piece each:
//   B₃:  (1−f)³/6, (4 − 6f² + 3f³)/6, (1 + 3f + 3f² − 3f³)/6, f³/6
//   B₃′: (1−f)²/2, 2f − 3f²/2, −1/2 − f + 3f²/2, −f²/2
// (at f = 0 and f = 1 these equal the reference's branch values). The taps are
// continuous weights, not decision inputs, and are formed in FP32.
__device__ __forceinline__ void bspline3_taps(float f, float* w) {
    const float g = 1.0f - f;
    const float f2 = f * f, f3 = f2 * f;
    w[0] = g * g * g * (1.0f / 6.0f);
    w[1] = fmaf(3.0f, f3, fmaf(-6.0f, f2, 4.0f)) * (1.0f / 6.0f);
    w[2] = fmaf(-3.0f, f3, fmaf(3.0f, f2, fmaf(3.0f, f, 1.0f))) * (1.0f / 6.0f);
    w[3] = f3 * (1.0f / 6.0f);
}

__device__ __forceinline__ void bspline3_deriv_taps(float f, float* d) {
    const float g = 1.0f - f;
    const float f2 = f * f;
    d[0] = 0.5f * g * g;
    d[1] = fmaf(-1.5f, f2, 2.0f * f);
    d[2] = fmaf(1.5f, f2, -0.5f - f);
    d[3] = -0.5f * f2;
}

}  // namespace mi
