// The per-sample chain of the Mattes metric on the device: fixed-grid point →
// point-map stages → continuous index → moving mask / inside test → trilinear value
// (and gradient) → moving-range reject → Parzen bins.
//
// Every step that feeds a discrete decision (the inside test, the mask rounding, the
// range reject and both Parzen truncations) is computed in FP64 with each multiply,
// add and divide rounded separately (__dmul_rn / __dadd_rn / __ddiv_rn, which nvcc
// never contracts into an FMA), in the reference host's operation order:
//   point      registration/scales.rs:259-271 (origin-seeded accumulation)
//   stages     core/matrix.rs:9-21 + transform/parametric.rs:549-553
//   index      registration/metric.rs:795-806 (origin subtracted first)
//   mask       registration/metric.rs:817-833, core/coord.rs:185-191 (floor(c+0.5))
//   inside     transform/interpolator.rs:29-34
//   trilinear  transform/interpolator.rs:103-152 (corner order, clamping, products)
//   bins       registration/mattes.rs:193-206, :464-478
// so validity and bin indices equal the host's exactly. The single liberty taken is
// the sign of an exact zero (a chain seeded with x rather than 0.0 + x), on which no
// decision depends. The interpolant gradient is not a decision input and is formed
// with FMAs.
#pragma once

#include <cstdint>

#include "internal.h"

namespace mi {

constexpr int PADDING = 2;  // registration/mattes.rs:92

enum : int { SAMPLE_OUTSIDE = 0, SAMPLE_OUT_OF_RANGE = 1, SAMPLE_VALID = 2 };

struct Sample {
    double x[3];    // fixed physical point
    double mv;      // interpolated moving value
    double mterm;   // moving Parzen term
    double g[3];    // moving physical gradient (GRAD only)
    int fi, mi;     // Parzen bins
};

__device__ __forceinline__ int parzen_bin(double term, int bins) {
    long long idx = (long long)term;  // truncation toward zero
    const long long lo = PADDING, hi = (long long)bins - PADDING - 1;
    idx = idx < lo ? lo : (idx > hi ? hi : idx);
    return (int)idx;
}

template <bool GRAD>
__device__ __forceinline__ int take_sample(const SamplerParams& P, uint32_t flat,
                                           const float* __restrict__ fixed,
                                           const float* __restrict__ moving,
                                           const uint8_t* __restrict__ mmask, Sample& o) {
    // Fixed-grid voxel of this sample (x-fastest).
    const uint32_t s0 = (uint32_t)P.fsize0, s1 = (uint32_t)P.fsize1;
    const uint32_t row = flat / s0;
    const double di = (double)(flat - row * s0);
    const uint32_t k = row / s1;
    const double dj = (double)(row - k * s1);
    const double dk = (double)k;
    double x[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        double acc = P.forigin[r];
        acc = __dadd_rn(acc, __dmul_rn(P.fi2p[r * 3 + 0], di));
        acc = __dadd_rn(acc, __dmul_rn(P.fi2p[r * 3 + 1], dj));
        acc = __dadd_rn(acc, __dmul_rn(P.fi2p[r * 3 + 2], dk));
        x[r] = acc;
    }
    // Point-map stages, each p ← mat_vec(M, p) + t.
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
        p0 = q[0]; p1 = q[1]; p2 = q[2];
    }
    // Continuous index in the moving image.
    const double e0 = __dsub_rn(p0, P.morigin[0]);
    const double e1 = __dsub_rn(p1, P.morigin[1]);
    const double e2 = __dsub_rn(p2, P.morigin[2]);
    double c[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        double acc = __dmul_rn(P.mp2i[r * 3 + 0], e0);
        acc = __dadd_rn(acc, __dmul_rn(P.mp2i[r * 3 + 1], e1));
        acc = __dadd_rn(acc, __dmul_rn(P.mp2i[r * 3 + 2], e2));
        c[r] = acc;
    }
    if (P.has_mmask) {
        int64_t mflat = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double r = floor(__dadd_rn(c[d], 0.5));
            if (!(r >= 0.0 && r < (double)P.msize[d])) return SAMPLE_OUTSIDE;
            const int64_t ri = (int64_t)r;
            mflat += d == 0 ? ri : (d == 1 ? ri * P.mstride1 : ri * P.mstride2);
        }
        if (!mmask[mflat]) return SAMPLE_OUTSIDE;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d)
        if (!(c[d] >= -0.5 && c[d] < P.mhi[d])) return SAMPLE_OUTSIDE;

    // Trilinear interpolation: weights w_d[0] = 1 − frac, w_d[1] = frac; the corner
    // weight is ((w0·w1)·w2) exactly as the host's running product (its leading
    // 1.0· is exact); the value is summed in corner order.
    double fr[3], om[3];
    int64_t b0[3], b1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double f = floor(c[d]);
        fr[d] = __dsub_rn(c[d], f);
        om[d] = __dsub_rn(1.0, fr[d]);
        const int64_t base = (int64_t)f;
        const int64_t hi = P.msize[d] - 1;
        int64_t i0 = base, i1 = base + 1;
        i0 = i0 < 0 ? 0 : (i0 > hi ? hi : i0);
        i1 = i1 < 0 ? 0 : (i1 > hi ? hi : i1);
        b0[d] = i0;
        b1[d] = i1;
    }
    const int64_t oy0 = b0[1] * P.mstride1, oy1 = b1[1] * P.mstride1;
    const int64_t oz0 = b0[2] * P.mstride2, oz1 = b1[2] * P.mstride2;
    double v[8];
    v[0] = (double)__ldg(moving + (b0[0] + oy0 + oz0));
    v[1] = (double)__ldg(moving + (b1[0] + oy0 + oz0));
    v[2] = (double)__ldg(moving + (b0[0] + oy1 + oz0));
    v[3] = (double)__ldg(moving + (b1[0] + oy1 + oz0));
    v[4] = (double)__ldg(moving + (b0[0] + oy0 + oz1));
    v[5] = (double)__ldg(moving + (b1[0] + oy0 + oz1));
    v[6] = (double)__ldg(moving + (b0[0] + oy1 + oz1));
    v[7] = (double)__ldg(moving + (b1[0] + oy1 + oz1));
    const double w00 = __dmul_rn(om[0], om[1]);
    const double w10 = __dmul_rn(fr[0], om[1]);
    const double w01 = __dmul_rn(om[0], fr[1]);
    const double w11 = __dmul_rn(fr[0], fr[1]);
    double mv = __dmul_rn(__dmul_rn(w00, om[2]), v[0]);
    mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(w10, om[2]), v[1]));
    mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(w01, om[2]), v[2]));
    mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(w11, om[2]), v[3]));
    mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(w00, fr[2]), v[4]));
    mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(w10, fr[2]), v[5]));
    mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(w01, fr[2]), v[6]));
    mv = __dadd_rn(mv, __dmul_rn(__dmul_rn(w11, fr[2]), v[7]));

    if (mv < P.moving_min || mv > P.moving_max) return SAMPLE_OUT_OF_RANGE;

    o.mv = mv;
    o.mterm = __dsub_rn(__ddiv_rn(mv, P.moving_bin_size), P.moving_nmin);
    o.mi = parzen_bin(o.mterm, P.bins);
    const double fv = (double)__ldg(fixed + flat);
    o.fi = parzen_bin(__dsub_rn(__ddiv_rn(fv, P.fixed_bin_size), P.fixed_nmin), P.bins);
    o.x[0] = x[0];
    o.x[1] = x[1];
    o.x[2] = x[2];
    if (GRAD) {
        // Exact gradient of the trilinear interpolant in index space, then
        // g_phys[d] = Σ_j g_idx[j]·M[j][d] (registration/metric.rs:848-861).
        const double gx = om[1] * om[2] * (v[1] - v[0]) + fr[1] * om[2] * (v[3] - v[2]) +
                          om[1] * fr[2] * (v[5] - v[4]) + fr[1] * fr[2] * (v[7] - v[6]);
        const double gy = om[0] * om[2] * (v[2] - v[0]) + fr[0] * om[2] * (v[3] - v[1]) +
                          om[0] * fr[2] * (v[6] - v[4]) + fr[0] * fr[2] * (v[7] - v[5]);
        const double gz = om[0] * om[1] * (v[4] - v[0]) + fr[0] * om[1] * (v[5] - v[1]) +
                          om[0] * fr[1] * (v[6] - v[2]) + fr[0] * fr[1] * (v[7] - v[3]);
#pragma unroll
        for (int d = 0; d < 3; ++d)
            o.g[d] = gx * P.mp2i[0 * 3 + d] + gy * P.mp2i[1 * 3 + d] + gz * P.mp2i[2 * 3 + d];
    }
    return SAMPLE_VALID;
}

// Cubic B-spline Parzen window B₃(u) and its derivative (mattes.rs:96-124; ITK's
// BSplineKernelFunction<3> / BSplineDerivativeKernelFunction<3>). These weights are
// not decision inputs, so FMAs are allowed.
__device__ __forceinline__ double bspline3(double u) {
    const double a = fabs(u);
    if (a < 1.0) return (4.0 - 6.0 * a * a + 3.0 * a * a * a) * (1.0 / 6.0);
    if (a < 2.0) {
        const double t = 2.0 - a;
        return t * t * t * (1.0 / 6.0);
    }
    return 0.0;
}

__device__ __forceinline__ double bspline3_deriv(double u) {
    if (u >= 0.0 && u < 1.0) return -2.0 * u + 1.5 * u * u;
    if (u > -1.0 && u < 0.0) return -2.0 * u - 1.5 * u * u;
    if (u >= 1.0 && u < 2.0) return -2.0 + 2.0 * u - 0.5 * u * u;
    if (u > -2.0 && u <= -1.0) return 2.0 + 2.0 * u + 0.5 * u * u;
    return 0.0;
}

}  // namespace mi
