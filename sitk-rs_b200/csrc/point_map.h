// The per-evaluation part of the sampler constants, written once for the host
// (every evaluation of a metric) and the device (the batched driver forms the next
// point map after each optimizer step): the point-map stages, the composite map from
// fixed grid index to moving continuous index used by the fast path, c ≈ cA·(i,j,k)
// + cb, and the bound cerr on its distance from the exact chain's c, with the
// inside-test margins derived from it. Same operations, same order, separately
// rounded on both sides (rsgd.h's mul/add), so both produce the same bits.
#pragma once

#include <cfloat>
#include <cmath>

#include "internal.h"
#include "rsgd.h"

namespace mi {

MI_HD inline void pm_mat3_mul(const double* a, const double* b, double* out) {
    using rsgd::add;
    using rsgd::mul;
    double t[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            t[r * 3 + c] = add(add(mul(a[r * 3], b[c]), mul(a[r * 3 + 1], b[3 + c])), mul(a[r * 3 + 2], b[6 + c]));
    for (int i = 0; i < 9; ++i) out[i] = t[i];
}

MI_HD inline void pm_mat3_vec(const double* a, const double* v, double* out) {
    using rsgd::add;
    using rsgd::mul;
    double t[3];
    for (int r = 0; r < 3; ++r) t[r] = add(add(mul(a[r * 3], v[0]), mul(a[r * 3 + 1], v[1])), mul(a[r * 3 + 2], v[2]));
    for (int i = 0; i < 3; ++i) out[i] = t[i];
}

// f32 roundings of x toward −∞ and +∞ (NaN stays NaN).
MI_HD inline float f32_down(double x) {
    float f = (float)x;
    if ((double)f > x) f = nextafterf(f, -INFINITY);
    return f;
}
MI_HD inline float f32_up(double x) {
    float f = (float)x;
    if ((double)f < x) f = nextafterf(f, INFINITY);
    return f;
}

// P holds the metric's fixed part (grids, moving image, histogram geometry); this
// fills the stage-dependent part. Returns false when the map is not finite.
MI_HD inline bool point_map_fill(SamplerParams& P, const double* stages, int nstage) {
    using rsgd::add;
    using rsgd::mul;
    using rsgd::sub;
    P.nstage = nstage;
    for (int s = 0; s < nstage; ++s)
        for (int i = 0; i < 12; ++i) P.stage[s][i] = stages[s * 12 + i];
    // T(x) = MT·x + tT, the stages folded (for the fast path only; the exact chain
    // replays them one by one)
    double MT[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, tT[3] = {0, 0, 0};
    for (int s = 0; s < nstage; ++s) {
        const double* S = P.stage[s];
        double nm[9], nt[3];
        pm_mat3_mul(S, MT, nm);
        pm_mat3_vec(S, tT, nt);
        for (int d = 0; d < 3; ++d) nt[d] = add(nt[d], S[9 + d]);
        for (int i = 0; i < 9; ++i) MT[i] = nm[i];
        for (int d = 0; d < 3; ++d) tT[d] = nt[d];
    }
    double MTf[9], A[9], tmp[3], b[3];
    pm_mat3_mul(MT, P.fi2p, MTf);
    pm_mat3_mul(P.mp2i, MTf, A);
    pm_mat3_vec(MT, P.forigin, tmp);
    for (int d = 0; d < 3; ++d) tmp[d] = add(tmp[d], sub(tT[d], P.morigin[d]));
    pm_mat3_vec(P.mp2i, tmp, b);
    for (int i = 0; i < 9; ++i) P.cA[i] = A[i];
    for (int d = 0; d < 3; ++d) P.cb[d] = b[d];
    // Magnitude bound of every intermediate of the exact chain, in moving voxels,
    // over the fixed grid's corners; the chain's rounding is ≲ 20·2^-53 of it and
    // cerr allows 2^-40 (≈ 400× margin).
    double cmax = 0.0;
    for (int corner = 0; corner < 8; ++corner) {
        const double idx[3] = {(corner & 1) ? (double)(P.fsize0 - 1) : 0.0, (corner & 2) ? (double)(P.fsize1 - 1) : 0.0,
                               (corner & 4) ? (double)(P.fsize2 - 1) : 0.0};
        double mag[3];
        for (int r = 0; r < 3; ++r)
            mag[r] = add(add(add(fabs(P.forigin[r]), mul(fabs(P.fi2p[r * 3]), idx[0])), mul(fabs(P.fi2p[r * 3 + 1]), idx[1])),
                         mul(fabs(P.fi2p[r * 3 + 2]), idx[2]));
        for (int s = 0; s < nstage; ++s) {
            const double* S = P.stage[s];
            double nmag[3];
            for (int r = 0; r < 3; ++r)
                nmag[r] = add(add(add(mul(fabs(S[r * 3]), mag[0]), mul(fabs(S[r * 3 + 1]), mag[1])),
                                  mul(fabs(S[r * 3 + 2]), mag[2])),
                              fabs(S[9 + r]));
            for (int r = 0; r < 3; ++r) mag[r] = nmag[r];
        }
        for (int r = 0; r < 3; ++r) mag[r] = add(mag[r], fabs(P.morigin[r]));
        for (int r = 0; r < 3; ++r) {
            const double cm = add(add(mul(fabs(P.mp2i[r * 3]), mag[0]), mul(fabs(P.mp2i[r * 3 + 1]), mag[1])),
                                  mul(fabs(P.mp2i[r * 3 + 2]), mag[2]));
            cmax = fmax(cmax, cm);
        }
    }
    if (!(cmax <= DBL_MAX)) return false;
    P.cerr = mul(mul(0x1p-40, add(1.0, cmax)), (double)(1 + nstage));
    {
        // the fast path's global decision bounds (sampler.cuh finish_fast), u = 2^-24,
        // M = vmax: a lerp fmaf(f, fl(b − a), a) of values within M is within 3uM of
        // a + f(b − a) (2uM from the rounded difference, uM from the FMA), and a lerp
        // passes its inputs' errors on unweighted, so the three levels give 9uM; the
        // FP32 fractions are within 2^-25 + cerr of the exact ones, each moving the value
        // by at most 2M, another 3uM + 6M·cerr. 13u covers the 12u and the reference's
        // own FP64 rounding; 16·cerr covers the brick path's 2·cerr.
        const double dv = mul(P.vmax, add(mul(16.0, P.cerr), 13.0 * 0x1p-24));
        const double rmag = fmax(fabs(P.moving_min), fabs(P.moving_max));
        const double e = add(mul(dv, 1.001), mul(add(mul(2.0, P.vmax), rmag), 0x1p-20));
        P.rlo_out = f32_down(sub(P.moving_min, e));
        P.rlo_in = f32_up(add(P.moving_min, e));
        P.rhi_in = f32_down(sub(P.moving_max, e));
        P.rhi_out = f32_up(add(P.moving_max, e));
        // |termf − term_ref| ≤ dv/binSize (the value) plus 2^-24 of each magnitude the
        // FP32 term carries (the reciprocal bin size, the normalised minimum, the FMA and
        // the rounding of termf ± dterm), each bounded by 4× here
        const double inv = P.inv_moving_bin_size;
        const double mag = add(add(add(mul(P.vmax, inv), fabs(P.moving_nmin)), (double)P.bins), 1.0);
        P.dterm = f32_up(mul(add(mul(dv, inv), mul(mag, 0x1p-22)), 1.001));
    }
    if (P.brick_bl > 0) {
        // The brick path: c = c(origin) + cA·δ by FP64 FMAs, δ ∈ [0, 2^bl)³; against the
        // grid-index FMA form it differs by a few FP64 units of the magnitudes, far
        // inside cerr's margin, so it is within 2·cerr of the exact chain.
        const double span = (double)((1 << P.brick_bl) - 1);
        const double ce = mul(2.0, P.cerr);
        for (int d = 0; d < 3; ++d) {
            double lo = 0.0, hi = 0.0;
            for (int e = 0; e < 3; ++e) {
                const double a = mul(P.cA[d * 3 + e], span);
                lo = add(lo, fmin(0.0, a));
                hi = add(hi, fmax(0.0, a));
            }
            P.lo_ext[d] = sub(lo, mul(2.0, ce));
            P.hi_ext[d] = add(hi, mul(2.0, ce));
        }
        P.face_lo = f32_up(ce);
        P.face_hi = f32_down(sub(1.0, ce));
    }
    P.ilo = add(-0.5, mul(2.0, P.cerr));
    P.olo = sub(-0.5, mul(2.0, P.cerr));
    for (int d = 0; d < 3; ++d) {
        P.ihi[d] = sub(P.mhi[d], mul(2.0, P.cerr));
        P.ohi[d] = add(P.mhi[d], mul(2.0, P.cerr));
    }
    P.bin_hi = (double)(P.bins - 3);  // bins − PADDING − 1
    return true;
}

}  // namespace mi
