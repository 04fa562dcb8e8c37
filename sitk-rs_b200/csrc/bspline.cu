// The Mattes metric through a cubic B-spline free-form deformation: the reference's
// sparse-support path (registration/mattes.rs:722-796 evaluate_sparse_support) with its
// BSplineTransform (transform/bspline.rs), on the metric's own samples, masks, ranges
// and histogram geometry.
//
// A B-spline transform has no affine form, so the fast composite map of the affine
// families does not apply: every sample takes the reference's exact FP64 chain —
// fixed point (origin-seeded), the control-point grid index, the valid-region test
// with its far-limit snap, the 4³ cubic weights, the displacement summed in support
// order, the moving continuous index, mask, inside test, trilinear value — each
// operation separately rounded in the reference's order, so every sample's validity
// and both Parzen bins are the reference's exactly.
//
//   k_bs_hist   pass 1: the joint histogram (FP64 Parzen taps quantised at the metric's
//               fine unit 2^-kf, u64 shared-memory copies flushed with u64 atomics) and
//               a record per sample (bins, Parzen fraction, moving gradient).
//   k_bs_tail   one CTA: the tail from the integer histogram (value, and the
//               pRatio·nFactor table into global memory).
//   k_bs_cell_deriv  one CTA per support cell of the grid (the samples grouped by cell
//               once per grid, k_bs_cell_of + a stable radix sort): each valid sample of
//               the cell adds weight_k·∇M[d]·Σ_taps B₃′·pRatio to coefficient (d, support
//               point k) of the cell's 4³·3; the CTA sums them and adds each sum once.
//
// Each coefficient receives the sums of the (up to 64) cells that share it through
// FP64 atomics, so the derivative's last bits can differ from run to run; the value,
// the valid count and the histogram are integer-exact and repeat bitwise.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cfloat>
#include <cmath>
#include <cstring>
#include <new>

#include "internal.h"
#include "sampler.cuh"
#include "eval_device.cuh"

namespace mi {

bool invert3(const double* m, double* inv);

namespace {

constexpr int BS_BLOCK = 256;

// The control-point grid (bspline.rs:209-218) and its valid-region limits, formed on
// the host once per call with the reference's expressions.
struct BSplineDev {
    int64_t gsize[3], gstride[3], nper;
    double gorigin[3], p2i[9];
    double max_limit[3], snap_ulp[3], snap_to[3];
    int smem_coef;  // pass 1 stages the coefficients in shared memory
};

// bspline.rs:94-106, every operation separately rounded in the reference's order
__device__ __forceinline__ double bs_cubic(double u) {
    const double a = fabs(u);
    if (a < 1.0) {
        const double sq = __dmul_rn(a, a);
        return __ddiv_rn(__dadd_rn(__dsub_rn(4.0, __dmul_rn(6.0, sq)), __dmul_rn(__dmul_rn(3.0, sq), a)), 6.0);
    } else if (a < 2.0) {
        const double sq = __dmul_rn(a, a);
        return __ddiv_rn(__dsub_rn(__dadd_rn(__dsub_rn(8.0, __dmul_rn(12.0, a)), __dmul_rn(6.0, sq)), __dmul_rn(sq, a)),
                         6.0);
    }
    return 0.0;
}

// The fixed grid point, origin-seeded (registration/scales.rs:259-271)
__device__ __forceinline__ void fixed_point(const SamplerParams& P, uint32_t i, uint32_t j, uint32_t k, double* x) {
    const double di = (double)i, dj = (double)j, dk = (double)k;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        double acc = P.forigin[r];
        acc = __dadd_rn(acc, __dmul_rn(P.fi2p[r * 3 + 0], di));
        acc = __dadd_rn(acc, __dmul_rn(P.fi2p[r * 3 + 1], dj));
        acc = __dadd_rn(acc, __dmul_rn(P.fi2p[r * 3 + 2], dk));
        x[r] = acc;
    }
}

// The grid index of x (bspline.rs:488-499), the valid-region test with the far-limit
// snap (:504-520), and the 1-D weights and support start (:525-557). False outside.
__device__ __forceinline__ bool bs_locate(const BSplineDev& S, const double* x, double (*w1)[4], int64_t* start) {
    double idx[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        double acc = -0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) acc = __dadd_rn(acc, __dmul_rn(S.p2i[r * 3 + c], __dsub_rn(x[c], S.gorigin[c])));
        idx[r] = acc;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (fabs(__dsub_rn(idx[d], S.max_limit[d])) <= S.snap_ulp[d])
            idx[d] = S.snap_to[d];
        else if (idx[d] >= S.max_limit[d] || idx[d] < 1.0)
            return false;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double s = floor(__dsub_rn(__dadd_rn(idx[d], 0.5), 1.5));
        start[d] = (int64_t)s;
        double u = __dsub_rn(idx[d], s);
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            w1[d][t] = bs_cubic(u);
            u = __dsub_rn(u, 1.0);
        }
    }
    return true;
}

__device__ __forceinline__ double bs_weight(const double (*w1)[4], int k) {
    return __dmul_rn(__dmul_rn(__dmul_rn(1.0, w1[0][k & 3]), w1[1][(k >> 2) & 3]), w1[2][k >> 4]);
}

__device__ __forceinline__ int64_t bs_flat(const BSplineDev& S, const int64_t* start, int k) {
    return (start[0] + (k & 3)) * S.gstride[0] + (start[1] + ((k >> 2) & 3)) * S.gstride[1] +
           (start[2] + (k >> 4)) * S.gstride[2];
}

enum { BS_OUTSIDE = 0, BS_OUT_OF_RANGE = 1, BS_VALID = 2 };

// One sample through the B-spline transform and the moving image: status, and for a
// valid sample the moving Parzen term and bin and the moving physical gradient.
__device__ int bs_sample(const SamplerParams& P, const BSplineDev& S, const double* coef, uint32_t flat,
                         const float* __restrict__ moving, const uint8_t* __restrict__ mmask, double& term, int& mi,
                         double* g) {
    uint32_t i, j, k;
    grid_index(P, flat, i, j, k);
    double x[3], y[3];
    fixed_point(P, i, j, k, x);
    double w1[3][4];
    int64_t start[3];
    if (bs_locate(S, x, w1, start)) {
        // bspline.rs:561-585: displacement summed over the 4³ support in order
        // weight q = ((1·wx)·wy)·wz as the reference forms it: the 16 (1·wx)·wy
        // products once, then one product per support point
        double wxy[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) wxy[q] = __dmul_rn(__dmul_rn(1.0, w1[0][q & 3]), w1[1][q >> 2]);
        double disp[3] = {0.0, 0.0, 0.0};
        const int64_t base = start[0] * S.gstride[0] + start[1] * S.gstride[1] + start[2] * S.gstride[2];
#pragma unroll
        for (int tz = 0; tz < 4; ++tz) {
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const double w = __dmul_rn(wxy[q], w1[2][tz]);
                const int64_t cp = base + (q & 3) + (q >> 2) * S.gstride[1] + tz * S.gstride[2];
#pragma unroll
                for (int d = 0; d < 3; ++d) disp[d] = __dadd_rn(disp[d], __dmul_rn(w, coef[d * S.nper + cp]));
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) y[d] = __dadd_rn(x[d], disp[d]);
    } else {
#pragma unroll
        for (int d = 0; d < 3; ++d) y[d] = x[d];
    }
    // the moving continuous index (registration/metric.rs:795-806)
    const double e0 = __dsub_rn(y[0], P.morigin[0]);
    const double e1 = __dsub_rn(y[1], P.morigin[1]);
    const double e2 = __dsub_rn(y[2], P.morigin[2]);
    double c[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        double acc = __dmul_rn(P.mp2i[r * 3 + 0], e0);
        acc = __dadd_rn(acc, __dmul_rn(P.mp2i[r * 3 + 1], e1));
        acc = __dadd_rn(acc, __dmul_rn(P.mp2i[r * 3 + 2], e2));
        c[r] = acc;
    }
    if (P.has_mmask) {
        uint32_t mflat = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double r = floor(__dadd_rn(c[d], 0.5));
            if (!(r >= 0.0 && r < (double)P.msz[d])) return BS_OUTSIDE;
            const uint32_t ri = (uint32_t)r;
            mflat += d == 0 ? ri : (d == 1 ? ri * P.ms1 : ri * P.ms2);
        }
        if (!__ldg(mmask + mflat)) return BS_OUTSIDE;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d)
        if (!(c[d] >= -0.5 && c[d] < P.mhi[d])) return BS_OUTSIDE;
    // the value's eight corners serve the gradient too (the same clamped cell)
    float v[8];
    const double mv = exact_value_corners(P, c, moving, v);
    // the interpolant's exact gradient on the same cell, in FP64 (a continuous weight)
    double fl[3], fr[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        fl[d] = floor(c[d]);
        fr[d] = c[d] - fl[d];
    }
    double gi[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const int b0 = t & 1, b1 = (t >> 1) & 1, b2 = t >> 2;
        const double w0 = b0 ? fr[0] : 1.0 - fr[0], wy = b1 ? fr[1] : 1.0 - fr[1], wz = b2 ? fr[2] : 1.0 - fr[2];
        const double b = (double)v[t];
        gi[0] += (b0 ? 1.0 : -1.0) * (wy * wz) * b;
        gi[1] += (b1 ? 1.0 : -1.0) * (w0 * wz) * b;
        gi[2] += (b2 ? 1.0 : -1.0) * (w0 * wy) * b;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) g[d] = gi[0] * P.mp2i[0 * 3 + d] + gi[1] * P.mp2i[1 * 3 + d] + gi[2] * P.mp2i[2 * 3 + d];
    if (mv < P.moving_min || mv > P.moving_max) return BS_OUT_OF_RANGE;
    term = __dsub_rn(__ddiv_rn(mv, P.moving_bin_size), P.moving_nmin);
    mi = parzen_bin(term, P.bins);
    return BS_VALID;
}

// Pass 1: histogram and records. The taps are the cubic B-spline of the FP64 fraction
// f = term − bin (the same polynomial pieces as the affine path), rounded to the fine
// unit 2^-kf of the metric's global histogram.
__global__ void __launch_bounds__(BS_BLOCK) k_bs_hist(const SamplerParams P, const BSplineDev S,
                                                       const double* __restrict__ coef, const EvalArgs a,
                                                       double fscale) {
    extern __shared__ __align__(16) unsigned long long bh[];
    const int B = P.bins, nb = B * B + B;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) bh[q] = 0ull;
    // the coefficients in shared memory when they fit (the launch sized it), else global
    const double* cf = coef;
    if (S.smem_coef) {
        double* sc = reinterpret_cast<double*>(bh + ((nb + 1) & ~1));
        for (int64_t q = threadIdx.x; q < 3 * S.nper; q += blockDim.x) sc[q] = __ldg(coef + q);
        cf = sc;
    }
    __syncthreads();
    // the next sample's index and this sample's fixed bin are requested before the
    // sample is evaluated, so those loads overlap it
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t flat = s < a.n ? (a.samples ? __ldg(a.samples + s) : s) : 0u;
    for (; s < a.n; s += stride) {
        const uint32_t sn = s + stride;
        const uint32_t cur = flat;
        flat = sn < a.n ? (a.samples ? __ldg(a.samples + sn) : sn) : 0u;
        const int fi = __ldg(a.fbin + s);
        double term, g[3];
        int mi = 0;
        const int st = bs_sample(P, S, cf, cur, a.moving, a.mmask, term, mi, g);
        if (st != BS_VALID) {
            a.rec_bins[s] = 0;
            continue;
        }
        const double f = term - (double)mi, h = 1.0 - f, f2 = f * f, f3 = f2 * f;
        const double w[4] = {h * h * h / 6.0, (3.0 * f3 - 6.0 * f2 + 4.0) / 6.0,
                             (-3.0 * f3 + 3.0 * f2 + 3.0 * f + 1.0) / 6.0, f3 / 6.0};
        unsigned long long* row = bh + fi * B + (mi - 1);
#pragma unroll
        for (int t = 0; t < 4; ++t) atomicAdd(row + t, __double2ull_rn(w[t] * fscale));
        atomicAdd(bh + B * B + fi, 1ull);
        a.rec_bins[s] = (uint16_t)(mi | (fi << 8));
        a.rec_f[s] = (float)f;
        a.rec_g[s] = (float)g[0];
        a.rec_g[(size_t)a.npad + s] = (float)g[1];
        a.rec_g[2 * (size_t)a.npad + s] = (float)g[2];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nb; q += blockDim.x)
        if (bh[q]) atomicAdd(a.ghist + q, bh[q]);
}

// The support cell of every sample: its grid start (exact, as pass 1 forms it) as one
// index over the (gsize − 3)³ cells, or NO_CELL outside the transform's valid region.
// Depends on the fixed points and the grid only, so it is formed once per grid.
constexpr uint32_t NO_CELL = 0xffffffffu;
__global__ void k_bs_cell_of(const SamplerParams P, const BSplineDev S, const uint32_t* __restrict__ samples,
                             uint32_t n, uint32_t* __restrict__ cell, uint32_t* __restrict__ idx,
                             uint32_t* __restrict__ count) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const uint32_t flat = samples ? __ldg(samples + s) : s;
        uint32_t i, j, k;
        grid_index(P, flat, i, j, k);
        double x[3], w1[3][4];
        int64_t st[3];
        fixed_point(P, i, j, k, x);
        uint32_t c = NO_CELL;
        if (bs_locate(S, x, w1, st)) {
            c = (uint32_t)(st[0] + (S.gsize[0] - 3) * (st[1] + (S.gsize[1] - 3) * st[2]));
            atomicAdd(count + c, 1u);
        }
        cell[s] = c;
        idx[s] = s;
    }
}

// The tail once (one CTA): value slices folded into the result, the pRatio·nFactor
// table into global memory for the cells, the global histogram re-zeroed.
__global__ void __launch_bounds__(BS_BLOCK) k_bs_tail(const SamplerParams P, const EvalArgs a,
                                                       float* __restrict__ pr_out) {
    extern __shared__ __align__(16) unsigned char bsh[];
    const int B = P.bins;
    const TailSmem ts = tail_layout(B, bsh);
    float* pr = reinterpret_cast<float*>(bsh + tail_smem(B));
    const TailCtx t = tail_prepare(B, P.moving_bin_size, a, ts);
    if (!t.degenerate) {
        pr_table(B, t, ts, pr);
        value_slices_share(B, a, t, ts, 0, 1);
    } else {
        for (int q = threadIdx.x; q < B * B; q += blockDim.x) pr[q] = 0.0f;
    }
    __threadfence_block();
    __syncthreads();
    for (int q = threadIdx.x; q < B * B; q += blockDim.x) pr_out[q] = pr[q];
    if (threadIdx.x < 32) fold_value(B, a, t);
    for (int q = threadIdx.x; q < B * B + B; q += blockDim.x) a.ghist[q] = 0ull;
}

// One CTA per support cell: the derivative of the 4³·3 coefficients over the cell's
// samples (sorted by cell), summed in the CTA and added once per coefficient. Thread t
// owns the four support points of column (kx, ky) = t mod 16 for the samples
// j ≡ ⌊t/16⌋ (mod 16) of each staged group; the sixteen partial sums are then combined
// in order. The support weights are continuous factors of the derivative, formed in
// FP32 from the FP64 grid index; the sums are FP64.
__global__ void __launch_bounds__(BS_BLOCK) k_bs_cell_deriv(const SamplerParams P, const BSplineDev S,
                                                             const EvalArgs a, const float* __restrict__ pr_g,
                                                             const uint32_t* __restrict__ order,
                                                             const uint32_t* __restrict__ off,
                                                             double* __restrict__ deriv) {
    extern __shared__ __align__(16) unsigned char csh[];
    const int B = P.bins;
    float* pr = reinterpret_cast<float*>(csh);                  // B²
    float* sg = pr + ((B * B + 3) & ~3);                        // [3][BS_BLOCK] weighted gradient
    float* sw = sg + 3 * BS_BLOCK;                              // [12][BS_BLOCK] 1-D weights
    __shared__ double red[3][BS_BLOCK];
    const uint32_t c = blockIdx.x;
    const uint32_t beg = off[c], end = off[c + 1];
    if (beg == end) return;
    for (int q = threadIdx.x; q < B * B; q += blockDim.x) pr[q] = __ldg(pr_g + q);
    const int64_t ncx = S.gsize[0] - 3, ncy = S.gsize[1] - 3;
    const int64_t st[3] = {(int64_t)(c % ncx), (int64_t)((c / ncx) % ncy), (int64_t)(c / (ncx * ncy))};
    // thread t: support column (kx, ky) = t & 15 for all four kz, samples j ≡ t >> 4 (mod 16)
    const int t = threadIdx.x, kxy = t & 15, phase = t >> 4;
    const int kx = kxy & 3, ky = kxy >> 2;
    double acc[4][3] = {};
    __syncthreads();
    for (uint32_t base = beg; base < end; base += BS_BLOCK) {
        const uint32_t j = base + t;
        float G[3] = {0.0f, 0.0f, 0.0f}, W[12];
#pragma unroll
        for (int q = 0; q < 12; ++q) W[q] = 0.0f;
        if (j < end) {
            const uint32_t s = __ldg(order + j);
            const uint16_t bins = a.rec_bins[s];
            if (bins) {
                const int mi = bins & 0xff, fi = bins >> 8;
                float dw[4];
                bspline3_deriv_taps(a.rec_f[s], dw);
                const float* row = pr + fi * B + (mi - 1);
                const float ws = fmaf(dw[3], row[3], fmaf(dw[2], row[2], fmaf(dw[1], row[1], dw[0] * row[0])));
                G[0] = ws * a.rec_g[s];
                G[1] = ws * a.rec_g[(size_t)a.npad + s];
                G[2] = ws * a.rec_g[2 * (size_t)a.npad + s];
                const uint32_t flat = a.samples ? __ldg(a.samples + s) : s;
                uint32_t i, jj, kk;
                grid_index(P, flat, i, jj, kk);
                double x[3];
                fixed_point(P, i, jj, kk, x);
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    double g = 0.0;
#pragma unroll
                    for (int q = 0; q < 3; ++q) g += S.p2i[r * 3 + q] * (x[q] - S.gorigin[q]);
                    float u = (float)(g - (double)st[r]);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float au = fabsf(u), sq = au * au;
                        W[r * 4 + q] = au < 1.0f ? (4.0f - 6.0f * sq + 3.0f * sq * au) * (1.0f / 6.0f)
                                                 : (au < 2.0f ? (2.0f - au) * (2.0f - au) * (2.0f - au) * (1.0f / 6.0f)
                                                              : 0.0f);
                        u -= 1.0f;
                    }
                }
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) sg[d * BS_BLOCK + t] = G[d];
#pragma unroll
        for (int q = 0; q < 12; ++q) sw[q * BS_BLOCK + t] = W[q];
        __syncthreads();
        const int cnt = (int)min((uint32_t)BS_BLOCK, end - base);
        for (int jj = phase; jj < cnt; jj += 16) {
            const float wxy = sw[kx * BS_BLOCK + jj] * sw[(4 + ky) * BS_BLOCK + jj];
            const double g0 = (double)sg[jj], g1 = (double)sg[BS_BLOCK + jj], g2 = (double)sg[2 * BS_BLOCK + jj];
#pragma unroll
            for (int kz = 0; kz < 4; ++kz) {
                const double w = (double)(wxy * sw[(8 + kz) * BS_BLOCK + jj]);
                acc[kz][0] += w * g0;
                acc[kz][1] += w * g1;
                acc[kz][2] += w * g2;
            }
        }
        __syncthreads();
    }
    // the 16 phases of each column, summed in phase order
    for (int kz = 0; kz < 4; ++kz) {
#pragma unroll
        for (int d = 0; d < 3; ++d) red[d][t] = acc[kz][d];
        __syncthreads();
        if (t < 16) {
            const int64_t cp = (st[0] + kx) * S.gstride[0] + (st[1] + ky) * S.gstride[1] + (st[2] + kz) * S.gstride[2];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double v = 0.0;
                for (int ph = 0; ph < 16; ++ph) v += red[d][t + 16 * ph];
                if (v != 0.0) atomicAdd(deriv + d * S.nper + cp, v);
            }
        }
        __syncthreads();
    }
}

}  // namespace

// Host side of the B-spline evaluation (see the entry point below).
mi_status evaluate_bspline(mi_metric* m, const double* fixed18, const double* coef, int64_t ncoef, double* value,
                           double* derivative, int64_t* valid, uint16_t* records = nullptr) {
    mi_context* ctx = m->ctx;
    if (m->metric_kind != MI_METRIC_MATTES)
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "the B-spline path is a Mattes-metric evaluation");
    BSplineDev S;
    S.smem_coef = 0;
    double mdir[9];
    for (int d = 0; d < 3; ++d) {
        const double sz = fixed18[d];
        S.gsize[d] = sz >= 1.0 ? (int64_t)sz : 0;  // static_cast<SizeValueType>, as ITK truncates
        if (S.gsize[d] == 0) return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "InvalidBSplineDomain: a zero grid size");
        S.gorigin[d] = fixed18[3 + d];
    }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) mdir[r * 3 + c] = fixed18[9 + r * 3 + c] * fixed18[6 + c];
    if (!invert3(mdir, S.p2i)) return set_error(ctx, MI_ERR_SINGULAR_DIRECTION, "singular B-spline grid direction");
    S.gstride[0] = 1;
    S.gstride[1] = S.gsize[0];
    S.gstride[2] = S.gsize[0] * S.gsize[1];
    S.nper = S.gsize[0] * S.gsize[1] * S.gsize[2];
    if (ncoef != 3 * S.nper)
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "coefficient count is not 3 × the control-point count");
    for (int d = 0; d < 3; ++d) {
        // bspline.rs:504-520
        const double max_limit = (double)S.gsize[d] - 0.5 * (3.0 - 1.0) - 1.0;
        const double scale = std::fabs(max_limit) > 1.0 ? std::fabs(max_limit) : 1.0;
        S.max_limit[d] = max_limit;
        S.snap_ulp[d] = 4.0 * DBL_EPSILON * scale;
        S.snap_to[d] = max_limit - 6.0 * DBL_EPSILON * scale;
    }
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if ((size_t)ncoef > m->bs_cap) {
        cudaFree(m->bs_coef);
        cudaFree(m->bs_deriv);
        m->bs_coef = m->bs_deriv = nullptr;
        m->bs_cap = 0;
        MI_CHECK_CUDA(ctx, cudaMalloc(&m->bs_coef, (size_t)ncoef * sizeof(double)));
        MI_CHECK_CUDA(ctx, cudaMalloc(&m->bs_deriv, (size_t)ncoef * sizeof(double)));
        m->bs_cap = (size_t)ncoef;
    }
    MI_CHECK_CUDA(ctx, cudaMemcpyAsync(m->bs_coef, coef, (size_t)ncoef * sizeof(double), cudaMemcpyHostToDevice, st));
    if (derivative) MI_CHECK_CUDA(ctx, cudaMemsetAsync(m->bs_deriv, 0, (size_t)ncoef * sizeof(double), st));
    Workspace& ws = m->ws;
    const int B = m->bins;
    const uint32_t n = (uint32_t)m->n_samples;
    SamplerParams P = m->base;
    EvalArgs a;
    std::memset(&a, 0, sizeof(a));
    a.moving = m->moving;
    a.mmask = m->mmask;
    a.samples = m->samples;
    a.fbin = m->fbin;
    a.n = n;
    a.npad = (n + 3u) & ~3u;
    a.hist_inv = std::ldexp(1.0, -ws.fine_scale_log2);
    a.ghist = ws.hist;
    a.rec_bins = ws.rec_bins;
    a.rec_f = ws.rec_f;
    a.rec_g = ws.rec_g;
    a.vsum = ws.vsum;
    a.sync = ws.done_counter;
    a.result = ws.result;
    const int64_t want = ((int64_t)n + BS_BLOCK - 1) / BS_BLOCK;
    // the samples grouped by support cell: formed once per grid (the cell of a sample
    // depends on the fixed point and the grid only)
    if (derivative && (!m->bs_have_key || std::memcmp(m->bs_key, fixed18, sizeof(m->bs_key)) != 0)) {
        m->bs_have_key = false;
        cudaFree(m->bs_order);
        cudaFree(m->bs_off);
        m->bs_order = nullptr;
        m->bs_off = nullptr;
        const bool any = S.gsize[0] > 3 && S.gsize[1] > 3 && S.gsize[2] > 3;
        const int64_t ncells = any ? (S.gsize[0] - 3) * (S.gsize[1] - 3) * (S.gsize[2] - 3) : 0;
        if (ncells >= (int64_t)0xffffffffu)
            return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "B-spline grid too large (≥ 2^32 support cells)");
        m->bs_ncells = ncells;
        if (ncells > 0 && n > 0) {
            uint32_t *cell = nullptr, *idx = nullptr, *cell_sorted = nullptr, *count = nullptr;
            void* tmp = nullptr;
            size_t sort_bytes = 0, scan_bytes = 0;
            cudaError_t e = cudaMalloc(&cell, (size_t)n * 4);
            if (e == cudaSuccess) e = cudaMalloc(&idx, (size_t)n * 4);
            if (e == cudaSuccess) e = cudaMalloc(&cell_sorted, (size_t)n * 4);
            if (e == cudaSuccess) e = cudaMalloc(&count, (size_t)(ncells + 1) * 4);
            if (e == cudaSuccess) e = cudaMalloc(&m->bs_order, (size_t)n * 4);
            if (e == cudaSuccess) e = cudaMalloc(&m->bs_off, (size_t)(ncells + 1) * 4);
            if (e == cudaSuccess) e = cudaMemsetAsync(count, 0, (size_t)(ncells + 1) * 4, st);
            if (e == cudaSuccess) {
                const int g = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)ctx->num_sms * 8));
                k_bs_cell_of<<<g, BS_BLOCK, 0, st>>>(P, S, m->samples, n, cell, idx, count);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess)
                e = cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, cell, cell_sorted, idx, m->bs_order, (int)n, 0,
                                                    32, st);
            if (e == cudaSuccess)
                e = cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, count, m->bs_off, (int)(ncells + 1), st);
            if (e == cudaSuccess) e = cudaMalloc(&tmp, std::max(sort_bytes, scan_bytes));
            if (e == cudaSuccess)
                e = cub::DeviceRadixSort::SortPairs(tmp, sort_bytes, cell, cell_sorted, idx, m->bs_order, (int)n, 0, 32,
                                                    st);
            if (e == cudaSuccess)
                e = cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, count, m->bs_off, (int)(ncells + 1), st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            cudaFree(tmp);
            cudaFree(cell);
            cudaFree(idx);
            cudaFree(cell_sorted);
            cudaFree(count);
            if (e != cudaSuccess) return cuda_status(ctx, e, "B-spline support cells");
        }
        std::memcpy(m->bs_key, fixed18, sizeof(m->bs_key));
        m->bs_have_key = true;
    }
    if (!m->bs_pr) MI_CHECK_CUDA(ctx, cudaMalloc(&m->bs_pr, (size_t)B * B * sizeof(float)));
    size_t hsm = (size_t)(((B * B + B) + 1) & ~1) * sizeof(unsigned long long);
    S.smem_coef = hsm + (size_t)ncoef * sizeof(double) <= 96 * 1024 ? 1 : 0;
    if (S.smem_coef) hsm += (size_t)ncoef * sizeof(double);
    const size_t tsm = tail_smem(B) + (size_t)B * B * sizeof(float);
    const size_t csm = (size_t)((B * B + 3) & ~3) * sizeof(float) + (size_t)15 * BS_BLOCK * sizeof(float);
    MI_CHECK_CUDA(ctx, cudaFuncSetAttribute(k_bs_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsm));
    MI_CHECK_CUDA(ctx, cudaFuncSetAttribute(k_bs_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm));
    MI_CHECK_CUDA(ctx, cudaFuncSetAttribute(k_bs_cell_deriv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm));
    const int ghist = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)ctx->num_sms * 4));
    k_bs_hist<<<ghist, BS_BLOCK, hsm, st>>>(P, S, m->bs_coef, a, std::ldexp(1.0, ws.fine_scale_log2));
    k_bs_tail<<<1, BS_BLOCK, tsm, st>>>(P, a, m->bs_pr);
    if (derivative && m->bs_ncells > 0 && n > 0)
        k_bs_cell_deriv<<<(unsigned)m->bs_ncells, BS_BLOCK, csm, st>>>(P, S, a, m->bs_pr, m->bs_order, m->bs_off,
                                                                        m->bs_deriv);
    MI_CHECK_CUDA(ctx, cudaGetLastError());
    MI_CHECK_CUDA(ctx, cudaMemcpyAsync(ws.host_result, ws.result, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (derivative)
        MI_CHECK_CUDA(ctx, cudaMemcpyAsync(derivative, m->bs_deriv, (size_t)ncoef * sizeof(double),
                                           cudaMemcpyDeviceToHost, st));
    if (records)
        MI_CHECK_CUDA(ctx, cudaMemcpyAsync(records, ws.rec_bins, (size_t)n * sizeof(uint16_t), cudaMemcpyDeviceToHost,
                                           st));
    MI_CHECK_CUDA(ctx, cudaStreamSynchronize(st));
    if (value) *value = ws.host_result[0];
    if (valid) *valid = (int64_t)ws.host_result[1];
    return MI_OK;
}

}  // namespace mi

extern "C" mi_status mi_metric_value_and_derivative_bspline(mi_metric* m, const double* fixed18, const double* coef,
                                                            int64_t ncoef, double* value, double* derivative,
                                                            int64_t* valid) {
    if (!m || !fixed18 || !coef || !value || ncoef < 1) return MI_ERR_INVALID_ARGUMENT;
    return mi::evaluate_bspline(m, fixed18, coef, ncoef, value, derivative, valid);
}

// Per-sample outcome of the B-spline path in the metric's sample order
// (mi_metric_sample_order): moving bin | fixed bin << 8 for a valid sample, 0
// otherwise. For the exactness tests.
extern "C" mi_status mi_metric_bspline_records(mi_metric* m, const double* fixed18, const double* coef,
                                               int64_t ncoef, uint16_t* records, int64_t n) {
    if (!m || !fixed18 || !coef || !records || ncoef < 1) return MI_ERR_INVALID_ARGUMENT;
    if (n < m->n_samples)
        return mi::set_error(m->ctx, MI_ERR_INVALID_ARGUMENT, "output array shorter than the sample count");
    double v = 0.0;
    return mi::evaluate_bspline(m, fixed18, coef, ncoef, &v, nullptr, nullptr, records);
}
