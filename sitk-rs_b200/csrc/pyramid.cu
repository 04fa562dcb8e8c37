// Multi-resolution pyramid level on the device: recursive (IIR) Gaussian smoothing,
// shrink geometry and linear resampling onto the coarse grid, with the reference's
// arithmetic (registration/method.rs:2416-2580 prepare_level; device counterpart
// cuda/ops/pyramid.rs).
//
//   smoothing   filters/recursive_gaussian.rs:81-290 (axis loop), :472-529 (one line,
//               ITK RecursiveSeparableImageFilter::FilterDataArray), coefficients
//               core/deriche.rs (Deriche / Farnebäck zero-order IIR)
//   shrink      filters/shrink.rs:51-95 (ShrinkImageFilter geometry)
//   resample    transform/resample.rs:226-290 with the linear interpolator
//               (transform/interpolator.rs:29-152)
//
// The volume is smoothed in FP64 from the f32 voxels, axis by axis, and narrowed to
// f32 once at the end, as the reference does. Every FP64 operation is a separately
// rounded __dmul_rn/__dadd_rn/__dsub_rn in the reference's order, so the device
// output is the same bits as a serial FP64 implementation of the same expressions.
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "internal.h"

namespace mi {
void index_to_physical(const mi_geometry& g, double* m);
bool invert3(const double* m, double* inv);
}  // namespace mi

namespace {

// Zero-order Deriche coefficients (core/deriche.rs: Coefficients::new with
// ZeroOrder, the published poles and zero-order column), in the order the line
// recursion reads them: n0..n3, d1..d4, m1..m4, bn1..bn4, bm1..bm4.
struct Deriche {
    double c[20];
};

void deriche_zero_order(double sigmad, Deriche& out) {
    const double w1 = 0.6681, l1 = -1.3932, w2 = 2.0787, l2 = -1.3732;  // poles
    const double a1 = 1.3530, b1 = 1.8151, a2 = -0.3531, b2 = 0.0902;   // zero-order column
    // denominator: compute_d_coefficients
    const double cos1 = std::cos(w1 / sigmad), cos2 = std::cos(w2 / sigmad);
    const double exp1 = std::exp(l1 / sigmad), exp2 = std::exp(l2 / sigmad);
    const double d4 = exp1 * exp1 * exp2 * exp2;
    const double d3 = -2.0 * cos1 * exp1 * exp2 * exp2 - 2.0 * cos2 * exp2 * exp1 * exp1;
    const double d2 = 4.0 * cos2 * cos1 * exp1 * exp2 + exp1 * exp1 + exp2 * exp2;
    const double d1 = -2.0 * (exp2 * cos2 + exp1 * cos1);
    const double sd = 1.0 + d1 + d2 + d3 + d4;
    // numerator: compute_n_coefficients
    const double sin1 = std::sin(w1 / sigmad), sin2 = std::sin(w2 / sigmad);
    double n0 = a1 + a2;
    double n1 = exp2 * (b2 * sin2 - (a2 + 2.0 * a1) * cos2) + exp1 * (b1 * sin1 - (a1 + 2.0 * a2) * cos1);
    double n2 = ((a1 + a2) * cos2 * cos1 - b1 * cos2 * sin1 - b2 * cos1 * sin2) * 2.0 * exp1 * exp2 +
                a2 * exp1 * exp1 + a1 * exp2 * exp2;
    double n3 = exp2 * exp1 * exp1 * (b2 * sin2 - a2 * cos2) + exp1 * exp2 * exp2 * (b1 * sin1 - a1 * cos1);
    const double sn0 = n0 + n1 + n2 + n3;
    // zero order: unit DC gain, symmetric anti-causal part
    const double alpha0 = 2.0 * sn0 / sd - n0;
    n0 = n0 / alpha0;
    n1 = n1 / alpha0;
    n2 = n2 / alpha0;
    n3 = n3 / alpha0;
    const double m1 = n1 - d1 * n0, m2 = n2 - d2 * n0, m3 = n3 - d3 * n0, m4 = -d4 * n0;
    const double sn = n0 + n1 + n2 + n3;
    const double sm = m1 + m2 + m3 + m4;
    const double c[20] = {n0, n1, n2, n3, d1, d2, d3, d4, m1, m2, m3, m4,
                          d1 * sn / sd, d2 * sn / sd, d3 * sn / sd, d4 * sn / sd,
                          d1 * sm / sd, d2 * sm / sd, d3 * sm / sd, d4 * sm / sd};
    std::memcpy(out.c, c, sizeof(c));
}

__global__ void k_widen(const float* __restrict__ in, double* __restrict__ out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

__global__ void k_narrow(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// a·x + b·y + c·z + d·w, each product rounded and the sum taken left to right
__device__ __forceinline__ double dot4(double a, double x, double b, double y, double c, double z, double d,
                                       double w) {
    return __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(a, x), __dmul_rn(b, y)), __dmul_rn(c, z)), __dmul_rn(d, w));
}

// One line per thread through the fourth-order causal + anti-causal recursion
// (recursive_gaussian.rs:472-529): the causal pass writes outs into `out`; the
// anti-causal pass runs backwards with a four-value window and adds each scratch
// value into out as soon as it is formed (outs[k] + scratch[k], the reference's
// final roll-in). The border value extends to infinity on both ends. Lines of
// axis `axis` are indexed by the other two coordinates; a line's element k sits at
// base + k·stride.
__global__ void k_gauss_lines(const double* __restrict__ in, double* __restrict__ out, int64_t nx, int64_t ny,
                              int64_t nz, int axis, Deriche C) {
    const double n0 = C.c[0], n1 = C.c[1], n2 = C.c[2], n3 = C.c[3];
    const double d1 = C.c[4], d2 = C.c[5], d3 = C.c[6], d4 = C.c[7];
    const double m1 = C.c[8], m2 = C.c[9], m3 = C.c[10], m4 = C.c[11];
    const double bn1 = C.c[12], bn2 = C.c[13], bn3 = C.c[14], bn4 = C.c[15];
    const double bm1 = C.c[16], bm2 = C.c[17], bm3 = C.c[18], bm4 = C.c[19];
    int64_t ln, stride, na;  // line length, element stride, lines along the first other axis
    if (axis == 0) {
        ln = nx;
        stride = 1;
        na = ny;
    } else if (axis == 1) {
        ln = ny;
        stride = nx;
        na = nx;
    } else {
        ln = nz;
        stride = nx * ny;
        na = nx;
    }
    const int64_t nlines = (nx * ny * nz) / ln;
    for (int64_t L = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; L < nlines;
         L += (int64_t)gridDim.x * blockDim.x) {
        // line L → (a, b): the two coordinates other than `axis`, first one fastest
        const int64_t a = L % na, b = L / na;
        int64_t base;
        if (axis == 0)
            base = a * nx + b * nx * ny;  // (y, z)
        else if (axis == 1)
            base = a + b * nx * ny;  // (x, z)
        else
            base = a + b * nx;  // (x, y)
        const double* __restrict__ data = in + base;
        double* __restrict__ o = out + base;
        // ---- causal pass
        const double v1 = data[0];
        const double x1 = data[stride], x2 = data[2 * stride], x3 = data[3 * stride];
        double o0 = dot4(v1, n0, v1, n1, v1, n2, v1, n3);
        double o1 = dot4(x1, n0, v1, n1, v1, n2, v1, n3);
        double o2 = dot4(x2, n0, x1, n1, v1, n2, v1, n3);
        double o3 = dot4(x3, n0, x2, n1, x1, n2, v1, n3);
        o0 = __dsub_rn(o0, dot4(v1, bn1, v1, bn2, v1, bn3, v1, bn4));
        o1 = __dsub_rn(o1, dot4(o0, d1, v1, bn2, v1, bn3, v1, bn4));
        o2 = __dsub_rn(o2, dot4(o1, d1, o0, d2, v1, bn3, v1, bn4));
        o3 = __dsub_rn(o3, dot4(o2, d1, o1, d2, o0, d3, v1, bn4));
        o[0] = o0;
        o[stride] = o1;
        o[2 * stride] = o2;
        o[3 * stride] = o3;
        // window: data[i-1..i-3] and outs[i-1..i-4]
        double p1 = x3, p2 = x2, p3 = x1;
        double q1 = o3, q2 = o2, q3 = o1, q4 = o0;
        for (int64_t i = 4; i < ln; ++i) {
            const double x = data[i * stride];
            double v = dot4(x, n0, p1, n1, p2, n2, p3, n3);
            v = __dsub_rn(v, dot4(q1, d1, q2, d2, q3, d3, q4, d4));
            o[i * stride] = v;
            p3 = p2;
            p2 = p1;
            p1 = x;
            q4 = q3;
            q3 = q2;
            q2 = q1;
            q1 = v;
        }
        // ---- anti-causal pass
        const double v2 = data[(ln - 1) * stride];
        const double y1 = data[(ln - 1) * stride], y2 = data[(ln - 2) * stride], y3 = data[(ln - 3) * stride];
        double s1 = dot4(v2, m1, v2, m2, v2, m3, v2, m4);  // scratch[ln-1]
        double s2 = dot4(y1, m1, v2, m2, v2, m3, v2, m4);  // scratch[ln-2]
        double s3 = dot4(y2, m1, y1, m2, v2, m3, v2, m4);  // scratch[ln-3]
        double s4 = dot4(y3, m1, y2, m2, y1, m3, v2, m4);  // scratch[ln-4]
        s1 = __dsub_rn(s1, dot4(v2, bm1, v2, bm2, v2, bm3, v2, bm4));
        s2 = __dsub_rn(s2, dot4(s1, d1, v2, bm2, v2, bm3, v2, bm4));
        s3 = __dsub_rn(s3, dot4(s2, d1, s1, d2, v2, bm3, v2, bm4));
        s4 = __dsub_rn(s4, dot4(s3, d1, s2, d2, s1, d3, v2, bm4));
        o[(ln - 1) * stride] = __dadd_rn(o[(ln - 1) * stride], s1);
        o[(ln - 2) * stride] = __dadd_rn(o[(ln - 2) * stride], s2);
        o[(ln - 3) * stride] = __dadd_rn(o[(ln - 3) * stride], s3);
        o[(ln - 4) * stride] = __dadd_rn(o[(ln - 4) * stride], s4);
        // window: data[i..i+3] and scratch[i..i+3], writing scratch[i-1]
        double e0 = data[(ln - 4) * stride], e1 = y3, e2 = y2, e3 = y1;
        double t0 = s4, t1 = s3, t2 = s2, t3 = s1;
        for (int64_t i = ln - 4; i > 0; --i) {
            double v = dot4(e0, m1, e1, m2, e2, m3, e3, m4);
            v = __dsub_rn(v, dot4(t0, d1, t1, d2, t2, d3, t3, d4));
            o[(i - 1) * stride] = __dadd_rn(o[(i - 1) * stride], v);
            e3 = e2;
            e2 = e1;
            e1 = e0;
            e0 = data[(i - 1) * stride];
            t3 = t2;
            t2 = t1;
            t1 = t0;
            t0 = v;
        }
    }
}

// Linear resampling of an f32 volume onto another grid through the identity
// (transform/resample.rs:226-290): output index → physical point (origin-first
// fold), the difference to the input origin, its image under the input's
// physical-to-index matrix (accumulated from 0.0), then the linear interpolator —
// inside iff c ∈ [−0.5, size − 0.5) per axis, corner weights the running products
// of (1 − frac, frac), corners clamped to the buffer, summed in corner order with
// zero-weight corners skipped (interpolator.rs:57-88) — or `fill` outside; narrowed
// to f32.
struct ResampleGeo {
    int64_t isz[3], osz[3];
    double oi2p[9], oorg[3];  // output index → physical
    double ip2i[9], iorg[3];  // input physical → index
};

// LINEAR: the linear interpolator (transform/interpolator.rs:103-152); otherwise the
// nearest-neighbour one (interpolator.rs:36-54: floor(c + 0.5), clamped), both behind
// the same inside test and the same index arithmetic.
template <bool LINEAR>
__global__ void k_resample(const float* __restrict__ in, float* __restrict__ out, ResampleGeo G, double fill) {
    const int64_t n = G.osz[0] * G.osz[1] * G.osz[2];
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const double idx[3] = {(double)(q % G.osz[0]), (double)((q / G.osz[0]) % G.osz[1]),
                               (double)(q / (G.osz[0] * G.osz[1]))};
        double phys[3], diff[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            double acc = G.oorg[r];
#pragma unroll
            for (int c = 0; c < 3; ++c) acc = __dadd_rn(acc, __dmul_rn(G.oi2p[r * 3 + c], idx[c]));
            phys[r] = acc;
        }
        // the identity AffineTransform's transform_point: mat_vec(I, p) + 0
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            double acc = 0.0;
#pragma unroll
            for (int c = 0; c < 3; ++c) acc = __dadd_rn(acc, __dmul_rn(r == c ? 1.0 : 0.0, phys[c]));
            diff[r] = __dsub_rn(__dadd_rn(acc, 0.0), G.iorg[r]);
        }
        double c[3];
        bool inside = true;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            double acc = 0.0;
#pragma unroll
            for (int j = 0; j < 3; ++j) acc = __dadd_rn(acc, __dmul_rn(G.ip2i[r * 3 + j], diff[j]));
            c[r] = acc;
            inside = inside && c[r] >= -0.5 && c[r] < (double)G.isz[r] - 0.5;
        }
        double v = fill;
        if (inside && !LINEAR) {
            int64_t off = 0, mul = 1;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                int64_t i = (int64_t)floor(__dadd_rn(c[d], 0.5));  // round half up
                i = i < 0 ? 0 : (i > G.isz[d] - 1 ? G.isz[d] - 1 : i);
                off += i * mul;
                mul *= G.isz[d];
            }
            v = (double)__ldg(in + off);
        } else if (inside) {
            double fr[3];
            int64_t b0[3], b1[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double f = floor(c[d]);
                fr[d] = __dsub_rn(c[d], f);
                const int64_t base = (int64_t)f, hi = G.isz[d] - 1;
                b0[d] = base < 0 ? 0 : (base > hi ? hi : base);
                b1[d] = base + 1 < 0 ? 0 : (base + 1 > hi ? hi : base + 1);
            }
            double acc = 0.0;
#pragma unroll
            for (int corner = 0; corner < 8; ++corner) {
                double w = 1.0;
                int64_t off = 0, mul = 1;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const int bit = (corner >> d) & 1;
                    w = __dmul_rn(w, bit ? fr[d] : __dsub_rn(1.0, fr[d]));
                    off += (bit ? b1[d] : b0[d]) * mul;
                    mul *= G.isz[d];
                }
                if (w != 0.0) acc = __dadd_rn(acc, __dmul_rn(w, (double)__ldg(in + off)));
            }
            v = acc;
        }
        out[q] = (float)v;
    }
}

int grid_of(int64_t n, int sms) {
    int64_t g = (n + 255) / 256;
    if (g > (int64_t)sms * 8) g = (int64_t)sms * 8;
    return g < 1 ? 1 : (int)g;
}

mi_status new_image(mi_context* ctx, const mi_geometry& geo, mi_image** out) {
    const int64_t n = geo.size[0] * geo.size[1] * geo.size[2];
    float* d = nullptr;
    MI_CHECK_CUDA(ctx, cudaMalloc(&d, (size_t)n * sizeof(float)));
    mi_image* img = new (std::nothrow) mi_image();
    if (!img) {
        cudaFree(d);
        return MI_ERR_OUT_OF_MEMORY;
    }
    img->ctx = ctx;
    img->geo = geo;
    img->data = d;
    img->n = n;
    *out = img;
    return MI_OK;
}

bool geo_valid(const mi_geometry* g) {
    if (!g) return false;
    for (int d = 0; d < 3; ++d)
        if (g->size[d] <= 0 || !(g->spacing[d] > 0.0)) return false;
    return true;
}

}  // namespace

extern "C" {

mi_status mi_image_smooth(mi_context* ctx, const mi_image* in, const double* sigma3, mi_image** out) {
    if (!ctx || !in || !sigma3 || !out) return MI_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    const mi_geometry& g = in->geo;
    for (int d = 0; d < 3; ++d) {
        if (!(sigma3[d] >= 0.0) || !std::isfinite(sigma3[d]))
            return mi::set_error(ctx, MI_ERR_INVALID_ARGUMENT, "smoothing sigma must be finite and >= 0");
        // recursive_gaussian.rs: AxisTooShortForRecursion
        if (sigma3[d] > 0.0 && g.size[d] < 4)
            return mi::set_error(ctx, MI_ERR_INVALID_ARGUMENT,
                                 "axis " + std::to_string(d) + " is shorter than the recursion's 4 samples");
    }
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    mi_image* res = nullptr;
    mi_status s = new_image(ctx, g, &res);
    if (s != MI_OK) return s;
    const int64_t n = in->n;
    cudaStream_t st = ctx->stream;
    double *a = nullptr, *b = nullptr;
    cudaError_t e = cudaMalloc(&a, (size_t)n * 8);
    if (e == cudaSuccess) e = cudaMalloc(&b, (size_t)n * 8);
    if (e == cudaSuccess) {
        k_widen<<<grid_of(n, ctx->num_sms), 256, 0, st>>>(in->data, a, n);
        e = cudaGetLastError();
    }
    for (int d = 0; d < 3 && e == cudaSuccess; ++d) {
        if (!(sigma3[d] > 0.0)) continue;
        Deriche C;
        deriche_zero_order(sigma3[d] / g.spacing[d], C);
        const int64_t nlines = n / g.size[d];
        k_gauss_lines<<<grid_of(nlines, ctx->num_sms), 256, 0, st>>>(a, b, g.size[0], g.size[1], g.size[2], d, C);
        e = cudaGetLastError();
        std::swap(a, b);
    }
    if (e == cudaSuccess) {
        k_narrow<<<grid_of(n, ctx->num_sms), 256, 0, st>>>(a, res->data, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(a);
    cudaFree(b);
    if (e != cudaSuccess) {
        mi_image_free(res);
        return mi::cuda_status(ctx, e, "mi_image_smooth");
    }
    *out = res;
    return MI_OK;
}

mi_status mi_shrink_geometry(const mi_geometry* in, const int64_t* factors3, mi_geometry* out) {
    if (!in || !factors3 || !out) return MI_ERR_INVALID_ARGUMENT;
    for (int d = 0; d < 3; ++d)
        if (factors3[d] <= 0 || in->size[d] <= 0) return MI_ERR_INVALID_ARGUMENT;  // InvalidShrinkFactor
    mi_geometry o = *in;
    double delta[3];
    for (int d = 0; d < 3; ++d) {
        const int64_t f = factors3[d];
        o.size[d] = std::max<int64_t>(in->size[d] / f, 1);
        o.spacing[d] = in->spacing[d] * (double)f;
        delta[d] = ((double)in->size[d] - 1.0) / 2.0 - (double)f * ((double)o.size[d] - 1.0) / 2.0;
    }
    // origin + Direction·diag(spacing)·δ, accumulated from 0.0 and added last
    for (int i = 0; i < 3; ++i) {
        double acc = 0.0;
        for (int j = 0; j < 3; ++j) acc += in->direction[i * 3 + j] * in->spacing[j] * delta[j];
        o.origin[i] = in->origin[i] + acc;
    }
    *out = o;
    return MI_OK;
}

static mi_status resample(mi_context* ctx, const mi_image* in, const mi_geometry* grid, double fill, bool linear,
                          mi_image** out) {
    if (!ctx || !in || !grid || !out) return MI_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!geo_valid(grid)) return mi::set_error(ctx, MI_ERR_INVALID_ARGUMENT, "bad output geometry");
    ResampleGeo G;
    double ii2p[9];
    mi::index_to_physical(in->geo, ii2p);
    if (!mi::invert3(ii2p, G.ip2i)) return mi::set_error(ctx, MI_ERR_SINGULAR_DIRECTION, "singular input direction");
    mi::index_to_physical(*grid, G.oi2p);
    for (int d = 0; d < 3; ++d) {
        G.isz[d] = in->geo.size[d];
        G.osz[d] = grid->size[d];
        G.oorg[d] = grid->origin[d];
        G.iorg[d] = in->geo.origin[d];
    }
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    mi_image* res = nullptr;
    mi_status s = new_image(ctx, *grid, &res);
    if (s != MI_OK) return s;
    const int64_t n = res->n;
    if (linear)
        k_resample<true><<<grid_of(n, ctx->num_sms), 256, 0, ctx->stream>>>(in->data, res->data, G, fill);
    else
        k_resample<false><<<grid_of(n, ctx->num_sms), 256, 0, ctx->stream>>>(in->data, res->data, G, fill);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        mi_image_free(res);
        return mi::cuda_status(ctx, e, linear ? "mi_image_resample" : "mi_image_resample_nearest");
    }
    *out = res;
    return MI_OK;
}

mi_status mi_image_resample(mi_context* ctx, const mi_image* in, const mi_geometry* grid, double fill,
                            mi_image** out) {
    return resample(ctx, in, grid, fill, true, out);
}

mi_status mi_image_resample_nearest(mi_context* ctx, const mi_image* in, const mi_geometry* grid, double fill,
                                    mi_image** out) {
    return resample(ctx, in, grid, fill, false, out);
}

mi_status mi_pyramid_level(mi_context* ctx, const mi_image* fixed, const mi_image* moving, double sigma,
                           int sigma_physical, const int64_t* factors3, mi_image** fixed_level,
                           mi_image** moving_level) {
    if (!ctx || !fixed || !moving || !factors3 || !fixed_level || !moving_level) return MI_ERR_INVALID_ARGUMENT;
    *fixed_level = nullptr;
    *moving_level = nullptr;
    // physical_sigma (method.rs:2344-2350): voxel units scale by the fixed spacing
    double s3[3];
    for (int d = 0; d < 3; ++d) s3[d] = sigma_physical ? sigma : sigma * fixed->geo.spacing[d];
    const bool smooth = s3[0] != 0.0 || s3[1] != 0.0 || s3[2] != 0.0;
    const bool native = factors3[0] == 1 && factors3[1] == 1 && factors3[2] == 1;
    mi_image* sf = nullptr;
    mi_status s = MI_OK;
    if (smooth)
        s = mi_image_smooth(ctx, fixed, s3, &sf);
    else
        s = mi_image_from_device(ctx, fixed->data, &fixed->geo, &sf);
    if (s != MI_OK) return s;
    mi_image* fl = sf;
    if (!native) {
        mi_geometry coarse;
        s = mi_shrink_geometry(&sf->geo, factors3, &coarse);
        if (s == MI_OK) s = mi_image_resample(ctx, sf, &coarse, 0.0, &fl);
        mi_image_free(sf);
        if (s != MI_OK) return s;
    }
    mi_image* ml = nullptr;
    if (smooth)
        s = mi_image_smooth(ctx, moving, s3, &ml);
    else
        s = mi_image_from_device(ctx, moving->data, &moving->geo, &ml);
    if (s != MI_OK) {
        mi_image_free(fl);
        return s;
    }
    *fixed_level = fl;
    *moving_level = ml;
    return MI_OK;
}

}  // extern "C"
