// The Mattes metric's shared-sampler siblings behind the same seam: mean squares
// and normalised cross-correlation, as the reference's device metrics compute them
// (registration/device.rs:203-620 DeviceMeanSquaresMetric / DeviceCorrelationMetric;
// cuda/ops/mean_squares.rs, cuda/ops/correlation.rs).
//
// Both are moment reductions: every per-sample term is a product of the sample's
// residual (or mean-subtracted values) with the moving gradient and the fixed point,
// so for any global-affine transform, J(x) = J(x_ref) + Σ_e (x − x_ref)_e·C_e, the
// derivative factors through a fixed set of parameter-free moments and the host
// contracts them with the transform's Jacobian form in FP64:
//
//   mean squares (one pass, 14 moments; mean_squares.rs:21-44)
//     sq = Σ d², S0[d] = Σ d·∇M[d], S1[d][e] = Σ d·∇M[d]·x_e, count   (d = m − f)
//     value = sq / count,  ∂/∂p_k = 2/count · (Σ_d Jref[d][k]·S0[d] + Σ_de C_e[d][k]·S1[d][e])
//   correlation (two passes; correlation.rs:31-52)
//     pass 1: Σf, Σm, count → f̄, m̄ (the last CTA folds them on the device)
//     pass 2: count, sff, smm, sfm, F0[3], F1[9], M0[3], M1[9] over f1 = f − f̄, m1 = m − m̄
//     value = −sfm²/(sff·smm), ∂/∂p_k = −2·sfm/(sff·smm)·(fdm_k − sfm/smm·mdm_k)
//
// The sampler is the Mattes metric's: the continuous index from the composite map,
// replaced by the reference's exact chain wherever a decision (inside test, mask
// rounding) or the gradient's cell could differ, so the valid-sample set is the
// reference's exactly. Values, gradients and every accumulator are FP64; each thread
// sums its samples in order, CTAs reduce in a fixed tree and the last CTA folds the
// CTA partials in CTA order, so a result is bit-identical run to run. Against the
// reference's serial sums the difference is reduction rounding only.
#include <cfloat>
#include <cmath>
#include <cstring>

#include "internal.h"
#include "sampler.cuh"
#include "eval_device.cuh"

namespace mi {
namespace {

constexpr int MOM_BLOCK = 256;
constexpr int MS_SLOTS = 14;    // sq, S0[3], S1[9], count
constexpr int NCC1_SLOTS = 3;   // Σf, Σm, count
constexpr int NCC2_SLOTS = 28;  // count, sff, smm, sfm, F0[3], F1[9], M0[3], M1[9]
enum { MODE_MS = 0, MODE_NCC1 = 1, MODE_NCC2 = 2 };

template <int MODE, bool GRAD>
__host__ __device__ constexpr int slots() {
    return MODE == MODE_MS ? (GRAD ? MS_SLOTS : 2) : (MODE == MODE_NCC1 ? NCC1_SLOTS : (GRAD ? NCC2_SLOTS : 4));
}

struct MomArgs {
    const float* fixed;        // each sample's fixed value, in sample order (the fixed volume
                               // itself when every voxel is a sample)
    const uint8_t* mmask;
    const uint32_t* samples;   // flat indices in brick order, or null for the whole grid
    uint32_t n;
    double* partials;          // [grid][slots]
    unsigned int* counter;     // arrivals of the current launch (reset by the last CTA)
    double* result;            // [slots] folded by the last CTA
    double* result_host;       // mapped host mirror the last CTA also writes (or null)
    const double* means;       // pass 2: pass 1's result (Σf, Σm, count)
};

// One sample in FP64: false when the sample maps outside the moving buffer or onto a
// masked voxel (MovingImage::value_and_physical_gradient, registration/metric.rs:
// 795-861). mv is the linear interpolator's value, g the moving physical gradient, x
// the fixed physical point minus x_ref.
template <bool GRAD>
__device__ __forceinline__ bool sample64(const SamplerParams& P, uint32_t flat, const uint8_t* __restrict__ mmask,
                                         double& mv, double* g, double* x) {
    uint32_t i, j, k;
    grid_index(P, flat, i, j, k);
    const double di = (double)i, dj = (double)j, dk = (double)k;
    double c[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
        c[r] = fma(P.cA[r * 3 + 2], dk, fma(P.cA[r * 3 + 1], dj, fma(P.cA[r * 3 + 0], di, P.cb[r])));
    const double ce = P.cerr;
    bool need = false;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (!(c[d] >= P.ilo && c[d] < P.ihi[d])) {
            if (c[d] < P.olo || c[d] >= P.ohi[d]) return false;
            need = true;
        }
    }
    if (P.has_mmask) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double h = c[d] + 0.5;
            if (floor(h - ce) != floor(h + ce)) need = true;
        }
    }
    double fl[3], fr[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        fl[d] = floor(c[d]);
        fr[d] = c[d] - fl[d];
        // the interpolant's gradient jumps across cell faces: take the reference's cell
        if (GRAD && (fr[d] <= ce || fr[d] >= 1.0 - ce)) need = true;
    }
    if (need) {
        exact_index(P, i, j, k, c);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (!(c[d] >= -0.5 && c[d] < P.mhi[d])) return false;
            fl[d] = floor(c[d]);
            fr[d] = c[d] - fl[d];
        }
    }
    if (P.has_mmask) {
        uint32_t mflat = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double r = floor(c[d] + 0.5);
            if (!(r >= 0.0 && r < (double)P.msz[d])) return false;
            const uint32_t ri = (uint32_t)r;
            mflat += d == 0 ? ri : (d == 1 ? ri * P.ms1 : ri * P.ms2);
        }
        if (!__ldg(mmask + mflat)) return false;
    }
    float v[8];
    fetch_corners(P, fl, v);
    // transform/interpolator.rs:103-152: corner weights Π_d (bit ? fr : 1 − fr), the
    // value summed in corner order; the index-space gradient from the same corners
    const double om[3] = {1.0 - fr[0], 1.0 - fr[1], 1.0 - fr[2]};
    double val = 0.0, gi[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const int b0 = t & 1, b1 = (t >> 1) & 1, b2 = t >> 2;
        const double w0 = b0 ? fr[0] : om[0], w1 = b1 ? fr[1] : om[1], w2 = b2 ? fr[2] : om[2];
        const double b = (double)v[t];
        val += w0 * w1 * w2 * b;
        if (GRAD) {
            gi[0] += (b0 ? 1.0 : -1.0) * (w1 * w2) * b;
            gi[1] += (b1 ? 1.0 : -1.0) * (w0 * w2) * b;
            gi[2] += (b2 ? 1.0 : -1.0) * (w0 * w1) * b;
        }
    }
    mv = val;
    if (GRAD) {
#pragma unroll
        for (int d = 0; d < 3; ++d)
            g[d] = gi[0] * P.mp2i[0 * 3 + d] + gi[1] * P.mp2i[1 * 3 + d] + gi[2] * P.mp2i[2 * 3 + d];
#pragma unroll
        for (int r = 0; r < 3; ++r)
            x[r] = (P.forigin[r] - P.xref[r]) + P.fi2p[r * 3 + 0] * di + P.fi2p[r * 3 + 1] * dj +
                   P.fi2p[r * 3 + 2] * dk;
    }
    return true;
}

template <int MODE, bool GRAD>
__global__ void __launch_bounds__(MOM_BLOCK) k_moments(const SamplerParams P, const MomArgs a) {
    constexpr int NS = slots<MODE, GRAD>();
    constexpr bool WANT_G = GRAD && MODE != MODE_NCC1;
    // correlation's pass 2 is a programmatic dependent of pass 1: it waits here for
    // pass 1's sums (and its use of the partials) before reading anything
    if (MODE == MODE_NCC1) pdl_launch_dependents();
    if (MODE == MODE_NCC2) pdl_wait();
    double acc[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) acc[q] = 0.0;
    double fbar = 0.0, mbar = 0.0;
    if (MODE == MODE_NCC2) {
        const double cnt = a.means[2];
        if (cnt > 0.0) {
            fbar = a.means[0] / cnt;
            mbar = a.means[1] / cnt;
        }
    }
    const uint32_t stride = gridDim.x * blockDim.x;
    // the next sample's index and this sample's fixed value (a coalesced read: the values
    // are gathered once, at set-up) are requested before the sampler runs, so those
    // loads overlap its corner gathers
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t flat = s < a.n ? (a.samples ? __ldg(a.samples + s) : s) : 0u;
    for (; s < a.n; s += stride) {
        const uint32_t sn = s + stride;
        const uint32_t cur = flat;
        flat = sn < a.n ? (a.samples ? __ldg(a.samples + sn) : sn) : 0u;
        const double fv = (double)__ldg(a.fixed + s);
        double mv, g[3], x[3];
        if (!sample64<WANT_G>(P, cur, a.mmask, mv, g, x)) continue;
        if (MODE == MODE_MS) {
            const double diff = mv - fv;
            acc[0] += diff * diff;
            if (WANT_G) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double dg = diff * g[d];
                    acc[1 + d] += dg;
#pragma unroll
                    for (int e = 0; e < 3; ++e) acc[4 + d * 3 + e] += dg * x[e];
                }
            }
            acc[NS - 1] += 1.0;
        } else if (MODE == MODE_NCC1) {
            acc[0] += fv;
            acc[1] += mv;
            acc[2] += 1.0;
        } else {
            const double f1 = fv - fbar, m1 = mv - mbar;
            acc[0] += 1.0;
            acc[1] += f1 * f1;
            acc[2] += m1 * m1;
            acc[3] += f1 * m1;
            if (WANT_G) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double fg = f1 * g[d], mg = m1 * g[d];
                    acc[4 + d] += fg;
                    acc[16 + d] += mg;
#pragma unroll
                    for (int e = 0; e < 3; ++e) {
                        acc[7 + d * 3 + e] += fg * x[e];
                        acc[19 + d * 3 + e] += mg * x[e];
                    }
                }
            }
        }
    }
    __shared__ double red[32];
#pragma unroll
    for (int q = 0; q < NS; ++q) {  // unrolled, so acc stays in registers
        const double v = block_sum(acc[q], red);
        if (threadIdx.x == 0) a.partials[(size_t)blockIdx.x * NS + q] = v;
    }
    if (last_to_arrive(a.counter)) {
        // fold in a fixed order: lane l of slot q sums the partials of CTAs l, l + L, …
        // (L = MOM_BLOCK / NS lanes per slot), sixteen loads issued together, then the
        // L lane sums in lane order
        constexpr int L = MOM_BLOCK / NS;
        __shared__ double fold[MOM_BLOCK];
        const int q = threadIdx.x / L, l = threadIdx.x - q * L;
        if (q < NS) {
            double v = 0.0;
            for (unsigned int b0 = l; b0 < gridDim.x; b0 += 16 * L) {
                double t[16];
#pragma unroll
                for (int u = 0; u < 16; ++u) {
                    const unsigned int b = b0 + u * L;
                    t[u] = b < gridDim.x ? __ldcg(a.partials + (size_t)b * NS + q) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < 16; ++u) v += t[u];
            }
            fold[q * L + l] = v;
        }
        __syncthreads();
        if (threadIdx.x < NS) {
            double t = 0.0;
            for (int k = 0; k < L; ++k) t += fold[threadIdx.x * L + k];
            a.result[threadIdx.x] = t;
            if (a.result_host) a.result_host[threadIdx.x] = t;
        }
        if (threadIdx.x == 0) *a.counter = 0u;
    }
}

// Each sample's fixed value, gathered once: the fixed image and the samples do not
// change over the metric's life, so the evaluations read them contiguously instead of
// gathering from the whole fixed volume.
__global__ void k_gather_fixed(const float* __restrict__ fixed, const uint32_t* __restrict__ samples, int64_t n,
                               float* __restrict__ out) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x)
        out[s] = fixed[samples[s]];
}

template <int MODE, bool GRAD>
int occupancy() {
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_moments<MODE, GRAD>, MOM_BLOCK, 0);
    return occ < 1 ? 1 : occ;
}

}  // namespace

mi_status moments_setup(mi_metric* m) {
    mi_context* ctx = m->ctx;
    MomentsWs& w = m->mom;
    const int occ = std::min({occupancy<MODE_MS, true>(), occupancy<MODE_MS, false>(), occupancy<MODE_NCC1, false>(),
                              occupancy<MODE_NCC2, true>(), occupancy<MODE_NCC2, false>()});
    const int64_t n = std::max<int64_t>(m->n_samples, 1);
    w.grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + MOM_BLOCK - 1) / MOM_BLOCK, (int64_t)ctx->num_sms * occ));
    cudaStream_t st = ctx->stream;
    MI_CHECK_CUDA(ctx, cudaMalloc(&w.partials, (size_t)w.grid * NCC2_SLOTS * sizeof(double)));
    MI_CHECK_CUDA(ctx, cudaMalloc(&w.result, 2 * NCC2_SLOTS * sizeof(double)));
    MI_CHECK_CUDA(ctx, cudaMalloc(&w.counter, 2 * sizeof(unsigned int)));
    MI_CHECK_CUDA(ctx, cudaMemsetAsync(w.counter, 0, 2 * sizeof(unsigned int), st));
    MI_CHECK_CUDA(ctx, cudaMemsetAsync(w.result, 0, 2 * NCC2_SLOTS * sizeof(double), st));
    if (m->samples && m->n_samples > 0) {
        MI_CHECK_CUDA(ctx, cudaMalloc(&w.fval, (size_t)m->n_samples * sizeof(float)));
        const int g = (int)std::max<int64_t>(1, std::min<int64_t>((m->n_samples + 255) / 256, (int64_t)ctx->num_sms * 8));
        k_gather_fixed<<<g, 256, 0, st>>>(m->fixed, m->samples, m->n_samples, w.fval);
        MI_CHECK_CUDA(ctx, cudaGetLastError());
    }
    MI_CHECK_CUDA(ctx, cudaHostAlloc(&w.host, NCC2_SLOTS * sizeof(double), cudaHostAllocMapped));
    MI_CHECK_CUDA(ctx, cudaHostGetDevicePointer(reinterpret_cast<void**>(&w.host_dev), w.host, 0));
    return MI_OK;
}

void moments_free(mi_metric* m) {
    MomentsWs& w = m->mom;
    cudaFree(w.partials);
    cudaFree(w.result);
    cudaFree(w.counter);
    cudaFree(w.fval);
    if (w.host) cudaFreeHost(w.host);
    w = MomentsWs{};
}

mi_status evaluate_moments(mi_metric* m, const SamplerParams& P, const double* jac0, const double* jacc, int nparams,
                           bool want_derivative, double* value, double* derivative, int64_t* valid) {
    mi_context* ctx = m->ctx;
    MomentsWs& w = m->mom;
    Workspace& ws = m->ws;
    cudaStream_t st = ctx->stream;
    const bool timing = ws.timing != 0;
    MomArgs a;
    a.fixed = w.fval ? w.fval : m->fixed;
    a.mmask = m->mmask;
    a.samples = m->samples;
    a.n = (uint32_t)m->n_samples;
    a.partials = w.partials;
    a.counter = w.counter;
    a.result = w.result;
    a.result_host = w.host_dev;  // the final pass writes the host mirror: no copy back
    a.means = nullptr;
    const bool ncc = m->metric_kind == MI_METRIC_CORRELATION;
    if (timing) MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[0], st));
    int ns;
    if (!ncc) {
        ns = want_derivative ? slots<MODE_MS, true>() : slots<MODE_MS, false>();
        if (want_derivative)
            k_moments<MODE_MS, true><<<w.grid, MOM_BLOCK, 0, st>>>(P, a);
        else
            k_moments<MODE_MS, false><<<w.grid, MOM_BLOCK, 0, st>>>(P, a);
    } else {
        // pass 1 folds its sums into result[NCC2_SLOTS..]; pass 2 reads them there
        MomArgs a1 = a;
        a1.result = w.result + NCC2_SLOTS;
        a1.result_host = nullptr;
        a1.counter = w.counter + 1;
        k_moments<MODE_NCC1, false><<<w.grid, MOM_BLOCK, 0, st>>>(P, a1);
        a.means = a1.result;
        ns = want_derivative ? slots<MODE_NCC2, true>() : slots<MODE_NCC2, false>();
        // pass 2 as a programmatic dependent of pass 1 (it waits for pass 1 on entry)
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)w.grid);
        cfg.blockDim = dim3(MOM_BLOCK);
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if (want_derivative)
            MI_CHECK_CUDA(ctx, cudaLaunchKernelEx(&cfg, k_moments<MODE_NCC2, true>, P, a));
        else
            MI_CHECK_CUDA(ctx, cudaLaunchKernelEx(&cfg, k_moments<MODE_NCC2, false>, P, a));
    }
    MI_CHECK_CUDA(ctx, cudaGetLastError());
    if (timing) MI_CHECK_CUDA(ctx, cudaEventRecord(ws.ev[4], st));
    MI_CHECK_CUDA(ctx, cudaStreamSynchronize(st));
    if (timing) {
        float t = 0.f;
        MI_CHECK_CUDA(ctx, cudaEventElapsedTime(&t, ws.ev[0], ws.ev[4]));
        ws.ms[0] += t;
        ws.timed_evals += 1;
    }
    const double* r = w.host;
    // the Jacobian at x_ref: J(x) = J(0) + Σ_e x_e·C_e, and the moments hold x − x_ref
    double jref[3 * MI_MAX_PARAMS];
    if (want_derivative)
        for (int i = 0; i < 3 * nparams; ++i) {
            double v = jac0[i];
            for (int e = 0; e < 3; ++e) v += P.xref[e] * jacc[e * 3 * nparams + i];
            jref[i] = v;
        }
    auto contract = [&](const double* m0, const double* m1, int k) {
        double gk = 0.0;
        for (int d = 0; d < 3; ++d) {
            gk += jref[d * nparams + k] * m0[d];
            for (int e = 0; e < 3; ++e) gk += jacc[e * 3 * nparams + d * nparams + k] * m1[d * 3 + e];
        }
        return gk;
    };
    if (want_derivative)
        for (int k = 0; k < nparams; ++k) derivative[k] = 0.0;
    if (!ncc) {
        // registration/cuda.rs:381-412 (contract)
        const double count = r[ns - 1];
        if (valid) *valid = (int64_t)count;
        if (count == 0.0) {
            *value = DBL_MAX;
            return MI_OK;
        }
        if (!want_derivative) {
            *value = r[0] / count;  // mean_squares_value divides
            return MI_OK;
        }
        const double inv = 1.0 / count;
        *value = r[0] * inv;
        for (int k = 0; k < nparams; ++k) derivative[k] = 2.0 * contract(r + 1, r + 4, k) * inv;
        return MI_OK;
    }
    // registration/cuda.rs:439-490 (contract_correlation)
    const double count = r[0], sff = r[1], smm = r[2], sfm = r[3];
    if (valid) *valid = (int64_t)count;
    const double m2f2 = smm * sff;
    if (count == 0.0 || m2f2 <= DBL_EPSILON) {
        *value = DBL_MAX;
        return MI_OK;
    }
    *value = -sfm * sfm / m2f2;
    if (want_derivative)
        for (int k = 0; k < nparams; ++k) {
            const double fdm = contract(r + 4, r + 7, k);
            const double mdm = contract(r + 16, r + 19, k);
            derivative[k] = -2.0 * sfm / (sff * smm) * (fdm - sfm / smm * mdm);
        }
    return MI_OK;
}

}  // namespace mi
