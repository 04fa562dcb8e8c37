// Batched registration: many pairs of uneven sizes advance one optimizer iteration
// per pass of three launches — the histogram pass over every active pair's chunks,
// the tail and derivative pass over the same chunks, and the optimizer step of every
// pair — with all optimizer state on the device. A pass is captured in a CUDA graph
// (several passes per graph) and replayed until every pair has stopped; the host
// only reads how many pairs are still active after each replay.
//
// Per pair the arithmetic is the single-pair path's: the same sampler, histogram,
// tail and moment code (eval_device.cuh), the same regular-step gradient descent
// (rsgd.h) and the same point-map constants (point_map.h). What differs is the
// launch shape: a pair's samples are cut into chunks of `chunk` samples, each CTA
// takes chunks in turn (a persistent grid over the chunk list), and the fixed-point
// unit of the histogram follows from the chunk size, so values agree with the
// single-pair path to that unit.
//
// The chunk size and the number of privatised histogram copies are chosen by a small
// autotuner that times the candidates on the batch itself and caches the choice per
// (bins, sample-count class).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <tuple>
#include <vector>

#include "eval_device.cuh"
#include "internal.h"
#include "point_map.h"
#include "rsgd.h"

namespace mi {
mi_status shift_corners(int kind, const double* params, int nparams, const double* fixed, int nfixed,
                        const mi_geometry& fg, rsgd::Corners& c);
}  // namespace mi

namespace mi {
namespace {

struct Chunk {
    int pair;
    int local;  // index among the pair's chunks
    uint32_t begin, end;
};

struct PairDev {
    SamplerParams P;
    JacobianForm J;
    EvalArgs a;
    rsgd::Corners corners;
    rsgd::State state;
    double scales[MI_MAX_PARAMS];
    double params[MI_MAX_PARAMS];
    double center[3];
    double value;
    double valid;
    int kind, nparams, nchunks;
    int active;
    int evaluations;
    unsigned int done;  // derivative chunks of this pair finished in the current pass
    unsigned long long stop_ns;  // device global timer when the pair stopped (0: running)
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// The device global timer into *t (one thread): the start and end marks of a run.
__global__ void k_stamp(unsigned long long* t) { *t = global_ns(); }

// The next point map of an affine or translation family (transforms.cpp: the
// AffineTransform offset center + t − A·center, mat_vec from 0.0; a translation is
// the identity matrix with the translation as offset).
__device__ void family_stage(int kind, const double* p, const double* center, double* stage) {
    using rsgd::add;
    using rsgd::mul;
    using rsgd::sub;
    if (kind == MI_TRANSFORM_TRANSLATION) {
        for (int i = 0; i < 9; ++i) stage[i] = (i % 4 == 0) ? 1.0 : 0.0;
        for (int d = 0; d < 3; ++d) stage[9 + d] = p[d];
        return;
    }
    for (int i = 0; i < 9; ++i) stage[i] = p[i];
    for (int r = 0; r < 3; ++r) {
        double acc = 0.0;
        for (int c = 0; c < 3; ++c) acc = add(acc, mul(p[r * 3 + c], center[c]));
        stage[9 + r] = sub(add(center[r], p[9 + r]), acc);
    }
}

// Copies a pair's sampler constants into shared memory (read by every sample).
__device__ __forceinline__ void load_params(const SamplerParams& src, SamplerParams& dst) {
    const unsigned int* s = reinterpret_cast<const unsigned int*>(&src);
    unsigned int* d = reinterpret_cast<unsigned int*>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(SamplerParams) / 4); i += blockDim.x) d[i] = s[i];
    __syncthreads();
}

__global__ void __launch_bounds__(HIST_BLOCK, HIST_MIN_BLOCKS)
k_batch_hist(PairDev* __restrict__ pairs, const Chunk* __restrict__ chunks, int nchunks, uint32_t* __restrict__ exq,
             uint32_t exq_cap) {
    extern __shared__ unsigned int sh[];
    __shared__ SamplerParams sP;
    // this CTA's queue for the exact chain: a chunk at a time, so at most a chunk's samples
    const ExactQueue q{MI_EXACT_DEFERRED ? exq + (size_t)blockIdx.x * exq_cap : nullptr, exq_cap};
    for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const Chunk ch = chunks[c];
        PairDev& pd = pairs[ch.pair];
        if (!pd.active) continue;
        load_params(pd.P, sP);
        hist_phase<true>(sP, pd.a, sh, SampleRange{ch.begin, ch.end, threadIdx.x & ~31u, blockDim.x}, q);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(DERIV_BLOCK)
k_batch_deriv(PairDev* __restrict__ pairs, const Chunk* __restrict__ chunks, int nchunks) {
    extern __shared__ double dsh[];
    __shared__ SamplerParams sP;
    __shared__ bool last;
    for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const Chunk ch = chunks[c];
        PairDev& pd = pairs[ch.pair];
        if (!pd.active) continue;
        load_params(pd.P, sP);
        const uint32_t gend = ch.end == pd.a.n ? pd.a.npad >> 2 : ch.end >> 2;
        const GroupWork w{ch.begin >> 2, gend, threadIdx.x, blockDim.x, pd.a.partials + ch.local,
                          (int64_t)pd.nchunks, ch.local, pd.nchunks};
        const TailCtx t = deriv_phase(sP, pd.a, dsh, w);
        // the last chunk of the pair to finish folds the pair's moments and value
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) last = atomicAdd(&pd.done, 1u) == (unsigned int)pd.nchunks - 1u;
        __syncthreads();
        if (last) {
            __threadfence();
            deriv_fold(sP, pd.J, pd.a, t, pd.a.partials, (unsigned int)pd.nchunks);
            if (threadIdx.x < 32) fold_value(sP.bins, pd.a, t);
            if (threadIdx.x == 0) pd.done = 0u;
            const int nb = sP.bins * sP.bins + sP.bins;
            for (int i = threadIdx.x; i < nb; i += blockDim.x) pd.a.ghist[i] = 0ull;
        }
        __syncthreads();
    }
}

// One thread per pair: the optimizer's decision on the evaluation just made, then
// the next point map.
__global__ void k_batch_update(PairDev* __restrict__ pairs, int npairs, mi_rsgd_config cfg,
                               unsigned int* __restrict__ active_count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npairs) return;
    PairDev& pd = pairs[i];
    if (!pd.active) return;
    pd.evaluations += 1;
    pd.value = pd.a.result[0];
    pd.valid = pd.a.result[1];
    double grad[MI_MAX_PARAMS];
    for (int k = 0; k < pd.nparams; ++k) grad[k] = pd.a.result[2 + k];
    if (rsgd::after_evaluation(pd.state, cfg, pd.corners, pd.scales, grad, pd.params)) {
        pd.active = 0;
        pd.stop_ns = global_ns();
        atomicSub(active_count, 1u);
        return;
    }
    double stage[12];
    family_stage(pd.kind, pd.params, pd.center, stage);
    point_map_fill(pd.P, stage, 1);
}

// Autotuner cache: (bins, log2 of the total sample count) → (chunk, coarse copies).
std::mutex g_tune_mu;
std::map<std::pair<int, int>, std::pair<int, int>> g_tune;

}  // namespace
}  // namespace mi

struct mi_batch {
    mi_context* ctx = nullptr;
    int npairs = 0, bins = 0, kind = 0, nparams = 0;
    std::vector<mi_metric*> metrics;
    std::vector<std::vector<double>> fixed_params;
    std::vector<mi::PairDev> host;  // host mirror of the device pair array
    mi::PairDev* d_pairs = nullptr;
    mi::Chunk* d_chunks = nullptr;
    int nchunks = 0;
    double* d_partials = nullptr;
    size_t partials_cap = 0;      // doubles
    unsigned int* d_active = nullptr;
    unsigned int* h_active = nullptr;  // pinned
    unsigned long long* d_marks = nullptr;  // device global timer at the start and end of the last run
    uint32_t* d_exq = nullptr;              // per-CTA queues of samples for the exact chain
    size_t exq_len = 0;
    std::vector<double> pair_seconds;       // per pair: start of the last run to its stop
    int grid_hist = 0, grid_deriv = 0;
    int chunk = 0, copies = 0, fine_copies = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_passes = 0;
    mi_rsgd_config graph_cfg{};
};

namespace mi {
namespace {

size_t batch_hist_smem(int B, int copies, int fine) {
    return ((size_t)copies * hist_copy_stride(B) + (size_t)fine * hist_fine_stride(B)) * sizeof(unsigned int);
}

void release_graph(mi_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->graph_passes = 0;
}

// Lays out the chunk list and the per-pair histogram units for a (chunk, copies)
// shape, and uploads the pair array.
mi_status shape_batch(mi_batch* b, int chunk, int copies) {
    mi_context* ctx = b->ctx;
    const int B = b->bins;
    int fine = std::max(1, copies / 2);
    while (fine > 1 && batch_hist_smem(B, copies, fine) > 52 * 1024) fine >>= 1;
    if (batch_hist_smem(B, copies, fine) > 200 * 1024)
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "histogram copies do not fit in shared memory");
    std::vector<Chunk> chunks;
    size_t poff = 0;
    for (int p = 0; p < b->npairs; ++p) {
        mi_metric* m = b->metrics[p];
        const uint32_t n = (uint32_t)m->n_samples;
        const int nc = std::max<int>(1, (int)((n + chunk - 1) / chunk));
        for (int c = 0; c < nc; ++c)
            chunks.push_back(Chunk{p, c, (uint32_t)c * (uint32_t)chunk, std::min<uint32_t>(n, (uint32_t)(c + 1) * chunk)});
        PairDev& pd = b->host[p];
        pd.nchunks = nc;
        pd.a.partials = b->d_partials + poff;
        poff += (size_t)NMOM * nc;
        // fixed-point units for this shape: a copy of the CTA histogram sees at most
        // ceil(chunk/256)·(256/copies) samples (the single-pair rule, mattes.cu)
        const double per_thread = std::ceil((double)std::min<uint32_t>(n, chunk) / HIST_BLOCK);
        const double lim = 4294967295.0 * 0.98;
        const double coarse_max = std::max(1.0, per_thread * (HIST_BLOCK / copies));
        const double fine_max = std::max(1.0, per_thread * (HIST_BLOCK / fine));
        int k = 22;
        while (k > 0 && std::ldexp(1.0, k) * (2.0 / 3.0) * coarse_max + coarse_max >= lim) --k;
        int kf = FINE_T + 22;
        while (kf > k && (std::ldexp(1.0, kf - FINE_T) * fine_max + fine_max >= lim ||
                          std::ldexp(1.0, kf) * (double)(m->n_samples + 1) >= 0x1p63))
            --kf;
        pd.a.hist_scale = (float)std::ldexp(1.0, k);
        pd.a.fine_scale = (float)std::ldexp(1.0, kf);
        pd.a.fine_shift = kf - k;
        pd.a.hist_inv = std::ldexp(1.0, -kf);
        pd.a.copies = copies;
        pd.a.fine_copies = fine;
    }
    if (poff > b->partials_cap) return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "batch chunk shape too fine");
    cudaFree(b->d_chunks);
    b->d_chunks = nullptr;
    MI_CHECK_CUDA(ctx, cudaMalloc(&b->d_chunks, chunks.size() * sizeof(Chunk)));
    MI_CHECK_CUDA(ctx, cudaMemcpy(b->d_chunks, chunks.data(), chunks.size() * sizeof(Chunk), cudaMemcpyHostToDevice));
    b->nchunks = (int)chunks.size();
    b->chunk = chunk;
    b->copies = copies;
    b->fine_copies = fine;
    const size_t hs = batch_hist_smem(B, copies, fine), ds = deriv_smem(B);
    // raise-only limits: another batch with fewer bins must not lower them under this one
    {
        mi_status ls = raise_smem_limit(ctx, (const void*)k_batch_hist, hs);
        if (ls == MI_OK) ls = raise_smem_limit(ctx, (const void*)k_batch_deriv, ds);
        if (ls != MI_OK) return ls;
    }
    int occ_h = 0, occ_d = 0;
    MI_CHECK_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_h, k_batch_hist, HIST_BLOCK, hs));
    MI_CHECK_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_d, k_batch_deriv, DERIV_BLOCK, ds));
    b->grid_hist = std::max(1, std::min(b->nchunks, ctx->num_sms * std::max(occ_h, 1)));
    b->grid_deriv = std::max(1, std::min(b->nchunks, ctx->num_sms * std::max(occ_d, 1)));
    if ((size_t)b->grid_hist * chunk > b->exq_len) {
        cudaFree(b->d_exq);
        b->d_exq = nullptr;
        b->exq_len = 0;
        MI_CHECK_CUDA(ctx, cudaMalloc(&b->d_exq, (size_t)b->grid_hist * chunk * sizeof(uint32_t)));
        b->exq_len = (size_t)b->grid_hist * chunk;
    }
    release_graph(b);
    return MI_OK;
}

mi_status upload_pairs(mi_batch* b) {
    MI_CHECK_CUDA(b->ctx, cudaMemcpyAsync(b->d_pairs, b->host.data(), b->host.size() * sizeof(PairDev),
                                          cudaMemcpyHostToDevice, b->ctx->stream));
    return MI_OK;
}

mi_status launch_pass(mi_batch* b, const mi_rsgd_config& cfg, bool update) {
    cudaStream_t st = b->ctx->stream;
    const int B = b->bins;
    k_batch_hist<<<b->grid_hist, HIST_BLOCK, batch_hist_smem(B, b->copies, b->fine_copies), st>>>(
        b->d_pairs, b->d_chunks, b->nchunks, b->d_exq, (uint32_t)b->chunk);
    k_batch_deriv<<<b->grid_deriv, DERIV_BLOCK, deriv_smem(B), st>>>(b->d_pairs, b->d_chunks, b->nchunks);
    if (update) k_batch_update<<<(b->npairs + 63) / 64, 64, 0, st>>>(b->d_pairs, b->npairs, cfg, b->d_active);
    MI_CHECK_CUDA(b->ctx, cudaGetLastError());
    return MI_OK;
}

// Point maps and optimizer state of every pair at its starting parameters.
mi_status seed_pairs(mi_batch* b, const mi_rsgd_config& cfg, const double* params) {
    for (int p = 0; p < b->npairs; ++p) {
        PairDev& pd = b->host[p];
        mi_metric* m = b->metrics[p];
        const double* pp = params + (size_t)p * b->nparams;
        for (int k = 0; k < b->nparams; ++k) pd.params[k] = pp[k];
        const std::vector<double>& fp = b->fixed_params[p];
        mi_status s = shift_corners(b->kind, pp, b->nparams, fp.empty() ? nullptr : fp.data(), (int)fp.size(), m->fgeo,
                                    pd.corners);
        if (s != MI_OK) return s;
        for (int k = 0; k < b->nparams; ++k) pd.scales[k] = 1.0;
        if (cfg.physical_shift_scales) rsgd::shift_scales(pd.corners, pd.scales);
        rsgd::start(pd.state, cfg, b->nparams);
        AffineForm f;
        s = transform_form(b->kind, pp, b->nparams, fp.empty() ? nullptr : fp.data(), (int)fp.size(), &f);
        if (s != MI_OK) return s;
        pd.P = m->base;
        pd.P.brick_bl = 0;  // the batch walks the sample list by grid index
        if (!point_map_fill(pd.P, f.stage, 1)) return set_error(b->ctx, MI_ERR_INVALID_ARGUMENT, "non-finite point map");
        pd.active = 1;
        pd.evaluations = 0;
        pd.stop_ns = 0ull;
        pd.done = 0u;
        pd.value = 0.0;
        pd.valid = 0.0;
    }
    return upload_pairs(b);
}

// Times each candidate shape on [histogram, derivative] passes at the starting
// point (no optimizer step) and keeps the fastest; cached per (bins, size class).
mi_status autotune(mi_batch* b, const mi_rsgd_config& cfg, const double* params) {
    int64_t total = 0;
    for (mi_metric* m : b->metrics) total += m->n_samples;
    const int cls = (int)std::ceil(std::log2((double)std::max<int64_t>(total, 1)));
    const auto key = std::make_pair(b->bins, cls);
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) return shape_batch(b, it->second.first, it->second.second);
    }
    const int chunks[] = {2048, 4096, 8192, 16384};
    const int copies_c[] = {2, 4, 8};
    cudaEvent_t e0, e1;
    MI_CHECK_CUDA(b->ctx, cudaEventCreate(&e0));
    MI_CHECK_CUDA(b->ctx, cudaEventCreate(&e1));
    float best = 1e30f;
    int best_chunk = 4096, best_copies = 4;
    mi_status st = MI_OK;
    const size_t coarse_cap = std::max<size_t>(48 * 1024, batch_hist_smem(b->bins, hist_copies(b->bins), 0));
    for (int ch : chunks) {
        for (int cp : copies_c) {
            if (batch_hist_smem(b->bins, cp, 0) > coarse_cap) continue;
            if ((st = shape_batch(b, ch, cp)) != MI_OK) break;
            if ((st = seed_pairs(b, cfg, params)) != MI_OK) break;
            if ((st = launch_pass(b, cfg, false)) != MI_OK) break;  // warm-up
            float acc = 0.0f;
            for (int r = 0; r < 3 && st == MI_OK; ++r) {
                cudaEventRecord(e0, b->ctx->stream);
                st = launch_pass(b, cfg, false);
                cudaEventRecord(e1, b->ctx->stream);
                cudaEventSynchronize(e1);
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                acc += ms;
            }
            if (st != MI_OK) break;
            if (acc < best) {
                best = acc;
                best_chunk = ch;
                best_copies = cp;
            }
        }
        if (st != MI_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != MI_OK) return st;
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        g_tune[key] = std::make_pair(best_chunk, best_copies);
    }
    return shape_batch(b, best_chunk, best_copies);
}

constexpr int PASSES_PER_GRAPH = 8;

mi_status build_graph(mi_batch* b, const mi_rsgd_config& cfg) {
    release_graph(b);
    cudaStream_t st = b->ctx->stream;
    MI_CHECK_CUDA(b->ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    mi_status s = MI_OK;
    for (int i = 0; i < PASSES_PER_GRAPH && s == MI_OK; ++i) s = launch_pass(b, cfg, true);
    if (s == MI_OK) {
        cudaError_t e = cudaMemcpyAsync(b->h_active, b->d_active, sizeof(unsigned int), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) s = cuda_status(b->ctx, e, "batch graph");
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (s != MI_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess) return cuda_status(b->ctx, e, "batch graph capture");
    b->graph = g;
    e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess) return cuda_status(b->ctx, e, "batch graph instantiate");
    b->graph_passes = PASSES_PER_GRAPH;
    b->graph_cfg = cfg;
    return MI_OK;
}

bool same_cfg(const mi_rsgd_config& a, const mi_rsgd_config& c) {
    return a.iterations == c.iterations && a.minimum_step == c.minimum_step &&
           a.gradient_tolerance == c.gradient_tolerance && a.relaxation == c.relaxation &&
           a.learning_rate == c.learning_rate && a.estimate_learning_rate == c.estimate_learning_rate &&
           a.physical_shift_scales == c.physical_shift_scales;
}

void free_batch(mi_batch* b) {
    if (!b) return;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    release_graph(b);
    cudaFree(b->d_pairs);
    cudaFree(b->d_chunks);
    cudaFree(b->d_partials);
    cudaFree(b->d_active);
    cudaFree(b->d_marks);
    cudaFree(b->d_exq);
    if (b->h_active) cudaFreeHost(b->h_active);
    for (mi_metric* m : b->metrics)
        if (m) mi_metric_destroy(m);
    delete b;
}

}  // namespace
}  // namespace mi

extern "C" {

mi_status mi_batch_create(mi_context* ctx, int npairs, const mi_image* const* fixed, const mi_image* const* moving,
                          const mi_sampling* sampling, int bins, int kind, const double* fixed_params, int nfixed,
                          mi_batch** out) {
    using namespace mi;
    if (!ctx || npairs < 1 || !fixed || !moving || !out) return MI_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int nparams = 0;
    if (kind == MI_TRANSFORM_AFFINE)
        nparams = 12;
    else if (kind == MI_TRANSFORM_TRANSLATION)
        nparams = 3;
    else
        return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "the batched form takes affine or translation transforms");
    if (kind == MI_TRANSFORM_AFFINE && nfixed != 3) return set_error(ctx, MI_ERR_INVALID_ARGUMENT, "affine needs a centre");
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    mi_batch* b = new (std::nothrow) mi_batch();
    if (!b) return MI_ERR_OUT_OF_MEMORY;
    b->ctx = ctx;
    b->npairs = npairs;
    b->bins = bins;
    b->kind = kind;
    b->nparams = nparams;
    b->metrics.assign(npairs, nullptr);
    b->fixed_params.resize(npairs);
    b->host.resize(npairs);
    mi_status s = MI_OK;
    size_t max_chunks = 0;
    for (int p = 0; p < npairs && s == MI_OK; ++p) {
        s = mi_metric_create(ctx, fixed[p], moving[p], nullptr, nullptr, sampling ? sampling + p : nullptr, bins,
                             &b->metrics[p]);
        if (s != MI_OK) break;
        mi_metric* m = b->metrics[p];
        if (kind == MI_TRANSFORM_AFFINE) b->fixed_params[p].assign(fixed_params + 3 * p, fixed_params + 3 * p + 3);
        PairDev& pd = b->host[p];
        std::memset(&pd, 0, sizeof(PairDev));
        pd.kind = kind;
        pd.nparams = nparams;
        if (kind == MI_TRANSFORM_AFFINE)
            for (int d = 0; d < 3; ++d) pd.center[d] = fixed_params[3 * p + d];
        // Jacobian form: constant for these families
        AffineForm f;
        std::vector<double> p0(nparams, 0.0);
        if (kind == MI_TRANSFORM_AFFINE) p0[0] = p0[4] = p0[8] = 1.0;
        s = transform_form(kind, p0.data(), nparams, kind == MI_TRANSFORM_AFFINE ? pd.center : nullptr,
                           kind == MI_TRANSFORM_AFFINE ? 3 : 0, &f);
        if (s != MI_OK) break;
        pd.J.nparams = nparams;
        for (int i = 0; i < 3 * nparams; ++i) {
            pd.J.jac0[i] = f.jac0[i];
            for (int e = 0; e < 3; ++e) pd.J.jacc[e][i] = f.jacc[e][i];
        }
        EvalArgs& a = pd.a;
        a.moving = m->moving;
        a.mmask = m->mmask;
        a.samples = m->samples;
        a.fbin = m->fbin;
        a.n = (uint32_t)m->n_samples;
        a.npad = (a.n + 3u) & ~3u;
        a.ghist = m->ws.hist;
        a.rec_bins = m->ws.rec_bins;
        a.rec_f = m->ws.rec_f;
        a.rec_g = m->ws.rec_g;
        a.vsum = m->ws.vsum;
        a.sync = m->ws.done_counter;
        a.result = m->ws.result;
        max_chunks += (size_t)std::max<int64_t>(1, (m->n_samples + 2047) / 2048);
    }
    if (s == MI_OK) {
        cudaError_t e = cudaMalloc(&b->d_pairs, (size_t)npairs * sizeof(PairDev));
        if (e == cudaSuccess) e = cudaMalloc(&b->d_partials, max_chunks * NMOM * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&b->d_active, sizeof(unsigned int));
        if (e == cudaSuccess) e = cudaMallocHost(&b->h_active, sizeof(unsigned int));
        if (e == cudaSuccess) e = cudaMalloc(&b->d_marks, 2 * sizeof(unsigned long long));
        if (e != cudaSuccess) s = cuda_status(ctx, e, "mi_batch_create");
        b->partials_cap = max_chunks * NMOM;
    }
    if (s == MI_OK) s = shape_batch(b, 4096, hist_copies(bins));
    if (s != MI_OK) {
        free_batch(b);
        return s;
    }
    *out = b;
    return MI_OK;
}

mi_status mi_batch_destroy(mi_batch* b) {
    if (!b) return MI_ERR_INVALID_ARGUMENT;
    mi::free_batch(b);
    return MI_OK;
}

mi_status mi_batch_register(mi_batch* b, const mi_rsgd_config* cfg, int autotune, double* params_inout,
                            mi_rsgd_result* results) {
    using namespace mi;
    if (!b || !cfg || !params_inout || !results) return MI_ERR_INVALID_ARGUMENT;
    mi_context* ctx = b->ctx;
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    mi_status s = MI_OK;
    if (autotune && (s = mi::autotune(b, *cfg, params_inout)) != MI_OK) return s;
    if ((s = seed_pairs(b, *cfg, params_inout)) != MI_OK) return s;
    const unsigned int n = (unsigned int)b->npairs;
    MI_CHECK_CUDA(ctx, cudaMemcpyAsync(b->d_active, &n, sizeof(n), cudaMemcpyHostToDevice, ctx->stream));
    if (!b->exec || !same_cfg(b->graph_cfg, *cfg))
        if ((s = build_graph(b, *cfg)) != MI_OK) return s;
    // every pair makes at most iterations + 1 evaluations
    const int max_replays = (cfg->iterations + 1 + b->graph_passes - 1) / b->graph_passes + 1;
    k_stamp<<<1, 1, 0, ctx->stream>>>(b->d_marks);
    for (int r = 0; r < max_replays; ++r) {
        MI_CHECK_CUDA(ctx, cudaGraphLaunch(b->exec, ctx->stream));
        MI_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (*b->h_active == 0u) break;
    }
    k_stamp<<<1, 1, 0, ctx->stream>>>(b->d_marks + 1);
    MI_CHECK_CUDA(ctx, cudaGetLastError());
    unsigned long long marks[2] = {0ull, 0ull};
    MI_CHECK_CUDA(ctx, cudaMemcpyAsync(marks, b->d_marks, sizeof(marks), cudaMemcpyDeviceToHost, ctx->stream));
    MI_CHECK_CUDA(ctx, cudaMemcpy(b->host.data(), b->d_pairs, b->host.size() * sizeof(PairDev), cudaMemcpyDeviceToHost));
    b->pair_seconds.assign(b->npairs, 0.0);
    for (int p = 0; p < b->npairs; ++p) {
        const unsigned long long stop = b->host[p].stop_ns ? b->host[p].stop_ns : marks[1];
        b->pair_seconds[p] = stop > marks[0] ? (double)(stop - marks[0]) * 1e-9 : 0.0;
    }
    for (int p = 0; p < b->npairs; ++p) {
        const PairDev& pd = b->host[p];
        for (int k = 0; k < b->nparams; ++k) params_inout[(size_t)p * b->nparams + k] = pd.params[k];
        results[p].value = pd.value;
        results[p].valid = (int64_t)pd.valid;
        results[p].iterations = pd.state.taken;
        results[p].stop_reason = pd.active ? MI_STOP_MAX_ITERATIONS : pd.state.stop;
        results[p].evaluations = pd.evaluations;
    }
    return MI_OK;
}

mi_status mi_batch_pair_seconds(const mi_batch* b, double* seconds, int n) {
    if (!b || !seconds || n < b->npairs) return MI_ERR_INVALID_ARGUMENT;
    if ((int)b->pair_seconds.size() != b->npairs) return MI_ERR_INVALID_ARGUMENT;
    for (int p = 0; p < b->npairs; ++p) seconds[p] = b->pair_seconds[p];
    return MI_OK;
}

mi_status mi_batch_shape(const mi_batch* b, int* chunk, int* copies, int* nchunks) {
    if (!b) return MI_ERR_INVALID_ARGUMENT;
    if (chunk) *chunk = b->chunk;
    if (copies) *copies = b->copies;
    if (nchunks) *nchunks = b->nchunks;
    return MI_OK;
}

}  // extern "C"
