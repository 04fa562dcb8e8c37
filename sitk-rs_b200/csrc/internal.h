// Internal types shared by the translation units of libmi_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "mi_b200.h"

struct mi_context {
    int device = 0;
    int num_sms = 0;
    size_t l2_bytes = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
};

struct mi_image {
    mi_context* ctx = nullptr;
    mi_geometry geo{};
    float* data = nullptr;  // device, x-fastest
    int64_t n = 0;
};

namespace mi {

// Division of a u32 by a run-time-invariant divisor through a multiply-high
// (Granlund & Montgomery, "Division by invariant integers using multiplication",
// PLDI 1994, round-up variant): q = (umulhi(n, m) + n) >> s with s = ceil(log2 d),
// m = floor(2^32·(2^s − d)/d) + 1, exact for every n < 2^32.
struct FastDiv {
    uint32_t d, m, s;
};

inline FastDiv make_fastdiv(uint32_t d) {
    FastDiv f{d, 0, 0};
    uint32_t s = 0;
    while (s < 32 && (1ull << s) < d) ++s;
    f.s = s;
    f.m = (uint32_t)(((1ull << 32) * ((1ull << s) - d)) / d + 1);
    return f;
}

// Sampler constants passed to every metric kernel by value. Matrices are row-major.
struct SamplerParams {
    // fixed grid (VirtualGrid, registration/scales.rs:228-271)
    int64_t fsize0, fsize1, fsize2;
    FastDiv div0, div1;
    double forigin[3];
    double fi2p[9];
    // fast path: the composite map from grid index to moving continuous index,
    // c ≈ cA·(i, j, k) + cb (FP64 FMAs), within cerr of the exact chain's c
    double cA[9], cb[3];
    double cerr;
    // inside-test bounds with a 2·cerr margin: surely inside c ∈ [ilo, ihi),
    // surely outside c < olo or c ≥ ohi
    double ilo, olo, ihi[3], ohi[3];
    double bin_hi;  // (double)(bins − 3), the top Parzen bin
    // the fixed grid's centre in index units ((size − 1)/2 per axis, exact in FP32): the
    // derivative pass's position moments are taken in (i,j,k) − xmid, exact integers or
    // half-integers, and mapped to x − x_ref = M_f·((i,j,k) − xmid) once, in FP64, by the fold
    float xmid[3];
    int msz[3];      // moving size, 32-bit (the volume is below 2^32 voxels)
    uint32_t ms1, ms2;  // moving strides, 32-bit
    cudaTextureObject_t mtex;  // the moving volume as a texture (point, clamp, unnormalised)
    int mbf16;                 // the texture holds BF16 bits (u16), widened exactly on fetch
    int mlayered;              // mtex is 2-D layered (one layer per z slice, gathered), else 3-D
    double inv_moving_bin_size;
    // point map stages (matrix_offset.rs:102-109)
    int nstage;
    double stage[MI_MAX_STAGES][12];
    // moving image (MovingImage, registration/metric.rs:681-924)
    int64_t msize[3];
    int64_t mstride1, mstride2;
    double morigin[3];
    double mp2i[9];
    double mhi[3];  // (double)size − 0.5, the is_inside upper bound
    int has_mmask;
    // histogram geometry (MattesGeometry, mattes.rs:133-186)
    int bins;
    double fixed_bin_size, moving_bin_size;
    double fixed_nmin, moving_nmin;
    double moving_min, moving_max;
    // The fast path's range and Parzen decisions (sampler.cuh finish_fast): FP32 copies
    // of the reciprocal bin size and normalised minimum, the top bin, and the metric's
    // global bounds, formed per point map by point_map_fill from vmax (the largest
    // |voxel| of the moving volume): the fast value is within dv = vmax·(16·cerr +
    // 13·2^-24) of the reference's for every sample, the range thresholds are the
    // range ends ∓ (dv plus rounding slack) rounded outward to f32, and dterm bounds
    // the Parzen term's distance from the reference's.
    double vmax;
    float inv_bin_f, nmin_f, bin_hi_f;
    float rlo_out, rlo_in, rhi_in, rhi_out, dterm;
    // derivative moments are taken about this point to limit cancellation
    double xref[3];
    // The brick path (brick.cuh): samples grouped in bricks of 2^brick_bl voxels per
    // axis (0: no brick layout); per brick the composite map at the brick's origin,
    // per sample c = c(origin) + cA·δ (FP64 FMAs, δ the offset inside the brick), within
    // 2·cerr of the exact chain. Formed per point map by point_map_fill:
    //   face_lo, face_hi  an FP32 fraction outside (face_lo, face_hi) may lie within
    //                     2·cerr of a cell face
    //   lo_ext, hi_ext    per axis, the least and greatest of c − c(origin) over a
    //                     brick, widened by 4·cerr (the per-brick inside test)
    int brick_bl;
    float face_lo, face_hi;
    double lo_ext[3], hi_ext[3];
};

// Per-metric device scratch and the host-side view of it.
struct Workspace {
    int staging = 0;                     // corner source of the histogram pass: 0 texture, 1 TMA-staged tiles
    int64_t tiled_evals = 0;             // evaluations whose histogram pass ran with staged tiles
    unsigned long long* hist = nullptr;  // [bins*bins] joint (2^-32 fixed point), [bins] fixed marginal, [1] valid
    double* partials = nullptr;          // [grid_deriv][12]
    double* vsum = nullptr;              // value slice sums
    uint32_t* exq = nullptr;             // per-CTA queues of samples for the exact chain
    uint32_t exq_cap_hist = 0, exq_cap_eval = 0;  // queue length per CTA of k_hist / of the fused kernel
    double* result = nullptr;            // [2 + MI_MAX_PARAMS]: value, valid, derivative
    unsigned int* done_counter = nullptr;
    double* host_result = nullptr;       // pinned mirror of result (mapped)
    double* host_result_dev = nullptr;   // the mirror's device address
    unsigned long long seq = 0;          // evaluations published through the mirror
    // per-sample records pass 1 hands pass 2 (struct of arrays, sample order):
    // moving bin (0 = not a valid sample), Parzen fraction, moving gradient
    uint16_t* rec_bins = nullptr;
    float* rec_f = nullptr;
    float* rec_g = nullptr;              // [3][n_samples]
    float hist_scale = 0.f;              // fixed-point scale of a joint-histogram tap
    int hist_scale_log2 = 0;
    int fine_scale_log2 = 0;              // scale of the fine part; the global bins' unit is 2^-this
    int grid_hist = 0, block_hist = 0;
    int grid_deriv = 0, block_deriv = 0;
    int grid_eval = 0;                    // fused form's cooperative grid (0: not available)
    int grid_split_hist = 0, grid_split_deriv = 0;
    bool fused = false;                   // evaluate with the fused cooperative kernel
    bool can_fuse = false;
    // optional device-time accounting
    int timing = 0;                      // 0 off, 1 whole evaluation, 2 also per kernel
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double ms[4] = {0, 0, 0, 0};
    int64_t timed_evals = 0;
};

}  // namespace mi

namespace mi {
// Buffers of the mean-squares and correlation reductions (moments.cu).
struct MomentsWs {
    int grid = 0;
    double* partials = nullptr;      // [grid][slots]
    double* result = nullptr;        // [2][28]: the folded moments, then correlation's pass-1 sums
    unsigned int* counter = nullptr; // [2] arrival counters
    double* host = nullptr;          // pinned, mapped mirror of the folded moments
    double* host_dev = nullptr;      // the mirror's device address
    float* fval = nullptr;           // each sample's fixed value, in sample order (null: the whole grid)
};
}  // namespace mi

struct mi_metric {
    mi_context* ctx = nullptr;
    int metric_kind = 0;          // MI_METRIC_MATTES, MI_METRIC_MEAN_SQUARES, MI_METRIC_CORRELATION
    mi_geometry fgeo{}, mgeo{};
    float* fixed = nullptr;       // device copy of the fixed volume
    float* moving = nullptr;      // device copy of the moving volume
    uint8_t* mmask = nullptr;     // device moving mask or null
    cudaArray_t marray = nullptr; // the moving volume in a block-linear 3-D array
    cudaTextureObject_t mtex = 0; // point-sampling, clamp-to-edge texture over marray
    uint32_t* samples = nullptr;  // device flat indices in walk order; null = the whole grid (not Mattes)
    uint8_t* fbin = nullptr;      // device fixed Parzen bin of every sample (exact, set-up time)
    int64_t n_samples = 0;
    // the Mattes metric's brick layout (brick.cuh), for the staged-tile histogram pass:
    // the walk order's runs of samples per brick of 2^brick_bl voxels per axis, each run
    // padded to chunks of 32
    int brick_bl = 0;
    uint32_t* codes = nullptr;      // [nchunks·32] offset in the brick | fixed bin; padding BRICK_PAD
    uint32_t* chunk_run = nullptr;  // [nchunks] run (non-empty brick) of each chunk
    uint32_t* run_brick = nullptr;  // [nruns] packed brick coordinates
    uint32_t* run_start = nullptr;  // [nruns] position of the run's first sample in the walk order
    int64_t nchunks = 0, nruns = 0;
    uint32_t* run_chunk0 = nullptr; // [nruns + 1] first chunk of every run
    // TMA-staged moving tiles (tile.cuh): available when the linear moving volume meets the
    // tensor-map rules; the map is re-encoded when an evaluation needs another box
    bool tile_capable = false;
    alignas(64) unsigned char tmap[128] = {};  // CUtensorMap of the moving volume
    int tile_box[3] = {0, 0, 0};
    int tile_grid = 0;              // one CTA per SM
    int64_t tile_per_thread = 0;    // most samples a tile-pass thread takes
    int bins = 0;
    mi_metric_info info{};
    mi::SamplerParams base{};     // everything except the stages
    mi::Workspace ws;
    mi::MomentsWs mom;
    double* bs_coef = nullptr;    // B-spline coefficients of the last call (bspline.cu)
    double* bs_deriv = nullptr;   // its derivative
    size_t bs_cap = 0;            // capacity of both, in doubles
    // the samples grouped by B-spline support cell, for the grid in bs_key
    double bs_key[18] = {};
    bool bs_have_key = false;
    uint32_t* bs_order = nullptr;  // sample indices sorted by cell (valid-region samples first)
    uint32_t* bs_off = nullptr;    // [cells + 1] offsets into bs_order
    int64_t bs_ncells = 0;
    float* bs_pr = nullptr;        // the pRatio·nFactor table of the last evaluation
};

namespace mi {

mi_status set_error(mi_context* ctx, mi_status s, const std::string& msg);
mi_status cuda_status(mi_context* ctx, cudaError_t e, const char* where);
// Raises (never lowers) a kernel's dynamic shared-memory limit on the context's device.
mi_status raise_smem_limit(mi_context* ctx, const void* fn, size_t bytes);

// Host-side transform families (transforms.cpp).
struct AffineForm {
    int nparams = 0;
    double stage[12];        // matrix row-major, offset
    double jac0[3 * MI_MAX_PARAMS];      // J(0), row-major 3×P
    double jacc[3][3 * MI_MAX_PARAMS];   // ∂J/∂x_e
};
mi_status transform_form(int kind, const double* params, int nparams, const double* fixed,
                         int nfixed, AffineForm* out);
// The family's own jacobian_wrt_parameters at point x, row-major 3×P.
mi_status transform_jacobian(int kind, const double* params, int nparams, const double* fixed, int nfixed,
                             const double* x, double* jac);

// Mean squares and correlation (moments.cu).
mi_status moments_setup(mi_metric* m);
void moments_free(mi_metric* m);
mi_status evaluate_moments(mi_metric* m, const SamplerParams& P, const double* jac0, const double* jacc, int nparams,
                           bool want_derivative, double* value, double* derivative, int64_t* valid);

// Core evaluation (mattes.cu).
mi_status evaluate(mi_metric* m, const double* stages, int nstage, const double* jac0,
                   const double* jacc, int nparams, bool want_derivative, double* value,
                   double* derivative, int64_t* valid);

}  // namespace mi

#define MI_CHECK_CUDA(ctx, expr)                                              \
    do {                                                                      \
        cudaError_t _e = (expr);                                              \
        if (_e != cudaSuccess) return mi::cuda_status((ctx), _e, #expr);      \
    } while (0)
