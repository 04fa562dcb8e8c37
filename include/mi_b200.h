/*
 * mi_b200.h — C ABI of the B200 (sm_100a) Mattes mutual-information metric.
 *
 * This is the drop-in boundary for the device metric seam of sitk-rs (crate `sitk`,
 * paths below are inside crates/sitk/src/). Every entry point takes plain pointers
 * and sizes and returns an mi_status; nothing here names a C++ or torch type, so a
 * Rust `extern "C"` block, ctypes or cgo can bind it as-is.
 *
 * Threading: a handle (context, image, metric) must not be used from two host
 * threads at once without external locking. The reference serialises its device
 * metric behind a Mutex (registration/device.rs:634, :707-712); callers of this
 * library keep the same discipline. Every call is synchronous on the context's
 * stream unless stated otherwise.
 *
 * Errors: no entry point falls back to the CPU. A refusal is named by its status,
 * mirroring DeviceMetricError (registration/device.rs:45-110) and CudaError
 * (cuda/error.rs:11-108); mi_last_error() returns the detail text of the last
 * failure on a context.
 */
#ifndef MI_B200_H
#define MI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MI_OK = 0,
    MI_ERR_INVALID_ARGUMENT = 1,      /* null handle/pointer, bad length, bad enum */
    MI_ERR_NO_DEVICE = 2,             /* CudaError::NoDevice (cuda/error.rs) */
    MI_ERR_CUDA = 3,                  /* CudaError::Driver: any other runtime failure */
    MI_ERR_OUT_OF_MEMORY = 4,
    MI_ERR_UNSUPPORTED_PIXEL_TYPE = 5,/* DeviceImage::upload refuses complex/vector (cuda/image.rs:212-223) */
    MI_ERR_SINGULAR_DIRECTION = 6,    /* DeviceMetricError::SingularDirection */
    MI_ERR_TOO_FEW_HISTOGRAM_BINS = 7,/* RegistrationError::TooFewHistogramBins (mattes.rs:158) */
    MI_ERR_CONSTANT_FIXED = 8,        /* RegistrationError::ConstantIntensity{which:"fixed"} */
    MI_ERR_CONSTANT_MOVING = 9,       /* RegistrationError::ConstantIntensity{which:"moving"} */
    MI_ERR_SAMPLE_INDEX_OUT_OF_GRID = 10, /* CudaError::SampleIndexOutOfGrid */
    MI_ERR_MASK_SIZE_MISMATCH = 11,   /* RegistrationError::MaskSizeMismatch */
    MI_ERR_NON_AFFINE_TRANSFORM = 12, /* DeviceMetricError::NonAffineTransform */
    MI_ERR_POINT_MAP_STAGE_COUNT = 13,/* CudaError::PointMapStageCount: no stage, or more than MI_MAX_STAGES */
    MI_ERR_TOO_MANY_HISTOGRAM_BINS = 14, /* bins > MI_MAX_BINS (the shared-memory histogram's limit): no reference counterpart */
    MI_ERR_TIMEOUT = 15,              /* a bounded device wait gave up (fused form's grid barrier) */
    MI_ERR_NOT_CONVERGED = 16         /* reserved */
} mi_status;

/* Point-map stages the device replays (cuda/ops/resident.rs:74 MAX_STAGES). */
#define MI_MAX_STAGES 8
#define MI_MAX_BINS 128
#define MI_MAX_PARAMS 12

/* DeviceImage pixel types (core PixelId scalar set; cuda/image.rs:182-261).
 * Every scalar type is cast on the device to f32 as (float)(double)x. */
typedef enum {
    MI_U8 = 0, MI_I8 = 1, MI_U16 = 2, MI_I16 = 3, MI_U32 = 4, MI_I32 = 5,
    MI_U64 = 6, MI_I64 = 7, MI_F32 = 8, MI_F64 = 9,
    MI_COMPLEX_F32 = 100, MI_VECTOR_F32 = 101  /* refused by name */
} mi_dtype;

/* 3-D image geometry (cuda/image.rs:122-155): size, spacing, origin, direction
 * (row-major 3×3). Voxels are stored x-fastest. */
typedef struct {
    int64_t size[3];
    double spacing[3];
    double origin[3];
    double direction[9];
} mi_geometry;

/* Fixed-image sampling (registration/metric.rs:84-94, :419-437). */
typedef enum {
    MI_SAMPLING_NONE = 0,     /* every voxel, grid order */
    MI_SAMPLING_REGULAR = 1,  /* every ceil(1/percentage)-th voxel */
    MI_SAMPLING_RANDOM = 2,   /* floor(N·percentage) SplitMix64 draws with replacement */
    MI_SAMPLING_EXPLICIT = 3  /* caller's flat voxel list (FixedSamples::selected_indices) */
} mi_sampling_strategy;

typedef struct {
    int strategy;             /* mi_sampling_strategy */
    double percentage;        /* REGULAR / RANDOM */
    uint64_t seed;            /* RANDOM */
    const int64_t* indices;   /* EXPLICIT: host array of flat fixed-grid voxel indices */
    int64_t n_indices;
} mi_sampling;

/* Transform families with an analytic Jacobian (transform/parametric.rs). */
typedef enum {
    MI_TRANSFORM_AFFINE = 0,          /* 12 params: matrix row-major, translation; fixed: center[3] */
    MI_TRANSFORM_EULER3D = 1,         /* 6: angles x,y,z, translation; fixed: center[3] (+computeZYX) */
    MI_TRANSFORM_VERSOR_RIGID3D = 2,  /* 6: versor right part, translation; fixed: center[3] */
    MI_TRANSFORM_TRANSLATION = 3      /* 3: translation; no fixed params */
} mi_transform_kind;

/* Histogram geometry and sample count of a metric (MattesGeometry, mattes.rs:133-186). */
typedef struct {
    int bins;
    int64_t n_samples;        /* after the fixed-mask filter */
    double fixed_min, fixed_max, moving_min, moving_max;
    double fixed_bin_size, moving_bin_size;
    double fixed_normalized_min, moving_normalized_min;
} mi_metric_info;

typedef struct mi_context mi_context;
typedef struct mi_image mi_image;
typedef struct mi_metric mi_metric;

/* ---- context (cuda/backend.rs:30-160: Backend / backend()) ---------------- */

/* One context per device; owns one CUDA stream. MI_ERR_NO_DEVICE when absent. */
mi_status mi_context_create(int device, mi_context** out);
mi_status mi_context_destroy(mi_context* ctx);
mi_status mi_context_sync(mi_context* ctx);
/* Detail text of the last failure on ctx (valid until the next call on ctx). */
const char* mi_last_error(const mi_context* ctx);
const char* mi_status_string(mi_status s);
/* The context's CUDA stream (a cudaStream_t), for callers that order their own work. */
void* mi_context_stream(mi_context* ctx);

/* ---- images (cuda/image.rs:182 DeviceImage::upload, :269 to_host) --------- */

mi_status mi_image_upload(mi_context* ctx, const void* host, mi_dtype dtype,
                          const mi_geometry* geometry, mi_image** out);
/* Copy an f32 volume that is already in device memory (x-fastest) into a new image. */
mi_status mi_image_from_device(mi_context* ctx, const float* device_ptr,
                               const mi_geometry* geometry, mi_image** out);
mi_status mi_image_to_host(const mi_image* img, float* dst, size_t n_elements);
mi_status mi_image_geometry(const mi_image* img, mi_geometry* out);
/* Device address of the image's f32 voxels (borrowed; valid until mi_image_free). */
const float* mi_image_device_ptr(const mi_image* img);
mi_status mi_image_free(mi_image* img);

/* MetaImage (.mha, or .mhd beside its raw file) reader for 3-D scalar volumes
 * (io/meta_image.rs read): the header's geometry (ElementSpacing; Offset / Position /
 * Origin and Orientation / Rotation / TransformMatrix in MetaIO's fixed precedence;
 * the last value of a repeated key), any of the ten scalar ElementTypes in either
 * byte order, pixels LOCAL or in a named file, zlib/gzip compressed or not; uploaded
 * with mi_image_upload's casts. Refused with MI_ERR_INVALID_ARGUMENT (detail in
 * mi_last_error): other dimensions than 3, more than one channel, ElementDataFile =
 * LIST, a LOCAL compressed header without CompressedDataSize, truncated data. */
mi_status mi_image_read_meta(mi_context* ctx, const char* path, mi_image** out);
/* The same on the host only: the geometry, and (when dst is not NULL) the voxels cast
 * to f32 as the upload casts them into dst (n_elements ≥ the voxel count). Needs no
 * device. */
mi_status mi_image_read_meta_host(const char* path, mi_geometry* geometry, float* dst, size_t n_elements);

/* NIfTI-1 reader for 3-D scalar volumes (io/nifti.rs read): a single .nii, a .hdr +
 * .img pair or an Analyze-7.5 pair, each optionally gzip-compressed (a name ending in
 * .gz is read through zlib); the header in either byte order; the ten scalar
 * datatypes; scl_slope / scl_inter applied (NIfTI only; integers cast to f32 first,
 * the result f32); geometry as the reference's reader forms it (the sform or qform
 * chosen as NiftiImageIO does, RAS+ turned into LPS, spacing in millimetres), and the
 * voxels uploaded with mi_image_upload's f32 cast. Refused by name: dimensions other
 * than 3 after trailing unit dimensions are dropped, vector and matrix intents,
 * unknown datatypes, truncated voxel data (MI_ERR_INVALID_ARGUMENT); complex and RGB
 * datatypes (MI_ERR_UNSUPPORTED_PIXEL_TYPE). */
mi_status mi_image_read_nifti(mi_context* ctx, const char* path, mi_image** out);
/* The same on the host only (geometry, and the f32 voxels when dst is not NULL). */
mi_status mi_image_read_nifti_host(const char* path, mi_geometry* geometry, float* dst, size_t n_elements);

/* ---- metric (registration/device.rs:632-800 DeviceMattesMetric) ----------- */

/* from_device / from_device_sampled (device.rs:644-696). The metric copies both
 * volumes, so the images may be freed afterwards. fixed_mask: optional image on the
 * fixed grid, nonzero = inside. moving_mask: optional host array of
 * size(moving) bytes on the moving grid, nonzero = inside. sampling: NULL means
 * MI_SAMPLING_NONE. */
mi_status mi_metric_create(mi_context* ctx, const mi_image* fixed, const mi_image* moving,
                           const mi_image* fixed_mask, const uint8_t* moving_mask,
                           const mi_sampling* sampling, int bins, mi_metric** out);

/* How the metric stores the moving volume it samples (no reference counterpart: the
 * reference widens it to f64, resident.rs:406-417). MI_STORAGE_BF16 rounds every
 * voxel to BF16 (to nearest, ties to even) once at creation; the range, the bins and
 * every interpolation then use the rounded values, exactly as an f32 volume holding
 * them would, and the corner gathers move half the bytes. */
#define MI_STORAGE_F32 0
#define MI_STORAGE_BF16 1

/* Which metric a handle evaluates. The Mattes metric is the default; mean squares
 * and normalised cross-correlation are the reference's other device metrics
 * (registration/device.rs:203-620 DeviceMeanSquaresMetric, DeviceCorrelationMetric)
 * over the same sample set, masks and sampler, behind the same value / derivative
 * entry points:
 *   mean squares: value = Σ(m − f)²/count, derivative = +∂value/∂p
 *   correlation:  value = −sfm²/(sff·smm) over mean-subtracted samples, derivative
 *                 = +∂value/∂p; a degenerate sample set (m2·f2 ≤ DBL_EPSILON)
 *                 gives DBL_MAX and a zero derivative.
 * No valid sample gives DBL_MAX for every metric. `bins` is ignored for these two,
 * and they refuse no constant image (the reference does not). mi_metric_info_get
 * reports bins = 0 and only the sample count for them. The Mattes-only hooks
 * (mi_metric_sample_decisions, mi_metric_set_fused) refuse them. */
#define MI_METRIC_MATTES 0
#define MI_METRIC_MEAN_SQUARES 1
#define MI_METRIC_CORRELATION 2

/* Layout of the moving volume's texture (the fast path's corner fetch). AUTO stores it,
 * for the Mattes metric, as a 2-D layered texture (one layer per z slice; a cell's
 * eight corners in two gathers) wherever the volume fits the device's layered limits,
 * and otherwise (and for mean squares and correlation, whose FP64 kernels measured
 * faster with it) as a 3-D texture read by eight point fetches; 3D always uses the
 * 3-D texture. Both give the same results bit for bit. No reference counterpart (a
 * device storage choice). */
#define MI_TEXTURE_AUTO 0
#define MI_TEXTURE_3D 1

typedef struct mi_metric_options {
    int moving_storage; /* MI_STORAGE_F32 (default) or MI_STORAGE_BF16 */
    int metric;         /* MI_METRIC_MATTES (default), MI_METRIC_MEAN_SQUARES, MI_METRIC_CORRELATION */
    int texture;        /* MI_TEXTURE_AUTO (default) or MI_TEXTURE_3D */
} mi_metric_options;

/* mi_metric_create with options (NULL: the defaults). */
mi_status mi_metric_create_ex(mi_context* ctx, const mi_image* fixed, const mi_image* moving,
                              const mi_image* fixed_mask, const uint8_t* moving_mask,
                              const mi_sampling* sampling, int bins, const mi_metric_options* options,
                              mi_metric** out);
mi_status mi_metric_info_get(const mi_metric* m, mi_metric_info* out);

/* The flat fixed-grid index of every sample, in the order the device walks them
 * (n ≥ info.n_samples entries). The set is the sampling strategy's draw gated by the
 * fixed mask (metric.rs:101-122, 494-581); the order is 8³ bricks of the fixed grid,
 * bricks and the voxels inside each x-fastest (the whole grid without a mask is
 * walked plainly x-fastest). Per-sample outputs (the records hooks) come in this
 * order. */
mi_status mi_metric_sample_order(mi_metric* m, uint32_t* out, int64_t n);

/* The Mattes value and derivative through a cubic B-spline free-form deformation
 * (transform/bspline.rs BSplineTransform; registration/mattes.rs:722-796
 * evaluate_sparse_support), on a Mattes metric handle. fixed18: the control-point
 * grid as ITK's fixed parameters [size(3), origin(3), spacing(3), direction(9,
 * row-major)]; coef: the 3·Π size coefficients, dimension-major, each grid x-fastest.
 * Every sample takes the reference's exact FP64 chain, so validity and both Parzen
 * bins are the reference's; derivative (may be NULL for the value alone) receives
 * ∂value/∂coef, summed with atomics (its last bits may vary between runs). */
mi_status mi_metric_value_and_derivative_bspline(mi_metric* m, const double* fixed18, const double* coef,
                                                 int64_t ncoef, double* value, double* derivative, int64_t* valid);
/* Test hook (no reference counterpart): each sample's outcome on the B-spline path in
 * the metric's sample order (mi_metric_sample_order): moving bin | fixed bin << 8 when
 * valid, else 0. n ≥ the sample count. */
mi_status mi_metric_bspline_records(mi_metric* m, const double* fixed18, const double* coef, int64_t ncoef,
                                    uint16_t* records, int64_t n);
mi_status mi_metric_destroy(mi_metric* m);

/* DeviceMattesMetric::value (device.rs:734-737): value = −MI at the point map given
 * as `nstage` stages of 12 doubles (matrix row-major, then offset), replayed in
 * order: p ← M·p + t (matrix_offset.rs:102-109). 1 ≤ nstage ≤ MI_MAX_STAGES, else
 * MI_ERR_POINT_MAP_STAGE_COUNT (resident.rs:698-703). `valid` may be NULL. */
mi_status mi_metric_value(mi_metric* m, const double* stages, int nstage, double* value,
                          int64_t* valid);

/* DeviceMattesMetric::evaluate (device.rs:767-800) for a transform family:
 * value = −MI and derivative = +∇(−MI) w.r.t. the family's parameters
 * (the optimizer subtracts it). Degenerate histograms give value = DBL_MAX and a
 * zero derivative (mattes.rs:590-609).
 * These evaluation calls return once the result is in host memory. The metric's
 * last kernel may still be clearing its histogram for the next evaluation on the
 * context's stream. Later work on that stream (including the next evaluation, and
 * mi_metric_destroy, which synchronises it) runs after it. */
mi_status mi_metric_value_and_derivative(mi_metric* m, int kind, const double* params,
                                         int nparams, const double* fixed_params, int nfixed,
                                         double* value, double* derivative, int64_t* valid);

/* The generic form (registration/cuda.rs:294-363 affine_form + :505-524
 * contract_mattes): any point map given as stages, plus a Jacobian that is affine in
 * the fixed point, J(x) = jac0 + Σ_e x_e·jac_c[e], jac0 row-major 3×nparams and
 * jac_c three such blocks. */
mi_status mi_metric_value_and_derivative_stages(mi_metric* m, const double* stages, int nstage,
                                                const double* jac0, const double* jac_c,
                                                int nparams, double* value, double* derivative,
                                                int64_t* valid);

/* Device-time accounting (no reference counterpart; used by benchmarks). enable = 1
 * records a CUDA event on the context stream before an evaluation's first launch and
 * one after its result copy; enable = 2 also records one after each kernel (each
 * event adds a little device time of its own); 0 turns it off. mi_metric_timing_read
 * returns the milliseconds accumulated since the last read — [0] whole evaluation
 * (first launch to the result copy), and with enable = 2 [1] histogram pass (the
 * whole fused kernel in the fused form), [2] the second kernel of the split form
 * (tail and derivative pass, or the value-only tail), [3] unused — and the
 * evaluation count, then resets them. */
mi_status mi_metric_timing_enable(mi_metric* m, int enable);
mi_status mi_metric_timing_read(mi_metric* m, double* ms4, int64_t* n_evals);

/* Launch form of an evaluation (no reference counterpart). The fused form is one
 * cooperative kernel (histogram, grid barrier, tail and derivative); the split form
 * is two kernels (histogram; tail and derivative) with the same arithmetic and the
 * same value bits. The split form is the default: the device time is the same and
 * a cooperative launch adds its latency to a synchronous call. mi_metric_set_fused(m,
 * 1) fails with MI_ERR_INVALID_ARGUMENT where a cooperative launch is not available;
 * mi_metric_get_fused reports the current form. A fused evaluation whose grid
 * barrier does not complete within its wait limit returns MI_ERR_TIMEOUT. */
mi_status mi_metric_set_fused(mi_metric* m, int fused);
mi_status mi_metric_get_fused(const mi_metric* m, int* fused);

/* Corner source of the split form's histogram pass (no reference counterpart; the
 * reference's sampler reads its FP64 copy of the moving volume per sample,
 * cuda/ops/resident.rs:153-333). Off (the default): the eight corners of a sample's
 * cell come through the moving volume's texture. On: per brick of the sample layout,
 * one TMA box load stages the part of the moving volume the brick can touch in shared
 * memory, and the corners are read from there (bricks whose cells reach the volume's
 * edge keep the texture). Same decisions, same corners, same bits. Refused with
 * MI_ERR_INVALID_ARGUMENT when the moving volume's x size is not a multiple of 4 or the
 * driver has no tensor-map encoder; an evaluation whose box does not fit two buffers
 * in shared memory runs the texture pass. A staged-tile wait that does not complete
 * within its limit returns MI_ERR_TIMEOUT. mi_metric_get_tile_staging reports the
 * setting and how many evaluations ran with staged tiles. */
mi_status mi_metric_set_tile_staging(mi_metric* m, int on);
mi_status mi_metric_get_tile_staging(const mi_metric* m, int* on, int64_t* tiled_evals);

/* The point-map stage (matrix row-major, offset: 12 doubles) a transform family
 * stores and multiplies (transform/parametric.rs:549-553, :1103-1107, :1331-1335),
 * and its Jacobian's affine form J(x) = jac0 + Σ_e x_e·jac_c[e] (jac0: 3×nparams
 * row-major; jac_c: three such blocks), formed on the host in the reference's
 * operation order. Any output may be NULL. No device work. */
mi_status mi_transform_form(int kind, const double* params, int nparams, const double* fixed_params,
                            int nfixed, double* stage12, double* jac0, double* jac_c);

/* Per-sample discrete decisions of the device sampler at a point map, in the
 * metric's sample order (test hook for the exactness contract): status 0 = outside
 * the moving buffer or masked, 1 = interpolated value outside the moving range,
 * 2 = valid; fixed_bin/moving_bin are the Parzen indices of valid samples (−1
 * otherwise); flat receives each sample's fixed-grid voxel; exact is 1 where the
 * sampler's fast path handed the sample to the exact FP64 chain. Any output may be
 * NULL. n is the capacity of each array and must be ≥ n_samples. */
mi_status mi_metric_sample_decisions(mi_metric* m, const double* stages, int nstage,
                                     int8_t* status, int32_t* fixed_bin, int32_t* moving_bin,
                                     int64_t* flat, int8_t* exact, int64_t n);

/* ---- registration driver (registration/optimizer.rs, scales.rs, method.rs) ---- */

/* Why an optimisation stopped (optimizer.rs:73-93, same order). */
typedef enum {
    MI_STOP_MAX_ITERATIONS = 0,
    MI_STOP_STEP_TOO_SMALL = 1,
    MI_STOP_CONVERGED = 2,
    MI_STOP_GRADIENT_CONVERGED = 3
} mi_stop_reason;

/* RegularStepGradientDescentOptimizer (optimizer.rs:271-440) as the driver runs it
 * (method.rs:3140-3400). */
typedef struct {
    int iterations;              /* number_of_iterations */
    double minimum_step;         /* minimum_step_length */
    double gradient_tolerance;   /* gradient_magnitude_tolerance (ITK default 1e-4) */
    double relaxation;           /* relaxation_factor (ITK default 0.5) */
    double learning_rate;        /* step-length scale when estimate_learning_rate == 0 */
    int estimate_learning_rate;  /* 1: EstimateLearningRate::Once (scales.rs estimate_learning_rate) */
    int physical_shift_scales;   /* 1: scales from physical shift (scales.rs:572-871); 0: unit */
    /* Optional evaluation record (no counterpart in the reference): when non-NULL,
     * evaluation k < trace_rows writes row k = [value, params[nparams],
     * derivative[nparams]] (1 + 2·nparams doubles, host memory). */
    double* trace;
    int trace_rows;
} mi_rsgd_config;

typedef struct {
    double value;       /* metric value at the returned parameters */
    int64_t valid;      /* valid samples at the returned parameters */
    int iterations;     /* steps taken */
    int stop_reason;    /* mi_stop_reason */
    int evaluations;    /* metric evaluations made */
} mi_rsgd_result;

/* One level of registration: regular-step gradient descent over the device metric
 * from params_inout (updated in place), for a transform family with the given fixed
 * parameters (method.rs:3140 `drive`, optimizer.rs:352-440). */
mi_status mi_register_rsgd(mi_metric* m, int kind, const double* fixed_params, int nfixed,
                           const mi_rsgd_config* cfg, double* params_inout, int nparams,
                           mi_rsgd_result* out);

/* CenteredTransformInitializer in Geometry mode (registration/initializer.rs:56-105):
 * center = the fixed image's geometric centre, translation = moving centre − fixed
 * centre. Host only. */
mi_status mi_centered_initialize(const mi_geometry* fixed, const mi_geometry* moving, double* center3,
                                 double* translation3);

/* ---- pyramid level (registration/method.rs:2416 prepare_level; device
 *      counterpart cuda/ops/pyramid.rs) ---------------------------------------- */

/* Recursive (IIR, Deriche) Gaussian smoothing of an image, zero order on every axis
 * (filters/recursive_gaussian.rs:81 recursive_gaussian): sigma3 in physical units
 * per axis, 0 = that axis untouched. FP64 throughout, narrowed to f32 once; the
 * result is a new image on the same grid. An axis with sigma > 0 needs at least 4
 * voxels (AxisTooShortForRecursion → MI_ERR_INVALID_ARGUMENT). */
mi_status mi_image_smooth(mi_context* ctx, const mi_image* in, const double* sigma3, mi_image** out);

/* ShrinkImageFilter's output geometry (filters/shrink.rs:51-95): size/f (at least
 * 1), spacing·f, origin moved by Direction·diag(spacing)·δ with δ the
 * centre-preserving shift. Host only. */
mi_status mi_shrink_geometry(const mi_geometry* in, const int64_t* factors3, mi_geometry* out);

/* ResampleImageFilter through the identity with the linear interpolator
 * (transform/resample.rs:226-290): a new image on `grid`, `fill` outside the input
 * buffer. */
mi_status mi_image_resample(mi_context* ctx, const mi_image* in, const mi_geometry* grid, double fill,
                            mi_image** out);

/* The same with the nearest-neighbour interpolator (transform/interpolator.rs:36-54:
 * floor(c + 0.5) per axis, clamped): how the device driver carries a fixed mask onto
 * a pyramid level (registration/method.rs:3068-3110 level_mask_on_device; nonzero =
 * inside, fill 0). */
mi_status mi_image_resample_nearest(mi_context* ctx, const mi_image* in, const mi_geometry* grid, double fill,
                                    mi_image** out);

/* One level of the multi-resolution schedule as prepare_level builds it without a
 * virtual domain, fixed-initial transform or masks: both images smoothed with
 * `sigma` (physical units when sigma_physical, else voxels scaled by the fixed
 * spacing, method.rs:2344-2350), the smoothed fixed image resampled onto its own
 * shrunk grid (skipped when every factor is 1); the moving image is only smoothed.
 * Returns two new images. */
mi_status mi_pyramid_level(mi_context* ctx, const mi_image* fixed, const mi_image* moving, double sigma,
                           int sigma_physical, const int64_t* factors3, mi_image** fixed_level,
                           mi_image** moving_level);

/* ---- batched registration (no reference counterpart) ----------------------- */

/* Many registrations of uneven image sizes advanced together: every optimizer
 * iteration is one pass of three launches over all still-active pairs (histogram
 * pass, tail and derivative pass, the regular-step gradient descent step of every
 * pair, with all optimizer state on the device), several passes captured in one CUDA
 * graph that is replayed until every pair has stopped. Per pair the sampler,
 * histogram, tail, moments, optimizer step and point-map constants are the
 * single-pair code; a pair's samples are cut into chunks, and the histogram's
 * fixed-point unit follows the chunk size, so values agree with mi_register_rsgd on
 * the same pair to that unit.
 *
 * mi_batch_create builds one metric per pair (fixed[p], moving[p], sampling[p] — an
 * array of npairs, or NULL for the whole grid — and the common bin count) for the
 * affine (fixed_params: npairs × 3 centres) or translation family (nfixed = 0).
 * mi_batch_register runs from params_inout (npairs × nparams, updated in place) with
 * one configuration for every pair (trace unused) and fills results[npairs];
 * autotune != 0 first times candidate shapes (chunk size, privatised histogram copies)
 * on this batch and keeps the fastest, cached per (bins, sample-count class).
 * mi_batch_shape reports the shape in use. */
typedef struct mi_batch mi_batch;
mi_status mi_batch_create(mi_context* ctx, int npairs, const mi_image* const* fixed, const mi_image* const* moving,
                          const mi_sampling* sampling, int bins, int kind, const double* fixed_params, int nfixed,
                          mi_batch** out);
mi_status mi_batch_register(mi_batch* b, const mi_rsgd_config* cfg, int autotune, double* params_inout,
                            mi_rsgd_result* results);
mi_status mi_batch_shape(const mi_batch* b, int* chunk, int* copies, int* nchunks);
/* Per-pair completion times of the last mi_batch_register (no reference counterpart):
 * seconds[p] is the device global timer's interval from the start of that run's first
 * pass to the optimizer step at which pair p stopped (to the end of the run for a pair
 * that ran out of iterations). n ≥ npairs; MI_ERR_INVALID_ARGUMENT before any run. */
mi_status mi_batch_pair_seconds(const mi_batch* b, double* seconds, int n);
mi_status mi_batch_destroy(mi_batch* b);

/* ---- synthetic pairs (no reference counterpart) ------------------------------ */

/* The counter-based synthetic registration pair built on the device (the CPU twin is
 * sitk_b200/synth.py make_pair_counter): an n³ volume with unit spacing and zero
 * origin, a ramp plus nblobs Gaussian blobs (blobs5: σ, amplitude, cx, cy, cz per
 * blob, added in order inside their ±3.5σ boxes); fixed = volume + noise·N(0,1); moving
 * = the noiseless volume resampled (trilinear, clamp-to-edge) at m·(x − c) + c + t
 * (affine12: m row-major, then t; c the grid centre) + its own noise. The noise of
 * voxel i is a function of (seed, field, i) only: SplitMix64-mixed counters, Box–Muller.
 * Returns two new images. */
mi_status mi_synth_pair(mi_context* ctx, int n, int nblobs, const double* blobs5, const double* affine12,
                        uint64_t seed, double noise, mi_image** fixed, mi_image** moving);

/* ---- learned initialiser (no reference counterpart) ------------------------- */

/* C[M×N] (FP32, leading dimension ldc) = A[M×K]·B[N×K]ᵀ with A and B BF16, row-major,
 * K contiguous (leading dimensions lda, ldb ≥ K): the tensor-core GEMM the
 * initialiser's convolution-as-GEMM layers run on (tcgen05.mma, FP32 accumulation in
 * tensor memory). All pointers are device memory; the call is synchronous. */
mi_status mi_gemm_bf16_tn(mi_context* ctx, int M, int N, int K, const void* A, int lda, const void* B, int ldb,
                          float* C, int ldc);

/* The initialiser network: a 3-D convolutional encoder (2 → 16 → 32 → 64 → 128
 * channels, 3³ kernels, stride 2, padding 1, ReLU; 32³ → 2³) and an MLP head (1024 →
 * 256 ReLU → 12) that maps a fixed/moving pair resampled to 32³ onto 12 normalised
 * affine parameters. Every layer runs on the tensor-core GEMM (BF16 operands, FP32
 * accumulation); master weights and Adam moments are FP32. Layers are numbered 0–3
 * (convolutions; W is out × 27·in with column ((kz·3 + ky)·3 + kx)·in + c), 4 and 5
 * (fully connected; W is out × in, fc1's input index ((z·2 + y)·2 + x)·128 + c).
 * Network inputs are device arrays of B × 32³ × 2 FP32, channels last (x fastest
 * over the grid, then the two channels per voxel: fixed, moving). */
typedef struct mi_initnet mi_initnet;

/* Weights He-uniform from a SplitMix64 stream keyed by seed (the last layer scaled by
 * 0.1), biases 0; buffers for batches of up to max_batch pairs. */
mi_status mi_initnet_create(mi_context* ctx, uint64_t seed, int max_batch, mi_initnet** out);
mi_status mi_initnet_destroy(mi_initnet* net);
/* Copies layer `which`'s weights (out × in, row-major) and bias out — or, with grads
 * != 0, the gradients of the last training step. Either pointer may be NULL. */
mi_status mi_initnet_get(mi_initnet* net, int which, int grads, float* w, float* b);
mi_status mi_initnet_set(mi_initnet* net, int which, const float* w, const float* b);
/* out (device, B × 12) = the network on x (device, B × 32³ × 2). */
mi_status mi_initnet_forward(mi_initnet* net, int batch, const float* x, float* out);
/* Forward, mean squared error against target (device, B × 12), backward; then one
 * Adam step (β1 0.9, β2 0.999, ε 1e-8) when lr > 0. loss (host) may be NULL. */
mi_status mi_initnet_train_step(mi_initnet* net, int batch, const float* x, const float* target, float lr,
                                float* loss);
/* One pair's network input (device, 32³ × 2): fixed and moving resampled (linear, fill
 * 0) onto the 32³ grid with the fixed image's centre and direction and spacing ·
 * size / 32, each normalised to zero mean and unit variance. */
mi_status mi_initnet_prepare(mi_context* ctx, const mi_image* fixed, const mi_image* moving, float* out);

/* ---- allocation-free value (no counterpart in the reference) --------------- */

/* Largest histogram the allocation-free entry point can hold. */
#define MI_NOALLOC_MAX_BINS 64

/* The metric value for callers that cannot allocate device memory (no counterpart in
 * the reference): an application that embeds the metric under a fixed device-memory
 * budget it manages itself, or a real-time loop that must not reach the allocator
 * (cudaMalloc and cudaFree may synchronise the device). It calls no cudaMalloc,
 * cudaFree or allocating routine; its only scratch is one fixed-size array in the
 * library's device memory (a joint histogram of at most MI_NOALLOC_MAX_BINS bins and
 * one counter, 33 KB), which every GPU that loads the library holds until the process
 * exits.
 *
 * Inputs and outputs belong to the caller and are device pointers: the fixed and
 * moving volumes (f32, x-fastest) with their geometries; an optional list of
 * n_samples flat fixed-grid voxels (NULL = every voxel); the histogram geometry
 * `info` (bins and intensity ranges, e.g. from mi_metric_info_get); the point map as
 * `nstage` stages of 12 doubles (1 ≤ nstage ≤ MI_MAX_STAGES, else
 * MI_ERR_POINT_MAP_STAGE_COUNT); and `result`, two doubles that receive −MI and the
 * valid-sample count. No masks. Work is queued on the context's stream and the call
 * returns without waiting: result is ready once that stream has reached it.
 *
 * The sample list is device memory the host cannot inspect. An index at or beyond the
 * fixed grid's voxel count is skipped on the device (neither volume is read for it)
 * and the call reports the failure through `result`: result[0] = NaN and result[1] =
 * −(number of such indices).
 *
 * The first call on a device looks the scratch array up for that device; make that
 * first call before any stream capture begins. The address found then belongs to the
 * device's primary context: do not call this entry point on a device after
 * cudaDeviceReset in the same process. Every call on a device shares the array (each
 * call clears it first, on its stream), so calls whose work overlaps on the GPU race:
 * serialise them. bins > MI_NOALLOC_MAX_BINS is refused with
 * MI_ERR_TOO_MANY_HISTOGRAM_BINS. */
mi_status mi_metric_value_noalloc(mi_context* ctx, const float* fixed, const mi_geometry* fixed_geometry,
                                  const float* moving, const mi_geometry* moving_geometry,
                                  const uint32_t* samples, int64_t n_samples, const mi_metric_info* info,
                                  const double* stages, int nstage, double* result);

#ifdef __cplusplus
}
#endif

#endif /* MI_B200_H */
