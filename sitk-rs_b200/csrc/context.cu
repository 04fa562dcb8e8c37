// Context, error model and image upload/to_host.
//
// Mirrors the reference's device runtime contract: one backend per device with one
// stream (cuda/backend.rs:30-160), DeviceImage upload of any scalar pixel type to a
// device f32 volume cast as (float)(double)x (cuda/image.rs:98-106, :182-261), and
// to_host (cuda/image.rs:269-280). Complex and vector pixels are refused by name.

#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>

#include "internal.h"

namespace mi {

mi_status set_error(mi_context* ctx, mi_status s, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return s;
}

mi_status cuda_status(mi_context* ctx, cudaError_t e, const char* where) {
    mi_status s = MI_ERR_CUDA;
    if (e == cudaErrorMemoryAllocation) s = MI_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) s = MI_ERR_NO_DEVICE;
    std::string msg = std::string(where) + ": " + cudaGetErrorString(e);
    return set_error(ctx, s, msg);
}

// A kernel's dynamic shared-memory limit is a property of the function on the
// current device, shared by every metric in the process: it is only ever raised,
// so a metric created later with a smaller need does not shrink it under an
// earlier one.
mi_status raise_smem_limit(mi_context* ctx, const void* fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> lim;
    std::lock_guard<std::mutex> g(mu);
    size_t& cur = lim[{ctx->device, fn}];
    if (bytes <= cur) return MI_OK;
    const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return cuda_status(ctx, e, "cudaFuncSetAttribute");
    cur = bytes;
    return MI_OK;
}

}  // namespace mi

namespace {

template <typename T>
__global__ void k_cast_to_f32(const T* __restrict__ src, float* __restrict__ dst, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) dst[i] = (float)(double)src[i];
}

size_t dtype_size(int dt) {
    switch (dt) {
        case MI_U8: case MI_I8: return 1;
        case MI_U16: case MI_I16: return 2;
        case MI_U32: case MI_I32: case MI_F32: return 4;
        case MI_U64: case MI_I64: case MI_F64: return 8;
        default: return 0;
    }
}

bool geometry_ok(const mi_geometry* g) {
    if (!g) return false;
    for (int d = 0; d < 3; ++d)
        if (g->size[d] <= 0) return false;
    return true;
}

template <typename T>
void launch_cast(const void* src, float* dst, int64_t n, int sms, cudaStream_t st) {
    int block = 256;
    int64_t want = (n + block - 1) / block;
    int grid = (int)(want < (int64_t)sms * 8 ? want : (int64_t)sms * 8);
    if (grid < 1) grid = 1;
    k_cast_to_f32<T><<<grid, block, 0, st>>>((const T*)src, dst, n);
}

}  // namespace

extern "C" {

const char* mi_status_string(mi_status s) {
    switch (s) {
        case MI_OK: return "ok";
        case MI_ERR_INVALID_ARGUMENT: return "invalid argument";
        case MI_ERR_NO_DEVICE: return "no CUDA device";
        case MI_ERR_CUDA: return "CUDA runtime error";
        case MI_ERR_OUT_OF_MEMORY: return "out of device memory";
        case MI_ERR_UNSUPPORTED_PIXEL_TYPE: return "unsupported pixel type (complex or vector)";
        case MI_ERR_SINGULAR_DIRECTION: return "moving image's direction matrix is singular";
        case MI_ERR_TOO_FEW_HISTOGRAM_BINS: return "too few histogram bins (need at least 5)";
        case MI_ERR_CONSTANT_FIXED: return "constant intensity: fixed";
        case MI_ERR_CONSTANT_MOVING: return "constant intensity: moving";
        case MI_ERR_SAMPLE_INDEX_OUT_OF_GRID: return "sample index outside the fixed grid";
        case MI_ERR_MASK_SIZE_MISMATCH: return "mask size does not match its image";
        case MI_ERR_NON_AFFINE_TRANSFORM: return "transform's Jacobian is not affine in the point";
        case MI_ERR_POINT_MAP_STAGE_COUNT: return "too many point-map stages";
        case MI_ERR_TOO_MANY_HISTOGRAM_BINS: return "too many histogram bins for the device histogram";
        case MI_ERR_TIMEOUT: return "a bounded device wait gave up";
        case MI_ERR_NOT_CONVERGED: return "not converged";
    }
    return "unknown status";
}

mi_status mi_context_create(int device, mi_context** out) {
    if (!out) return MI_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return MI_ERR_NO_DEVICE;
    if (device < 0 || device >= count) return MI_ERR_INVALID_ARGUMENT;
    mi_context* c = new (std::nothrow) mi_context();
    if (!c) return MI_ERR_OUT_OF_MEMORY;
    c->device = device;
    e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    int l2 = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device);
    c->l2_bytes = (size_t)l2;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return e == cudaErrorNoDevice ? MI_ERR_NO_DEVICE : MI_ERR_CUDA;
    }
    *out = c;
    return MI_OK;
}

mi_status mi_context_destroy(mi_context* ctx) {
    if (!ctx) return MI_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    if (ctx->stream) {
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
    }
    delete ctx;
    return MI_OK;
}

mi_status mi_context_sync(mi_context* ctx) {
    if (!ctx) return MI_ERR_INVALID_ARGUMENT;
    MI_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MI_OK;
}

const char* mi_last_error(const mi_context* ctx) {
    return ctx ? ctx->last_error.c_str() : "null context";
}

void* mi_context_stream(mi_context* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

mi_status mi_image_upload(mi_context* ctx, const void* host, mi_dtype dtype,
                          const mi_geometry* geometry, mi_image** out) {
    if (!ctx || !host || !out) return MI_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (dtype == MI_COMPLEX_F32 || dtype == MI_VECTOR_F32)
        return mi::set_error(ctx, MI_ERR_UNSUPPORTED_PIXEL_TYPE,
                             "DeviceImage holds scalar voxels only; complex and vector pixels are refused");
    size_t es = dtype_size(dtype);
    if (es == 0) return mi::set_error(ctx, MI_ERR_INVALID_ARGUMENT, "unknown pixel type");
    if (!geometry_ok(geometry)) return mi::set_error(ctx, MI_ERR_INVALID_ARGUMENT, "bad geometry");
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    int64_t n = geometry->size[0] * geometry->size[1] * geometry->size[2];
    float* d = nullptr;
    MI_CHECK_CUDA(ctx, cudaMalloc(&d, (size_t)n * sizeof(float)));
    cudaError_t e = cudaSuccess;
    if (dtype == MI_F32) {
        e = cudaMemcpyAsync(d, host, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream);
    } else {
        void* tmp = nullptr;
        e = cudaMalloc(&tmp, (size_t)n * es);
        if (e == cudaSuccess) e = cudaMemcpyAsync(tmp, host, (size_t)n * es, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) {
            switch (dtype) {
                case MI_U8: launch_cast<uint8_t>(tmp, d, n, ctx->num_sms, ctx->stream); break;
                case MI_I8: launch_cast<int8_t>(tmp, d, n, ctx->num_sms, ctx->stream); break;
                case MI_U16: launch_cast<uint16_t>(tmp, d, n, ctx->num_sms, ctx->stream); break;
                case MI_I16: launch_cast<int16_t>(tmp, d, n, ctx->num_sms, ctx->stream); break;
                case MI_U32: launch_cast<uint32_t>(tmp, d, n, ctx->num_sms, ctx->stream); break;
                case MI_I32: launch_cast<int32_t>(tmp, d, n, ctx->num_sms, ctx->stream); break;
                case MI_U64: launch_cast<unsigned long long>(tmp, d, n, ctx->num_sms, ctx->stream); break;
                case MI_I64: launch_cast<long long>(tmp, d, n, ctx->num_sms, ctx->stream); break;
                case MI_F64: launch_cast<double>(tmp, d, n, ctx->num_sms, ctx->stream); break;
                default: break;
            }
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (tmp) cudaFree(tmp);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(d);
        return mi::cuda_status(ctx, e, "mi_image_upload");
    }
    mi_image* img = new (std::nothrow) mi_image();
    if (!img) {
        cudaFree(d);
        return MI_ERR_OUT_OF_MEMORY;
    }
    img->ctx = ctx;
    img->geo = *geometry;
    img->data = d;
    img->n = n;
    *out = img;
    return MI_OK;
}

mi_status mi_image_from_device(mi_context* ctx, const float* device_ptr, const mi_geometry* geometry,
                               mi_image** out) {
    if (!ctx || !device_ptr || !out) return MI_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!geometry_ok(geometry)) return mi::set_error(ctx, MI_ERR_INVALID_ARGUMENT, "bad geometry");
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    int64_t n = geometry->size[0] * geometry->size[1] * geometry->size[2];
    float* d = nullptr;
    MI_CHECK_CUDA(ctx, cudaMalloc(&d, (size_t)n * sizeof(float)));
    cudaError_t e = cudaMemcpyAsync(d, device_ptr, (size_t)n * 4, cudaMemcpyDeviceToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(d);
        return mi::cuda_status(ctx, e, "mi_image_from_device");
    }
    mi_image* img = new (std::nothrow) mi_image();
    if (!img) {
        cudaFree(d);
        return MI_ERR_OUT_OF_MEMORY;
    }
    img->ctx = ctx;
    img->geo = *geometry;
    img->data = d;
    img->n = n;
    *out = img;
    return MI_OK;
}

mi_status mi_image_to_host(const mi_image* img, float* dst, size_t n_elements) {
    if (!img || !dst) return MI_ERR_INVALID_ARGUMENT;
    if ((int64_t)n_elements < img->n)
        return mi::set_error(img->ctx, MI_ERR_INVALID_ARGUMENT, "destination smaller than the image");
    MI_CHECK_CUDA(img->ctx, cudaSetDevice(img->ctx->device));
    MI_CHECK_CUDA(img->ctx, cudaMemcpyAsync(dst, img->data, (size_t)img->n * 4, cudaMemcpyDeviceToHost,
                                            img->ctx->stream));
    MI_CHECK_CUDA(img->ctx, cudaStreamSynchronize(img->ctx->stream));
    return MI_OK;
}

mi_status mi_image_geometry(const mi_image* img, mi_geometry* out) {
    if (!img || !out) return MI_ERR_INVALID_ARGUMENT;
    *out = img->geo;
    return MI_OK;
}

const float* mi_image_device_ptr(const mi_image* img) { return img ? img->data : nullptr; }

mi_status mi_image_free(mi_image* img) {
    if (!img) return MI_ERR_INVALID_ARGUMENT;
    cudaSetDevice(img->ctx->device);
    cudaStreamSynchronize(img->ctx->stream);
    cudaFree(img->data);
    delete img;
    return MI_OK;
}

}  // extern "C"
