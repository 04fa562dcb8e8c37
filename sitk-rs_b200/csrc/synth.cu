// Device twin of the counter-based synthetic pair (sitk_b200/synth.py,
// make_pair_counter): a ramp plus Gaussian blobs, a fixed image with counter-based
// Gaussian noise, and a moving image that is the noiseless volume resampled
// (trilinear, clamp-to-edge) through a centred affine, plus its own noise. Same
// expressions and order as the numpy version, in FP64 with separately rounded
// operations; the two agree to the rounding of exp, log and cos. No reference
// counterpart: the reference's benchmarks name no dataset and this builds their
// synthetic stand-ins.
#include <cmath>
#include <new>

#include "internal.h"

namespace {

constexpr unsigned long long GAMMA = 0x9E3779B97F4A7C15ull;

__host__ __device__ inline unsigned long long mix64(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// N(0, 1) number i of the field keyed `key` (synth.py counter_normal)
__device__ inline double counter_normal(unsigned long long key, unsigned long long i) {
    const unsigned long long a = mix64(key + (2ull * i + 1ull) * GAMMA);
    const unsigned long long b = mix64(key + (2ull * i + 2ull) * GAMMA);
    const double u1 = __dmul_rn((double)(a >> 11), 0x1p-53);
    const double u2 = __dmul_rn((double)(b >> 11), 0x1p-53);
    const double r = sqrt(__dmul_rn(-2.0, log(__dsub_rn(1.0, u1))));
    return __dmul_rn(r, cos(__dmul_rn(__dmul_rn(2.0, 3.141592653589793), u2)));
}

struct Blob {
    double sigma, amp, c[3];
    int lo[3], hi[3];  // the ±3.5σ box, clipped to the grid
};

// ramp + blobs (render_phantom) into base (FP64); fixed = base + noise·z
__global__ void k_synth_base(int n, int nblobs, const Blob* __restrict__ blobs, unsigned long long key,
                             double noise, double* __restrict__ base, float* __restrict__ fixed) {
    const long long nv = (long long)n * n * n;
    const double den = __dmul_rn(1.75, (double)(n - 1 > 1 ? n - 1 : 1));
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nv; q += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(q % n), y = (int)((q / n) % n), z = (int)(q / ((long long)n * n));
        const double s = __dadd_rn(__dadd_rn((double)x, __dmul_rn(0.5, (double)y)), __dmul_rn(0.25, (double)z));
        double v = __dadd_rn(20.0, __ddiv_rn(__dmul_rn(40.0, s), den));
        for (int b = 0; b < nblobs; ++b) {
            const Blob& B = blobs[b];
            if (x < B.lo[0] || x >= B.hi[0] || y < B.lo[1] || y >= B.hi[1] || z < B.lo[2] || z >= B.hi[2]) continue;
            const double dx = __dsub_rn((double)x, B.c[0]);
            const double dy = __dsub_rn((double)y, B.c[1]);
            const double dz = __dsub_rn((double)z, B.c[2]);
            const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dz, dz), __dmul_rn(dy, dy)), __dmul_rn(dx, dx));
            const double g = exp(__ddiv_rn(__dmul_rn(-0.5, d2), __dmul_rn(B.sigma, B.sigma)));
            v = __dadd_rn(v, __dmul_rn(B.amp, g));
        }
        base[q] = v;
        fixed[q] = (float)__dadd_rn(v, __dmul_rn(noise, counter_normal(key, (unsigned long long)q)));
    }
}

// moving(x) = base(m·(x − c) + c + t) (trilinear, coordinates clamped to the grid,
// synth.py resample_linear) + noise·z
__global__ void k_synth_warp(int n, const double* __restrict__ base, double m0, double m1, double m2, double m3,
                             double m4, double m5, double m6, double m7, double m8, double t0, double t1, double t2,
                             double cc, unsigned long long key, double noise, float* __restrict__ moving) {
    const long long nv = (long long)n * n * n;
    const double m[9] = {m0, m1, m2, m3, m4, m5, m6, m7, m8};
    const double t[3] = {t0, t1, t2};
    const double hi = (double)(n - 1);
    for (long long qi = (long long)blockIdx.x * blockDim.x + threadIdx.x; qi < nv;
         qi += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(qi % n), y = (int)((qi / n) % n), z = (int)(qi / ((long long)n * n));
        const double px = __dsub_rn((double)x, cc), py = __dsub_rn((double)y, cc), pz = __dsub_rn((double)z, cc);
        double q[3];
        for (int r = 0; r < 3; ++r) {
            double acc = __dadd_rn(__dadd_rn(__dmul_rn(m[r * 3], px), __dmul_rn(m[r * 3 + 1], py)), __dmul_rn(m[r * 3 + 2], pz));
            acc = __dadd_rn(__dadd_rn(acc, cc), t[r]);
            q[r] = fmin(fmax(acc, 0.0), hi);
        }
        long long i0[3];
        double fr[3];
        for (int d = 0; d < 3; ++d) {
            long long f = (long long)floor(q[d]);
            if (f > n - 2) f = n - 2;
            i0[d] = f;
            fr[d] = __dsub_rn(q[d], (double)f);
        }
        double acc = 0.0;
        for (int dz = 0; dz < 2; ++dz) {
            const double wz = dz ? fr[2] : __dsub_rn(1.0, fr[2]);
            for (int dy = 0; dy < 2; ++dy) {
                const double wy = dy ? fr[1] : __dsub_rn(1.0, fr[1]);
                for (int dx = 0; dx < 2; ++dx) {
                    const double wx = dx ? fr[0] : __dsub_rn(1.0, fr[0]);
                    const long long off = (i0[0] + dx) + (long long)n * ((i0[1] + dy) + (long long)n * (i0[2] + dz));
                    acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(__dmul_rn(wz, wy), wx), base[off]));
                }
            }
        }
        moving[qi] = (float)__dadd_rn(acc, __dmul_rn(noise, counter_normal(key, (unsigned long long)qi)));
    }
}

mi_status new_cube(mi_context* ctx, int n, mi_image** out) {
    mi_geometry g{};
    for (int d = 0; d < 3; ++d) {
        g.size[d] = n;
        g.spacing[d] = 1.0;
        g.origin[d] = 0.0;
    }
    g.direction[0] = g.direction[4] = g.direction[8] = 1.0;
    const int64_t nv = (int64_t)n * n * n;
    float* d = nullptr;
    MI_CHECK_CUDA(ctx, cudaMalloc(&d, (size_t)nv * sizeof(float)));
    mi_image* img = new (std::nothrow) mi_image();
    if (!img) {
        cudaFree(d);
        return MI_ERR_OUT_OF_MEMORY;
    }
    img->ctx = ctx;
    img->geo = g;
    img->data = d;
    img->n = nv;
    *out = img;
    return MI_OK;
}

}  // namespace

extern "C" {

mi_status mi_synth_pair(mi_context* ctx, int n, int nblobs, const double* blobs5, const double* affine12,
                        uint64_t seed, double noise, mi_image** fixed, mi_image** moving) {
    if (!ctx || n < 2 || nblobs < 0 || (nblobs > 0 && !blobs5) || !affine12 || !fixed || !moving)
        return MI_ERR_INVALID_ARGUMENT;
    *fixed = nullptr;
    *moving = nullptr;
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    std::vector<Blob> hb(nblobs > 0 ? nblobs : 1);
    for (int b = 0; b < nblobs; ++b) {
        Blob& B = hb[b];
        B.sigma = blobs5[b * 5];
        B.amp = blobs5[b * 5 + 1];
        const int r = (int)std::ceil(3.5 * B.sigma);
        for (int d = 0; d < 3; ++d) {
            B.c[d] = blobs5[b * 5 + 2 + d];
            B.lo[d] = std::max((int)B.c[d] - r, 0);
            B.hi[d] = std::min((int)B.c[d] + r + 1, n);
        }
    }
    mi_image *f = nullptr, *m = nullptr;
    mi_status s = new_cube(ctx, n, &f);
    if (s == MI_OK) s = new_cube(ctx, n, &m);
    if (s != MI_OK) {
        mi_image_free(f);
        return s;
    }
    const long long nv = (long long)n * n * n;
    Blob* db = nullptr;
    double* base = nullptr;
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaMalloc(&db, hb.size() * sizeof(Blob));
    if (e == cudaSuccess) e = cudaMemcpyAsync(db, hb.data(), hb.size() * sizeof(Blob), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMalloc(&base, (size_t)nv * sizeof(double));
    const unsigned long long kf = mix64((unsigned long long)seed + 1ull * GAMMA);
    const unsigned long long km = mix64((unsigned long long)seed + 2ull * GAMMA);
    const int grid = (int)std::min<long long>((nv + 255) / 256, (long long)ctx->num_sms * 16);
    if (e == cudaSuccess) {
        k_synth_base<<<grid, 256, 0, st>>>(n, nblobs, db, kf, noise, base, f->data);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        const double* a = affine12;
        k_synth_warp<<<grid, 256, 0, st>>>(n, base, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10],
                                          a[11], (double)(n - 1) / 2.0, km, noise, m->data);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(db);
    cudaFree(base);
    if (e != cudaSuccess) {
        mi_image_free(f);
        mi_image_free(m);
        return mi::cuda_status(ctx, e, "mi_synth_pair");
    }
    *fixed = f;
    *moving = m;
    return MI_OK;
}

}  // extern "C"
