// Learned initialiser: a small 3-D convolutional encoder with an MLP head that reads a
// fixed/moving pair downsampled to 32³ and proposes the 12 affine parameters a
// registration starts from. It is trained on pairs the library generates and
// registers itself (labels: the regular-step optimizer's converged result).
//
//   input 2 × 32³ → conv 3³ stride 2 (+ReLU): 16 × 16³ → 32 × 8³ → 64 × 4³ → 128 × 2³
//   → flatten 1024 → fc 256 (+ReLU) → fc 12
//
// Every convolution runs as a GEMM over im2col rows (channels-last activations; the
// column index of an im2col row is ((kz·3 + ky)·3 + kx)·Cin + c), forward and
// backward, on the tcgen05 BF16 GEMM (gemm_tc.cuh) with FP32 accumulation: forward
// Y = Xcol·Wᵀ; weight gradient dW = dYᵀ·Xcol; input gradient dXcol = dY·W, gathered
// back to the input grid (col2im as a gather, so deterministic). Operands that a TN
// GEMM needs K-contiguous are transposed into BF16 first. Master weights, biases and
// Adam moments are FP32. No reference counterpart.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "gemm_tc.cuh"
#include "internal.h"

namespace mi {

cudaError_t gemm_bf16_tn(int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb,
                         float* C, int ldc, unsigned int* err, cudaStream_t st);

namespace {

template <int NT>
cudaError_t launch_gemm(int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, float* C,
                        int ldc, int splits, unsigned int* err, cudaStream_t st) {
    const size_t sm = tc::gemm_smem<NT>();
    cudaError_t e = cudaFuncSetAttribute(tc::k_gemm_tn<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    dim3 grid((M + tc::TILE_M - 1) / tc::TILE_M, (N + NT - 1) / NT, splits);
    tc::k_gemm_tn<NT><<<grid, tc::THREADS, sm, st>>>(M, N, K, A, lda, B, ldb, C, ldc, err);
    return cudaGetLastError();
}

int n_tile(int N) { return N <= 16 ? 16 : N <= 32 ? 32 : N <= 64 ? 64 : 128; }

cudaError_t gemm_dispatch(int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb,
                          float* C, int ldc, int splits, unsigned int* err, cudaStream_t st) {
    switch (n_tile(N)) {
        case 16: return launch_gemm<16>(M, N, K, A, lda, B, ldb, C, ldc, splits, err, st);
        case 32: return launch_gemm<32>(M, N, K, A, lda, B, ldb, C, ldc, splits, err, st);
        case 64: return launch_gemm<64>(M, N, K, A, lda, B, ldb, C, ldc, splits, err, st);
        default: return launch_gemm<128>(M, N, K, A, lda, B, ldb, C, ldc, splits, err, st);
    }
}

}  // namespace

// C[M×N] = A[M×K]·B[N×K]ᵀ on the stream; the N tile follows N.
cudaError_t gemm_bf16_tn(int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb,
                         float* C, int ldc, unsigned int* err, cudaStream_t st) {
    return gemm_dispatch(M, N, K, A, lda, B, ldb, C, ldc, 1, err, st);
}

namespace {

constexpr int NCONV = 4;
constexpr int CH[NCONV + 1] = {2, 16, 32, 64, 128};
constexpr int DIM[NCONV + 1] = {32, 16, 8, 4, 2};
constexpr int FC1_IN = 128 * 8, FC1_OUT = 256, FC2_OUT = 12;
constexpr int NLAYER = NCONV + 2;

inline int kraw(int l) { return 27 * CH[l]; }          // im2col width of conv l (0-based)
inline int kpad(int l) { return (kraw(l) + 7) & ~7; }  // padded to 16-byte rows

inline int grid1(int64_t n) {
    const int64_t g = (n + 255) / 256;
    return (int)(g < 65535 * 16 ? (g < 1 ? 1 : g) : 65535 * 16);
}

#define GSTRIDE(i, n) for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

__global__ void k_to_bf16(const float* __restrict__ in, __nv_bfloat16* __restrict__ out, int64_t n) {
    GSTRIDE(i, n) out[i] = __float2bfloat16(in[i]);
}

// out[c][r] = in[r][c] (rows × cols in, cols × rows out), FP32 or BF16 in, BF16 out
template <typename T>
__global__ void k_transpose(const T* __restrict__ in, int rows, int cols, int ldi, __nv_bfloat16* __restrict__ out,
                            int ldo) {
    __shared__ float tile[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
        const int r = r0 + dy, c = c0 + threadIdx.x;
        tile[dy][threadIdx.x] = (r < rows && c < cols) ? (float)in[(int64_t)r * ldi + c] : 0.0f;
    }
    __syncthreads();
    for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
        const int c = c0 + dy, r = r0 + threadIdx.x;
        if (c < cols && r < rows) out[(int64_t)c * ldo + r] = __float2bfloat16(tile[threadIdx.x][dy]);
    }
}

template <typename T>
cudaError_t transpose(const T* in, int rows, int cols, int ldi, __nv_bfloat16* out, int ldo, cudaStream_t st) {
    dim3 g((cols + 31) / 32, (rows + 31) / 32), b(32, 8);
    k_transpose<T><<<g, b, 0, st>>>(in, rows, cols, ldi, out, ldo);
    return cudaGetLastError();
}

// im2col of a channels-last volume (B × D³ × Cin, BF16) for a 3³ stride-2 pad-1
// convolution: row (b, z, y, x) of the D/2 output grid, column ((kz·3+ky)·3+kx)·Cin + c
__global__ void k_im2col(const __nv_bfloat16* __restrict__ x, int B, int D, int Cin, int kp,
                         __nv_bfloat16* __restrict__ col) {
    const int Do = D / 2;
    const int64_t rows = (int64_t)B * Do * Do * Do;
    GSTRIDE(i, rows * kp) {
        const int64_t row = i / kp;
        const int k = (int)(i - row * kp);
        __nv_bfloat16 v = __float2bfloat16(0.0f);
        if (k < 27 * Cin) {
            const int c = k % Cin, t = k / Cin;
            const int kx = t % 3, ky = (t / 3) % 3, kz = t / 9;
            int64_t r = row;
            const int xo = (int)(r % Do);
            r /= Do;
            const int yo = (int)(r % Do);
            r /= Do;
            const int zo = (int)(r % Do);
            const int b = (int)(r / Do);
            const int xi = 2 * xo + kx - 1, yi = 2 * yo + ky - 1, zi = 2 * zo + kz - 1;
            if (xi >= 0 && xi < D && yi >= 0 && yi < D && zi >= 0 && zi < D)
                v = x[((((int64_t)b * D + zi) * D + yi) * D + xi) * Cin + c];
        }
        col[i] = v;
    }
}

// the transpose of im2col as a gather: dX(b, z, y, x, c) = Σ over the output voxels
// and kernel taps that read it of dXcol (FP32), in a fixed order
__global__ void k_col2im(const float* __restrict__ dcol, int B, int D, int Cin, int kp, float* __restrict__ dx) {
    const int Do = D / 2;
    const int64_t n = (int64_t)B * D * D * D * Cin;
    GSTRIDE(i, n) {
        int64_t r = i;
        const int c = (int)(r % Cin);
        r /= Cin;
        const int xi = (int)(r % D);
        r /= D;
        const int yi = (int)(r % D);
        r /= D;
        const int zi = (int)(r % D);
        const int b = (int)(r / D);
        float acc = 0.0f;
        for (int kz = 0; kz < 3; ++kz) {
            const int tz = zi + 1 - kz;
            if (tz < 0 || (tz & 1) || tz / 2 >= Do) continue;
            for (int ky = 0; ky < 3; ++ky) {
                const int ty = yi + 1 - ky;
                if (ty < 0 || (ty & 1) || ty / 2 >= Do) continue;
                for (int kx = 0; kx < 3; ++kx) {
                    const int tx = xi + 1 - kx;
                    if (tx < 0 || (tx & 1) || tx / 2 >= Do) continue;
                    const int64_t row = (((int64_t)b * Do + tz / 2) * Do + ty / 2) * Do + tx / 2;
                    acc += dcol[row * kp + ((kz * 3 + ky) * 3 + kx) * Cin + c];
                }
            }
        }
        dx[i] = acc;
    }
}

// z = y + bias (kept, FP32); x = ReLU(z) as BF16 (relu = 0: identity, x as FP32 into y)
__global__ void k_bias_act(float* __restrict__ y, const float* __restrict__ bias, int64_t rows, int cols,
                           __nv_bfloat16* __restrict__ x, int relu) {
    GSTRIDE(i, rows * cols) {
        const float z = y[i] + bias[i % cols];
        y[i] = z;
        if (x) x[i] = __float2bfloat16(relu ? fmaxf(z, 0.0f) : z);
    }
}

// dz = dx ⊙ (z > 0), FP32 and BF16 copies
__global__ void k_relu_back(const float* __restrict__ dx, const float* __restrict__ z, int64_t n, float* __restrict__ dz,
                            __nv_bfloat16* __restrict__ dzb) {
    GSTRIDE(i, n) {
        const float v = z[i] > 0.0f ? dx[i] : 0.0f;
        dz[i] = v;
        dzb[i] = __float2bfloat16(v);
    }
}

// column sums of rows × cols (FP32): per column, fixed chunks of rows summed in
// order, then the chunk sums in order
constexpr int SUM_CHUNK = 4096;
__global__ void k_colsum_part(const float* __restrict__ m, int64_t rows, int cols, float* __restrict__ part) {
    const int64_t nchunks = (rows + SUM_CHUNK - 1) / SUM_CHUNK;
    GSTRIDE(i, nchunks * cols) {
        const int c = (int)(i % cols);
        const int64_t ch = i / cols;
        float acc = 0.0f;
        const int64_t r1 = min(rows, (ch + 1) * SUM_CHUNK);
        for (int64_t r = ch * SUM_CHUNK; r < r1; ++r) acc += m[r * cols + c];
        part[ch * cols + c] = acc;
    }
}
__global__ void k_colsum_fold(const float* __restrict__ part, int64_t nchunks, int cols, float* __restrict__ out) {
    GSTRIDE(c, cols) {
        float acc = 0.0f;
        for (int64_t ch = 0; ch < nchunks; ++ch) acc += part[ch * cols + c];
        out[c] = acc;
    }
}

// loss = mean (out − t)², dout = 2(out − t)/n (one CTA, fixed order)
__global__ void k_mse(const float* __restrict__ out, const float* __restrict__ t, int n, float* __restrict__ dout,
                      float* __restrict__ loss) {
    __shared__ float red[256];
    float acc = 0.0f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float d = out[i] - t[i];
        dout[i] = 2.0f * d / (float)n;
        acc += d * d;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = red[0] / (float)n;
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int64_t n, float lr, float b1, float b2, float c1, float c2, float eps) {
    GSTRIDE(i, n) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// out[i] = Σ_s part[s·mn + i], slices in order
__global__ void k_sum_slices(const float* __restrict__ part, int splits, int64_t mn, float* __restrict__ out) {
    GSTRIDE(i, mn) {
        float acc = 0.0f;
        for (int s = 0; s < splits; ++s) acc += part[(int64_t)s * mn + i];
        out[i] = acc;
    }
}

// K slices for a GEMM whose M × N tiles alone would leave most SMs idle: about two
// CTAs per SM in all, at least 4 k tiles per slice
int k_splits(int M, int N, int K) {
    const int tiles = ((M + tc::TILE_M - 1) / tc::TILE_M) * ((N + n_tile(N) - 1) / n_tile(N));
    const int ktiles = (K + tc::TILE_K - 1) / tc::TILE_K;
    int s = (296 + tiles - 1) / tiles;
    s = std::min(s, std::max(1, ktiles / 4));
    return std::max(1, s);
}

// mean and standard deviation of an n-voxel image (one CTA, FP64), then the image
// normalised into channel `ch` of a channels-last two-channel volume
__global__ void k_normalise(const float* __restrict__ img, int64_t n, float* __restrict__ out, int ch) {
    __shared__ double s1[256], s2[256];
    double a = 0.0, b = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = img[i];
        a += v;
        b += v * v;
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            s1[threadIdx.x] += s1[threadIdx.x + s];
            s2[threadIdx.x] += s2[threadIdx.x + s];
        }
        __syncthreads();
    }
    const double mean = s1[0] / (double)n;
    const double var = fmax(s2[0] / (double)n - mean * mean, 1e-12);
    const float inv = (float)(1.0 / sqrt(var));
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) out[2 * i + ch] = (float)((img[i] - mean)) * inv;
}

struct Layer {
    int out, in, kp;      // W is out × kp (FP32 master; columns ≥ the true width stay 0)
    float *w, *b, *gw, *gb, *mw, *vw, *mb, *vb;
    __nv_bfloat16 *wb, *wtb;  // BF16 W (out × kp) and Wᵀ (kp × out)
};

}  // namespace
}  // namespace mi

struct mi_initnet {
    mi_context* ctx = nullptr;
    int max_batch = 0;
    mi::Layer L[mi::NLAYER];
    int step = 0;
    // activations (sized for max_batch)
    __nv_bfloat16* x0 = nullptr;               // input, BF16 channels-last
    __nv_bfloat16* col[mi::NCONV] = {};        // im2col rows
    float* z[mi::NLAYER] = {};                 // pre-activations (FP32)
    __nv_bfloat16* xb[mi::NLAYER] = {};        // activations (BF16): conv outputs, fc1
    float* out = nullptr;                      // fc2 output (alias of z[5])
    // backward scratch
    float *dz = nullptr, *dx = nullptr, *dcol = nullptr, *part = nullptr, *loss = nullptr;
    __nv_bfloat16 *dzb = nullptr, *tA = nullptr, *tB = nullptr;
    float* slices = nullptr;  // split-K partial products
    unsigned int* err = nullptr;
};

namespace mi {
namespace {

int64_t rows_of(int l, int B) {  // GEMM rows (output voxels × batch) of layer l
    if (l < NCONV) return (int64_t)B * DIM[l + 1] * DIM[l + 1] * DIM[l + 1];
    return B;
}

void free_net(mi_initnet* n) {
    if (!n) return;
    for (auto& l : n->L) {
        cudaFree(l.w);
        cudaFree(l.b);
        cudaFree(l.gw);
        cudaFree(l.gb);
        cudaFree(l.mw);
        cudaFree(l.vw);
        cudaFree(l.mb);
        cudaFree(l.vb);
        cudaFree(l.wb);
        cudaFree(l.wtb);
    }
    cudaFree(n->x0);
    for (auto p : n->col) cudaFree(p);
    for (auto p : n->z) cudaFree(p);
    for (auto p : n->xb) cudaFree(p);
    cudaFree(n->dz);
    cudaFree(n->dx);
    cudaFree(n->dcol);
    cudaFree(n->part);
    cudaFree(n->loss);
    cudaFree(n->dzb);
    cudaFree(n->tA);
    cudaFree(n->tB);
    cudaFree(n->slices);
    cudaFree(n->err);
    delete n;
}

// BF16 copies of every weight (and of its transpose) after an update
cudaError_t refresh_bf16(mi_initnet* n) {
    cudaStream_t st = n->ctx->stream;
    for (auto& l : n->L) {
        const int64_t cnt = (int64_t)l.out * l.kp;
        k_to_bf16<<<grid1(cnt), 256, 0, st>>>(l.w, l.wb, cnt);
        cudaError_t e = transpose<float>(l.w, l.out, l.kp, l.kp, l.wtb, l.out, st);
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

// C (M × N, contiguous) = A·Bᵀ, split over K where the tiles alone are few
cudaError_t mm(mi_initnet* n, int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb,
               float* C) {
    cudaStream_t st = n->ctx->stream;
    const int S = k_splits(M, N, K);
    if (S == 1) return gemm_dispatch(M, N, K, A, lda, B, ldb, C, N, 1, n->err, st);
    cudaError_t e = gemm_dispatch(M, N, K, A, lda, B, ldb, n->slices, N, S, n->err, st);
    if (e != cudaSuccess) return e;
    k_sum_slices<<<grid1((int64_t)M * N), 256, 0, st>>>(n->slices, S, (int64_t)M * N, C);
    return cudaGetLastError();
}

// floats of split-K scratch the GEMM (M, N, K) needs
size_t slice_floats(int M, int N, int K) {
    const int S = k_splits(M, N, K);
    return S > 1 ? (size_t)S * M * N : 0;
}

cudaError_t colsum(mi_initnet* n, const float* m, int64_t rows, int cols, float* out) {
    cudaStream_t st = n->ctx->stream;
    const int64_t nchunks = (rows + SUM_CHUNK - 1) / SUM_CHUNK;
    k_colsum_part<<<grid1(nchunks * cols), 256, 0, st>>>(m, rows, cols, n->part);
    k_colsum_fold<<<grid1(cols), 256, 0, st>>>(n->part, nchunks, cols, out);
    return cudaGetLastError();
}

// forward pass of B samples (input x: B × 32³ × 2 FP32, channels-last)
cudaError_t forward(mi_initnet* n, int B, const float* x) {
    cudaStream_t st = n->ctx->stream;
    const int64_t nin = (int64_t)B * 32 * 32 * 32 * 2;
    k_to_bf16<<<grid1(nin), 256, 0, st>>>(x, n->x0, nin);
    const __nv_bfloat16* cur = n->x0;
    cudaError_t e = cudaSuccess;
    for (int l = 0; l < NCONV && e == cudaSuccess; ++l) {
        const Layer& L = n->L[l];
        const int64_t rows = rows_of(l, B);
        k_im2col<<<grid1(rows * L.kp), 256, 0, st>>>(cur, B, DIM[l], CH[l], L.kp, n->col[l]);
        e = mm(n, (int)rows, L.out, L.kp, n->col[l], L.kp, L.wb, L.kp, n->z[l]);
        if (e == cudaSuccess) k_bias_act<<<grid1(rows * L.out), 256, 0, st>>>(n->z[l], L.b, rows, L.out, n->xb[l], 1);
        cur = n->xb[l];
    }
    // fc1 on the flattened conv output (B × 1024), fc2 without activation
    if (e == cudaSuccess) {
        const Layer& F1 = n->L[NCONV];
        e = mm(n, B, F1.out, F1.kp, n->xb[NCONV - 1], FC1_IN, F1.wb, F1.kp, n->z[NCONV]);
        if (e == cudaSuccess)
            k_bias_act<<<grid1((int64_t)B * F1.out), 256, 0, st>>>(n->z[NCONV], F1.b, B, F1.out, n->xb[NCONV], 1);
    }
    if (e == cudaSuccess) {
        const Layer& F2 = n->L[NCONV + 1];
        e = mm(n, B, F2.out, F2.kp, n->xb[NCONV], FC1_OUT, F2.wb, F2.kp, n->z[NCONV + 1]);
        if (e == cudaSuccess)
            k_bias_act<<<grid1((int64_t)B * F2.out), 256, 0, st>>>(n->z[NCONV + 1], F2.b, B, F2.out, nullptr, 0);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    return e;
}

// gradients of the mean squared error against target t (B × 12) into every layer's
// gw / gb; loss into n->loss
cudaError_t backward(mi_initnet* n, int B, const float* t) {
    cudaStream_t st = n->ctx->stream;
    cudaError_t e = cudaSuccess;
    float* out = n->z[NCONV + 1];
    // dOut
    k_mse<<<1, 256, 0, st>>>(out, t, B * FC2_OUT, n->dz, n->loss);
    // layers from the top; n->dz holds dZ of the current layer (FP32, rows × out)
    for (int l = NLAYER - 1; l >= 0 && e == cudaSuccess; --l) {
        Layer& L = n->L[l];
        const int64_t rows = rows_of(l, B);
        // input of the layer (BF16, rows × kp): im2col rows or the previous activation
        const __nv_bfloat16* xin = l < NCONV ? n->col[l] : n->xb[l - 1];
        const int ldx = l < NCONV ? L.kp : (l == NCONV ? FC1_IN : FC1_OUT);
        // bias gradient
        e = colsum(n, n->dz, rows, L.out, L.gb);
        // dW (out × kp) = dZᵀ · X: both operands transposed to K = rows contiguous
        if (e == cudaSuccess) e = transpose<float>(n->dz, (int)rows, L.out, L.out, n->tA, (int)rows, st);
        if (e == cudaSuccess) e = transpose<__nv_bfloat16>(xin, (int)rows, L.kp, ldx, n->tB, (int)rows, st);
        if (e == cudaSuccess) e = mm(n, L.out, L.kp, (int)rows, n->tA, (int)rows, n->tB, (int)rows, L.gw);
        if (l == 0 || e != cudaSuccess) break;
        // dX of the layer input (rows × kp) = dZ · W
        const int64_t cnt = rows * L.out;
        k_to_bf16<<<grid1(cnt), 256, 0, st>>>(n->dz, n->dzb, cnt);
        e = mm(n, (int)rows, L.kp, L.out, n->dzb, L.out, L.wtb, L.out, n->dcol);
        if (e != cudaSuccess) break;
        // back to the previous layer's activation layout, then through its ReLU
        const int pl = l - 1;
        const int64_t prows = rows_of(pl, B);
        const int pout = n->L[pl].out;
        if (l < NCONV) {
            k_col2im<<<grid1(prows * pout), 256, 0, st>>>(n->dcol, B, DIM[l], CH[l], L.kp, n->dx);
        } else {
            // fc layers read the previous activation row by row: dcol already is dX
            cudaMemcpyAsync(n->dx, n->dcol, (size_t)prows * pout * sizeof(float), cudaMemcpyDeviceToDevice, st);
        }
        k_relu_back<<<grid1(prows * pout), 256, 0, st>>>(n->dx, n->z[pl], prows * pout, n->dz, n->dzb);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace
}  // namespace mi

extern "C" {

mi_status mi_initnet_create(mi_context* ctx, uint64_t seed, int max_batch, mi_initnet** out) {
    using namespace mi;
    if (!ctx || !out || max_batch < 1) return MI_ERR_INVALID_ARGUMENT;
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    mi_initnet* n = new (std::nothrow) mi_initnet();
    if (!n) return MI_ERR_OUT_OF_MEMORY;
    n->ctx = ctx;
    n->max_batch = max_batch;
    const int B = max_batch;
    cudaError_t e = cudaSuccess;
    auto alloc = [&](auto** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc((void**)p, bytes);
        if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
    };
    // weights: He-uniform from a SplitMix64 stream seeded by `seed`
    uint64_t state = seed;
    auto next_u = [&]() {
        uint64_t z = (state += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * 0x1p-53;
    };
    size_t max_rows_kp = 0, max_rows_out = 0;
    for (int l = 0; l < NLAYER; ++l) {
        Layer& L = n->L[l];
        int fan_in;
        if (l < NCONV) {
            L.out = CH[l + 1];
            L.in = kraw(l);
            L.kp = kpad(l);
        } else if (l == NCONV) {
            L.out = FC1_OUT;
            L.in = L.kp = FC1_IN;
        } else {
            L.out = FC2_OUT;
            L.in = L.kp = FC1_OUT;
        }
        fan_in = L.in;
        const size_t wn = (size_t)L.out * L.kp;
        alloc(&L.w, wn * 4);
        alloc(&L.b, L.out * 4);
        alloc(&L.gw, wn * 4);
        alloc(&L.gb, L.out * 4);
        alloc(&L.mw, wn * 4);
        alloc(&L.vw, wn * 4);
        alloc(&L.mb, L.out * 4);
        alloc(&L.vb, L.out * 4);
        alloc(&L.wb, wn * 2);
        alloc(&L.wtb, wn * 2);
        std::vector<float> hw(wn, 0.0f);
        const double bound = std::sqrt(6.0 / fan_in) * (l == NLAYER - 1 ? 0.1 : 1.0);
        for (int o = 0; o < L.out; ++o)
            for (int k = 0; k < L.in; ++k) hw[(size_t)o * L.kp + k] = (float)((2.0 * next_u() - 1.0) * bound);
        if (e == cudaSuccess) e = cudaMemcpy(L.w, hw.data(), wn * 4, cudaMemcpyHostToDevice);
        const int64_t rows = rows_of(l, B);
        max_rows_kp = std::max(max_rows_kp, (size_t)rows * L.kp);
        max_rows_out = std::max(max_rows_out, (size_t)rows * L.out);
        alloc(&n->z[l], (size_t)rows * L.out * 4);
        if (l < NLAYER - 1) alloc(&n->xb[l], (size_t)rows * L.out * 2);
        if (l < NCONV) alloc(&n->col[l], (size_t)rows * L.kp * 2);
    }
    size_t max_slices = 0;
    for (int l = 0; l < NLAYER; ++l) {
        const Layer& L = n->L[l];
        const int rows = (int)rows_of(l, B);
        max_slices = std::max({max_slices, slice_floats(rows, L.out, L.kp), slice_floats(L.out, L.kp, rows),
                               slice_floats(rows, L.kp, L.out)});
    }
    alloc(&n->slices, std::max<size_t>(max_slices, 1) * 4);
    size_t max_act = 0;  // largest activation / input of any layer, FP32 elements
    for (int l = 0; l < NLAYER; ++l) max_act = std::max(max_act, (size_t)rows_of(l, B) * n->L[l].out);
    max_act = std::max(max_act, (size_t)B * 32 * 32 * 32 * 2);
    alloc(&n->x0, (size_t)B * 32 * 32 * 32 * 2 * 2);
    alloc(&n->dz, max_act * 4);
    alloc(&n->dx, max_act * 4);
    alloc(&n->dcol, max_rows_kp * 4);
    alloc(&n->part, (max_rows_out / SUM_CHUNK + 1024) * 4 + 65536 * 4);
    alloc(&n->loss, 4);
    alloc(&n->dzb, max_act * 2);
    alloc(&n->tA, std::max(max_rows_out, max_act) * 2);
    alloc(&n->tB, max_rows_kp * 2);
    alloc(&n->err, 4);
    if (e == cudaSuccess) e = mi::refresh_bf16(n);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        mi::free_net(n);
        return mi::cuda_status(ctx, e, "mi_initnet_create");
    }
    *out = n;
    return MI_OK;
}

mi_status mi_initnet_destroy(mi_initnet* n) {
    if (!n) return MI_ERR_INVALID_ARGUMENT;
    cudaSetDevice(n->ctx->device);
    cudaStreamSynchronize(n->ctx->stream);
    mi::free_net(n);
    return MI_OK;
}

// Layer `which` (0–3 convolutions, 4 fc1, 5 fc2): W as out × in (im2col column order
// for the convolutions) and the bias. grads != 0 reads the last computed gradients.
mi_status mi_initnet_get(mi_initnet* n, int which, int grads, float* w, float* b) {
    if (!n || which < 0 || which >= mi::NLAYER) return MI_ERR_INVALID_ARGUMENT;
    const mi::Layer& L = n->L[which];
    std::vector<float> h((size_t)L.out * L.kp);
    MI_CHECK_CUDA(n->ctx, cudaStreamSynchronize(n->ctx->stream));
    MI_CHECK_CUDA(n->ctx, cudaMemcpy(h.data(), grads ? L.gw : L.w, h.size() * 4, cudaMemcpyDeviceToHost));
    if (w)
        for (int o = 0; o < L.out; ++o) std::memcpy(w + (size_t)o * L.in, h.data() + (size_t)o * L.kp, L.in * 4);
    if (b) MI_CHECK_CUDA(n->ctx, cudaMemcpy(b, grads ? L.gb : L.b, L.out * 4, cudaMemcpyDeviceToHost));
    return MI_OK;
}

mi_status mi_initnet_set(mi_initnet* n, int which, const float* w, const float* b) {
    if (!n || which < 0 || which >= mi::NLAYER || !w || !b) return MI_ERR_INVALID_ARGUMENT;
    mi::Layer& L = n->L[which];
    std::vector<float> h((size_t)L.out * L.kp, 0.0f);
    for (int o = 0; o < L.out; ++o) std::memcpy(h.data() + (size_t)o * L.kp, w + (size_t)o * L.in, L.in * 4);
    MI_CHECK_CUDA(n->ctx, cudaMemcpy(L.w, h.data(), h.size() * 4, cudaMemcpyHostToDevice));
    MI_CHECK_CUDA(n->ctx, cudaMemcpy(L.b, b, L.out * 4, cudaMemcpyHostToDevice));
    cudaError_t e = mi::refresh_bf16(n);
    if (e == cudaSuccess) e = cudaStreamSynchronize(n->ctx->stream);
    if (e != cudaSuccess) return mi::cuda_status(n->ctx, e, "mi_initnet_set");
    return MI_OK;
}

static mi_status check_err(mi_initnet* n, cudaError_t e, const char* where) {
    unsigned int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, n->err, 4, cudaMemcpyDeviceToHost, n->ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(n->ctx->stream);
    if (e != cudaSuccess) return mi::cuda_status(n->ctx, e, where);
    if (h) {
        cudaMemsetAsync(n->err, 0, 4, n->ctx->stream);
        return mi::set_error(n->ctx, MI_ERR_TIMEOUT, "tensor-core GEMM: an mbarrier wait gave up");
    }
    return MI_OK;
}

// out (device, B × 12) = the network on x (device, B × 32³ × 2 FP32, channels-last)
mi_status mi_initnet_forward(mi_initnet* n, int B, const float* x, float* out) {
    if (!n || B < 1 || B > n->max_batch || !x || !out) return MI_ERR_INVALID_ARGUMENT;
    MI_CHECK_CUDA(n->ctx, cudaSetDevice(n->ctx->device));
    cudaError_t e = mi::forward(n, B, x);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, n->z[mi::NLAYER - 1], (size_t)B * mi::FC2_OUT * 4, cudaMemcpyDeviceToDevice, n->ctx->stream);
    return check_err(n, e, "mi_initnet_forward");
}

// One training step on B samples: forward, mean squared error against t (device,
// B × 12), backward; Adam (β1 0.9, β2 0.999, ε 1e-8) when lr > 0. loss (host) may be NULL.
mi_status mi_initnet_train_step(mi_initnet* n, int B, const float* x, const float* t, float lr, float* loss) {
    using namespace mi;
    if (!n || B < 1 || B > n->max_batch || !x || !t) return MI_ERR_INVALID_ARGUMENT;
    MI_CHECK_CUDA(n->ctx, cudaSetDevice(n->ctx->device));
    cudaStream_t st = n->ctx->stream;
    cudaError_t e = forward(n, B, x);
    if (e == cudaSuccess) e = backward(n, B, t);
    if (e == cudaSuccess && lr > 0.0f) {
        n->step += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.0f - std::pow(b1, (float)n->step), c2 = 1.0f - std::pow(b2, (float)n->step);
        for (auto& L : n->L) {
            const int64_t wn = (int64_t)L.out * L.kp;
            k_adam<<<grid1(wn), 256, 0, st>>>(L.w, L.gw, L.mw, L.vw, wn, lr, b1, b2, c1, c2, 1e-8f);
            k_adam<<<grid1(L.out), 256, 0, st>>>(L.b, L.gb, L.mb, L.vb, L.out, lr, b1, b2, c1, c2, 1e-8f);
        }
        e = cudaGetLastError();
        if (e == cudaSuccess) e = refresh_bf16(n);
    }
    mi_status s = check_err(n, e, "mi_initnet_train_step");
    if (s == MI_OK && loss) MI_CHECK_CUDA(n->ctx, cudaMemcpy(loss, n->loss, 4, cudaMemcpyDeviceToHost));
    return s;
}

// The network's input for one pair: fixed and moving resampled (linear) onto a 32³ grid
// spanning the fixed image (centre-preserving, spacing · size/32), each normalised to
// zero mean and unit variance, interleaved channels-last into out (device, 32³ × 2).
mi_status mi_initnet_prepare(mi_context* ctx, const mi_image* fixed, const mi_image* moving, float* out) {
    if (!ctx || !fixed || !moving || !out) return MI_ERR_INVALID_ARGUMENT;
    mi_geometry g = fixed->geo;
    for (int d = 0; d < 3; ++d) {
        const double f = (double)fixed->geo.size[d] / 32.0;
        g.size[d] = 32;
        g.spacing[d] = fixed->geo.spacing[d] * f;
    }
    for (int i = 0; i < 3; ++i) {
        double acc = 0.0;
        for (int j = 0; j < 3; ++j) {
            const double delta = ((double)fixed->geo.size[j] - 1.0) / 2.0 - ((double)fixed->geo.size[j] / 32.0) * 31.0 / 2.0;
            acc += fixed->geo.direction[i * 3 + j] * fixed->geo.spacing[j] * delta;
        }
        g.origin[i] = fixed->geo.origin[i] + acc;
    }
    mi_image *rf = nullptr, *rm = nullptr;
    mi_status s = mi_image_resample(ctx, fixed, &g, 0.0, &rf);
    if (s == MI_OK) s = mi_image_resample(ctx, moving, &g, 0.0, &rm);
    if (s == MI_OK) {
        mi::k_normalise<<<1, 256, 0, ctx->stream>>>(rf->data, rf->n, out, 0);
        mi::k_normalise<<<1, 256, 0, ctx->stream>>>(rm->data, rm->n, out, 1);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) s = mi::cuda_status(ctx, e, "mi_initnet_prepare");
    }
    mi_image_free(rf);
    mi_image_free(rm);
    return s;
}

mi_status mi_gemm_bf16_tn(mi_context* ctx, int M, int N, int K, const void* A, int lda, const void* B, int ldb,
                          float* C, int ldc) {
    if (!ctx || M < 1 || N < 1 || K < 1 || !A || !B || !C || lda < K || ldb < K || ldc < N)
        return MI_ERR_INVALID_ARGUMENT;
    MI_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    unsigned int* err = nullptr;
    MI_CHECK_CUDA(ctx, cudaMalloc(&err, sizeof(unsigned int)));
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(unsigned int), ctx->stream);
    // a product whose M × N tiles alone would leave most SMs idle is split over K into
    // partial products summed in slice order, as the network's layers do
    const int S = ldc == N ? mi::k_splits(M, N, K) : 1;
    float* slices = nullptr;
    if (e == cudaSuccess && S > 1) e = cudaMalloc(&slices, (size_t)S * M * N * sizeof(float));
    const auto* a16 = static_cast<const __nv_bfloat16*>(A);
    const auto* b16 = static_cast<const __nv_bfloat16*>(B);
    if (e == cudaSuccess && S > 1) {
        e = mi::gemm_dispatch(M, N, K, a16, lda, b16, ldb, slices, N, S, err, ctx->stream);
        if (e == cudaSuccess) {
            mi::k_sum_slices<<<mi::grid1((int64_t)M * N), 256, 0, ctx->stream>>>(slices, S, (int64_t)M * N, C);
            e = cudaGetLastError();
        }
    } else if (e == cudaSuccess) {
        e = mi::gemm_bf16_tn(M, N, K, a16, lda, b16, ldb, C, ldc, err, ctx->stream);
    }
    unsigned int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(slices);
    cudaFree(err);
    if (e != cudaSuccess) return mi::cuda_status(ctx, e, "mi_gemm_bf16_tn");
    if (h) return mi::set_error(ctx, MI_ERR_TIMEOUT, "tensor-core GEMM: an mbarrier wait gave up");
    return MI_OK;
}

}  // extern "C"
