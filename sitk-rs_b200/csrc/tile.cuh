// The histogram pass with TMA-staged moving tiles (the brick layout's other corner
// source). Per brick, one cp.async.bulk.tensor 3-D box load brings the part of the
// moving volume the brick's samples can touch into shared memory; the samples then read
// their eight corners from there instead of through the texture unit.
//
// Shape: one CTA per SM, sixteen consumer warps and one producer warp. The CTA walks a
// contiguous range of chunks, brick (run) after brick, through a ring of `stages` tile
// buffers: the producer's lane 0 waits until the consumers have released a buffer
// (`empty` mbarrier, one arrival per consumer warp), computes the brick's origin and
// tile, and issues the box load completing on the buffer's `full` mbarrier; a consumer
// warp waits on `full`, takes the brick's chunks whose index is its warp index modulo
// sixteen, and arrives on `empty`. Every wait is bounded (TILE_WAIT_LIMIT polls): on
// time-out the warp raises the evaluation's error word and leaves its loop, so a launch
// that lost a load ends instead of hanging; the host then reports MI_ERR_TIMEOUT.
//
// Per sample the pass runs the texture pass's chain (prep_fast, finish_fast, the exact
// chain where a decision is open, hist_phase's taps and records) with the corners read
// from the tile, so it takes the same decisions, routes the same samples to the exact
// chain and forms the same histogram and records, to the bit. A brick is staged only
// when every cell its samples can use lies inside the moving volume (no clamp-to-edge
// needed) and inside the box; a staged sample whose cell would fall outside the box
// (which the construction excludes) and every sample of an unstaged brick read the
// texture. The box's x origin is a multiple of four voxels (16 bytes, the TMA rule for
// the innermost coordinate); loads only, no multicast.
#pragma once

#include <cuda.h>

#include <cstdint>

#include "brick.cuh"

namespace mi {
namespace {

constexpr int TILE_CONSUMER_WARPS = 16;
constexpr int TILE_BLOCK = (TILE_CONSUMER_WARPS + 1) * 32;
constexpr int TILE_MAX_STAGES = 4;
// A wait gives up after TILE_WAIT_LIMIT polls, each suspending the warp for at most
// TILE_WAIT_HINT_NS (about half a second in all).
constexpr uint32_t TILE_WAIT_LIMIT = 1u << 18;
constexpr uint32_t TILE_WAIT_HINT_NS = 2000u;

// Per-evaluation tile geometry and the shared-memory layout after the histogram.
struct TileArgs {
    int bx, by, bz;           // box in voxels (bx a multiple of 4)
    int stages;               // tile buffers in the ring
    uint32_t tile_floats;     // bx·by·bz
    uint32_t tile_stride;     // floats from one buffer to the next (a multiple of 32: 128-byte aligned)
    uint32_t tile_off;        // byte offset of buffer 0 (128-byte aligned)
    uint32_t meta_off;        // byte offset of the per-buffer brick constants
    uint32_t bar_off;         // byte offset of the mbarriers (full[stages], empty[stages])
    const uint32_t* run_chunk0;  // first chunk of every run, [nruns + 1]
    unsigned int* err;        // the evaluation's error word (sync[3])
};

// What the producer hands the consumers with a buffer: the brick's constants and its
// tile origin (ok = 0: the brick takes the texture path).
struct TileMeta {
    BrickBase b;
    int ox, oy, oz, ok;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(TILE_WAIT_HINT_NS)
        : "memory");
    return ok != 0u;
}
// Bounded wait for the phase of the given parity; false on time-out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t i = 0; i < TILE_WAIT_LIMIT; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tma_load_3d(float* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

// The brick's tile: every cell its samples can use lies in [floor(co + lo_ext),
// floor(co + hi_ext) + 1] per axis (lo_ext/hi_ext carry the bound's margin). Staged when
// that range lies inside the moving volume and inside the box with the x origin rounded
// down to a multiple of four.
__device__ __forceinline__ TileMeta tile_meta(const SamplerParams& P, const TileArgs& T, uint32_t packed) {
    TileMeta t;
    t.b = brick_base(P, packed);
    const double l0 = floor(t.b.co[0] + P.lo_ext[0]), h0 = floor(t.b.co[0] + P.hi_ext[0]) + 1.0;
    const double l1 = floor(t.b.co[1] + P.lo_ext[1]), h1 = floor(t.b.co[1] + P.hi_ext[1]) + 1.0;
    const double l2 = floor(t.b.co[2] + P.lo_ext[2]), h2 = floor(t.b.co[2] + P.hi_ext[2]) + 1.0;
    const bool in = l0 >= 0.0 && l1 >= 0.0 && l2 >= 0.0 && h0 <= (double)(P.msz[0] - 1) &&
                    h1 <= (double)(P.msz[1] - 1) && h2 <= (double)(P.msz[2] - 1);
    t.ox = in ? ((int)l0 & ~3) : 0;
    t.oy = in ? (int)l1 : 0;
    t.oz = in ? (int)l2 : 0;
    t.ok = in && h0 - (double)t.ox < (double)T.bx && h1 - (double)t.oy < (double)T.by &&
                   h2 - (double)t.oz < (double)T.bz
               ? 1
               : 0;
    return t;
}

// One sample of the walk (flat index `flat`, walk position `ws`, fixed bin `fi`): the
// texture pass's chain with the corners from the staged tile when the brick is staged.
template <bool RECORD>
__device__ __forceinline__ void tile_sample(const SamplerParams& P, const EvalArgs& a, const BrickHist& h,
                                            const TileArgs& T, const TileMeta& t, const float* tile, uint32_t flat,
                                            uint32_t ws, int fi) {
    Prep p;
    int st;
    if (t.ok) {
        st = prep_fast_src<RECORD>(P, flat, a.mmask, p, [&](const double* fl, float* v) {
            const int x = (int)fl[0] - t.ox, y = (int)fl[1] - t.oy, z = (int)fl[2] - t.oz;
            if ((unsigned)x < (unsigned)(T.bx - 1) && (unsigned)y < (unsigned)(T.by - 1) &&
                (unsigned)z < (unsigned)(T.bz - 1)) {
                const int sx = T.bx, sxy = T.bx * T.by;
                const float* q = tile + (z * T.by + y) * T.bx + x;
                v[0] = q[0];
                v[1] = q[1];
                v[2] = q[sx];
                v[3] = q[sx + 1];
                v[4] = q[sxy];
                v[5] = q[sxy + 1];
                v[6] = q[sxy + sx];
                v[7] = q[sxy + sx + 1];
            } else {
                fetch_corners(P, fl, v);
            }
        });
    } else {
        st = prep_fast<RECORD>(P, flat, a.mmask, p);
    }
    Sample o;
    if (st == SAMPLE_VALID) st = finish_fast<RECORD>(P, p, o);
    if (st == SAMPLE_EXACT || st == SAMPLE_EXACT_CELL) {
        Sample e;
        st = st == SAMPLE_EXACT ? sample_exact<RECORD>(P, flat, a.moving, a.mmask, e)
                                : sample_exact_cell<RECORD>(P, flat, p.v, e);
        brick_account<RECORD>(a, h, P.bins, st, e, ws, fi);
    } else {
        brick_account<RECORD>(a, h, P.bins, st, o, ws, fi);
    }
}

// Pass 1 with staged tiles (see the file comment). Launched with TILE_BLOCK threads.
template <bool RECORD>
__device__ __forceinline__ void tile_hist_phase(const SamplerParams& P, const EvalArgs& a, const CUtensorMap* tmap,
                                                const TileArgs& T, unsigned char* smem) {
    const int B = P.bins;
    unsigned int* sh = reinterpret_cast<unsigned int*>(smem);
    brick_hist_zero(a, sh, B);
    float* tiles = reinterpret_cast<float*>(smem + T.tile_off);
    TileMeta* meta = reinterpret_cast<TileMeta*>(smem + T.meta_off);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + T.bar_off);
    uint64_t* empty = full + T.stages;
    if (threadIdx.x == 0) {
        for (int s = 0; s < T.stages; ++s) {
            mbar_init(full + s, 1u);
            mbar_init(empty + s, (uint32_t)TILE_CONSUMER_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const uint32_t nch = a.nchunks;
    const uint32_t c0 = (uint32_t)(((uint64_t)blockIdx.x * nch) / gridDim.x);
    const uint32_t c1 = (uint32_t)(((uint64_t)(blockIdx.x + 1) * nch) / gridDim.x);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int S = T.stages;
    if (c0 < c1) {
        const uint32_t r0 = __ldg(a.chunk_run + c0), nr = __ldg(a.chunk_run + c1 - 1) - r0 + 1;
        if (warp == TILE_CONSUMER_WARPS) {
            // producer: lane 0 fills the ring
            if (lane == 0) {
                for (uint32_t ri = 0; ri < nr; ++ri) {
                    const int s = (int)(ri % (uint32_t)S);
                    if (ri >= (uint32_t)S && !mbar_wait(empty + s, ((ri / (uint32_t)S) - 1u) & 1u)) {
                        atomicOr(T.err, 2u);
                        break;
                    }
                    const TileMeta t = tile_meta(P, T, __ldg(a.run_brick + r0 + ri));
                    meta[s] = t;
                    if (t.ok) {
                        // the buffer's last readers were generic-proxy loads ordered before the
                        // empty barrier; order them before the async-proxy write
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        mbar_expect_tx(full + s, T.tile_floats * 4u);
                        tma_load_3d(tiles + (size_t)s * T.tile_stride, tmap, t.ox, t.oy, t.oz, full + s);
                    } else {
                        mbar_arrive(full + s);
                    }
                }
            }
        } else {
            const BrickHist h = brick_hist_lane(a, sh, B);
            const uint32_t* __restrict__ codes = a.codes;
            const int fshift = 3 * P.brick_bl;
            for (uint32_t ri = 0; ri < nr; ++ri) {
                const int s = (int)(ri % (uint32_t)S);
                if (!mbar_wait(full + s, (ri / (uint32_t)S) & 1u)) {
                    atomicOr(T.err, 2u);
                    break;
                }
                const TileMeta t = meta[s];
                const float* tile = tiles + (size_t)s * T.tile_stride;
                const uint32_t r = r0 + ri;
                const uint32_t cr0 = max(__ldg(T.run_chunk0 + r), c0), cr1 = min(__ldg(T.run_chunk0 + r + 1), c1);
                // this warp's chunks of the brick: index ≡ warp (mod 16)
                const uint32_t first = cr0 + (((uint32_t)warp + 16u - (cr0 & 15u)) & 15u);
                // walk position of the run's padded position 0
                const uint32_t wbase = __ldg(a.run_start + r) - __ldg(T.run_chunk0 + r) * BRICK_CHUNK;
                uint32_t code = first < cr1 ? __ldg(codes + (size_t)first * BRICK_CHUNK + lane) : BRICK_PAD;
                for (uint32_t c = first; c < cr1; c += TILE_CONSUMER_WARPS) {
                    const uint32_t cn = c + TILE_CONSUMER_WARPS;
                    const uint32_t code_n = cn < cr1 ? __ldg(codes + (size_t)cn * BRICK_CHUNK + lane) : BRICK_PAD;
                    if (code != BRICK_PAD) {
                        // the record's position in the walk: from the run's start, or the voxel
                        // itself when the walk is the whole grid in voxel order
                        const uint32_t flat = brick_flat(P, t.b.packed, code);
                        tile_sample<RECORD>(P, a, h, T, t, tile, flat, a.samples ? wbase + c * BRICK_CHUNK + lane : flat,
                                            (int)(code >> fshift));
                    }
                    code = code_n;
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(empty + s);
            }
        }
    }
    __syncthreads();
    brick_hist_flush(a, sh, B);
}

}  // namespace
}  // namespace mi
