// staging.cuh -- TMA staging of a column tile's z-planes into shared memory.
//
// A block owns a tile of tx x ty columns and marches down k.  Each
// input array of a sweep is copied chunk by chunk (CH planes at a time) into
// shared memory by the Tensor Memory Accelerator: one thread arms the chunk's
// mbarrier with the expected byte count and issues one
// cp.async.bulk.tensor.3d per array; all threads wait on the mbarrier.  Two
// buffers alternate, so chunk s+1 streams in while chunk s is consumed.
//
// Boxes (x, y, z) for a tile of tx x ty columns, all starting at 16-byte
// aligned x (the TMA rule):
//   halo arrays (read at x/y neighbours): x from x0 - XOFF, width
//     BW = tx + 2*XOFF with XOFF = 16 / sizeof(element), y from y0 - 1,
//     height ty + 2;  shared layout [CH][ty+2][BW]
//   own arrays (read at the thread's column): x0, y0, tx x ty;
//     shared layout [CH][ty*tx]
// Coordinates outside the domain (including the negative halo origin) are
// zero-filled by the TMA unit.  Loads only, never multicast.
#pragma once

#include <cuda.h>

#include "device_common.cuh"

#define OWN_PLANE TILE_THREADS

// Halo layout of a tile of tx x ty columns (tx * ty = TILE_THREADS): planes of
// (tx + 2 XOFF) x (ty + 2) elements.  The two supported shapes, 32 x 4 and
// 16 x 8, have equal planes in FP32 (40 x 6 = 24 x 10 = 240) and nearly equal
// ones in FP64 (36 x 6 = 216, 20 x 10 = 200), so one slot size serves both.
template <typename V>
struct Halo {
    static constexpr int XOFF = 16 / (int)sizeof(V);
    static constexpr int P32 = (32 + 2 * XOFF) * (4 + 2), P16 = (16 + 2 * XOFF) * (8 + 2);
    static constexpr int PLANE_MAX = P32 > P16 ? P32 : P16;
    int bw, plane, hc;  // row width, plane size, the thread's own column
    __device__ __forceinline__ Halo(int tx, int tx_log2, int ty)
        : bw(tx + 2 * XOFF), plane((tx + 2 * XOFF) * (ty + 2)),
          hc((((int)threadIdx.x >> tx_log2) + 1) * (tx + 2 * XOFF) + ((int)threadIdx.x & (tx - 1)) + XOFF) {}
};

__device__ __forceinline__ unsigned smem_addr(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred P;\n mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n selp.u32 %0, 1, 0, P;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Waits for the chunk of buffer b; gives up after MBAR_TIMEOUT_NS and raises
// the handle's error flag (the grid barrier then ends the kernel).
#define MBAR_TIMEOUT_NS 2000000000ull
#define DRAIN_TIMEOUT_NS 500000000ull
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, GridBarrier *gb) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*(volatile int *)&gb->error) return false;
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > MBAR_TIMEOUT_NS) {
            atomicExch(&gb->error, 1);
            return false;
        }
    }
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

// L2 prefetch of the box a load at the same coordinates would copy: no shared
// memory and no mbarrier, only the DRAM reads of a later chunk started early.
__device__ __forceinline__ void tma_prefetch_3d(const CUtensorMap *map, int x, int y, int z) {
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];\n" ::"l"(map), "r"(x),
                 "r"(y), "r"(z)
                 : "memory");
}

// Box loads of one array for planes [k0, k0 + CHN) of the tile at (x0, y0).
template <typename V, int CHN>
__device__ __forceinline__ void tma_halo(V *dst, const CUtensorMap *map, int x0, int y0, int k0,
                                         uint64_t *bar) {
    tma_load_3d(dst, map, x0 - Halo<V>::XOFF, y0 - 1, k0, bar);
}
template <typename V, int CHN>
__device__ __forceinline__ void tma_own(V *dst, const CUtensorMap *map, int x0, int y0, int k0,
                                        uint64_t *bar) {
    tma_load_3d(dst, map, x0, y0, k0, bar);
}
template <typename V>
__device__ __forceinline__ void tma_halo_prefetch(const CUtensorMap *map, int x0, int y0, int k0) {
    tma_prefetch_3d(map, x0 - Halo<V>::XOFF, y0 - 1, k0);
}
__device__ __forceinline__ void tma_own_prefetch(const CUtensorMap *map, int x0, int y0, int k0) {
    tma_prefetch_3d(map, x0, y0, k0);
}
// bytes of a halo box of CHN planes for a tile tx wide and ty high
template <typename V, int CHN>
__device__ __forceinline__ unsigned halo_bytes(int tx, int ty) {
    return (unsigned)(CHN * (tx + 2 * Halo<V>::XOFF) * (ty + 2) * sizeof(V));
}
template <typename V, int CHN>
constexpr unsigned own_bytes() {
    return (unsigned)(CHN * OWN_PLANE * sizeof(V));
}
// Stride of a halo box's slot in a staging buffer: the largest box of the
// supported shapes, rounded up to 128 bytes (the TMA writes shared memory at
// 128-byte aligned addresses); the transaction count stays halo_bytes.
template <typename V, int CHN>
constexpr unsigned halo_slot() {
    return ((unsigned)(CHN * Halo<V>::PLANE_MAX * sizeof(V)) + 127u) & ~127u;
}

// Block-uniform state of the staging buffers: mbarriers and the parity each
// buffer's next completion will have.  `pending` (meaningful in thread 0, the
// one that issues) marks buffers with a copy issued and not yet consumed.
struct StageBars {
    uint64_t *bar;      // bar[0 .. STAGES-1] in shared memory
    unsigned parity;    // bit b: expected parity of buffer b
    GridBarrier *gb;
    unsigned pending;
    __device__ __forceinline__ void issued(int b) { pending |= 1u << b; }
    // A wait that gives up leaves its buffer pending, with the parity it was
    // waiting for, so drain() can still wait for that copy.
    __device__ __forceinline__ bool wait(int b) {
        const bool ok = mbar_wait(bar + b, (parity >> b) & 1u, gb);
        if (ok) {
            parity ^= 1u << b;
            pending &= ~(1u << b);
        }
        return ok;
    }
    // On an error exit: waits, bounded by DRAIN_TIMEOUT_NS per buffer, for
    // every copy this thread issued and nothing consumed, so no TMA write
    // into the block's shared memory is in flight when the block exits.
    __device__ __forceinline__ void drain() {
        for (int b = 0; b < STAGES; ++b) {
            if (!((pending >> b) & 1u)) continue;
            const unsigned long long t0 = global_ns();
            while (!mbar_try_wait(bar + b, (parity >> b) & 1u) && global_ns() - t0 < DRAIN_TIMEOUT_NS) {
            }
        }
        pending = 0;
    }
};
