// TMA (cp.async.bulk.tensor) tile staging for the stencil phases.
//
// A 2-D tensor map describes one array of the padded field layout: inner
// extent P (the pitch, elements), outer extent R rows, row stride P * size.
// Boxes are loaded into shared memory by one thread and completed on an
// mbarrier with an expected byte count; reads outside the tensor extents are
// filled with zeros by the hardware.
//
// Alignment: every box starts at an x coordinate that is a multiple of 32
// elements (the tile origins below) and its inner extent in bytes is a
// multiple of 16, as cp.async.bulk.tensor requires.  No multicast is used.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "cp_device.cuh"

namespace cp {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with the given parity; false after limitNs
// (2 s by default).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* err,
                                          unsigned long long limitNs = kBarrierNs) {
    unsigned spins = 0;
    unsigned long long t0 = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (((++spins) & 1023u) == 0) {
            const unsigned long long t = globaltimer_ns();
            if (t0 == 0) t0 = t;
            else if (t - t0 > limitNs) {
                atomicCAS(err, 0, (int)CP_ERR_TIMEOUT);
                return false;
            }
        }
    }
    return true;
}

// Order this thread's later async-proxy (TMA) reads of global memory after
// generic-proxy writes made visible to it (e.g. by a grid barrier).
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Tile geometry of the level-0 stencil phases: R x C unknowns with a
// one-cell halo, loaded as boxes of (R + 2) x BoxW elements whose origin is
// (x = C * tJ, y = R * tI) in array coordinates (the unknowns start at
// i = j = 1, so the halo column/row sits exactly on a multiple of C / R).
// The coarse (level-1) box of the prolongation covers rows (R / 2) tI ..
// (R / 2) tI + R / 2 + 1 and columns (C / 2) tJ .. (C / 2) tJ + C / 2 + 3.
// Rows by element size: 32 for float (a CTA walks half as many tiles as with
// 16, -6 % per CG iteration at 2048 x 1024, measured; 16 x 128 timed the
// same, 64 rows slower), 16 for double (32 rows fill 217 KB of shared memory
// for two stages and measured slower).
#ifndef CP_TILE_R_FLOAT
#define CP_TILE_R_FLOAT 32
#endif
#ifndef CP_TILE_C_FLOAT
#define CP_TILE_C_FLOAT 64
#endif
template <typename TV>
struct TileGeom {
    static constexpr int R = sizeof(TV) == 4 ? CP_TILE_R_FLOAT : 16;
    static constexpr int C = sizeof(TV) == 4 ? CP_TILE_C_FLOAT : 64;
    static constexpr int BoxR = R + 2;
    static constexpr int BoxW = C + 4;        // >= C + 2 and a multiple of 16 bytes for 4- and 8-byte types
    static constexpr int CBoxR = R / 2 + 2;
    static constexpr int CBoxW = C / 2 + 4;
};

}  // namespace cp
