// Asynchronous copies into shared memory: mbarriers with bounded waits, bulk
// (1-D) and tensor-tile (3-D) TMA loads, and the host-side tensor-map encoder.
//
// Every copy completes on an mbarrier through the transaction count; every
// wait is bounded (kSpinLimit polls) and, when it gives up, records
// AMCFD_E_TIMEOUT in the device status block so the host reports an error
// instead of hanging.  No copy here uses cluster multicast.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "amcfd.h"
#include "dev.cuh"

namespace amcfd {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Arrival count 1: one thread arms the barrier with the expected bytes.
__device__ __forceinline__ void mbar_init(uint64_t *bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrival count n: completes a phase once n threads have arrived.
__device__ __forceinline__ void mbar_init_n(uint64_t *bar, uint32_t n)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(n) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes) : "memory");
}

// Poll phase `parity` of `bar` at most `limit` times.
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity, long long limit)
{
    const uint32_t a = smem_u32(bar);
    for (long long it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// Bounded wait; on timeout records AMCFD_E_TIMEOUT (detail `where`) and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, Status *st, int where = -1)
{
    if (mbar_try(bar, parity, kSpinLimit)) return true;
    if (atomicCAS(&st->error, 0, AMCFD_E_TIMEOUT) == 0) st->error_where = where;
    return false;
}

// Orders earlier generic-proxy accesses of shared memory before later async-proxy copies.
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Orders earlier generic-proxy writes of global memory before later async-proxy
// copies that read them.
__device__ __forceinline__ void fence_proxy_async_global()
{
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

// 1-D bulk copy global -> shared (both 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

// 3-D tensor-tile load of the box at (x, y, z) (x a multiple of 16 bytes;
// out-of-range coordinates read zeros).  `map` is the address of a
// __grid_constant__ kernel parameter.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z),
          "r"(smem_u32(bar)) : "memory");
}

// Host: tiled 3-D tensor map (zero fill out of range); dims innermost first,
// strides in bytes of dims 1 and 2; swizzle_bytes 0 (none), 32, 64 or 128.
// Returns 0 or a CUDA driver error code.
int encode_tiled_3d(CUtensorMap *map, CUtensorMapDataType dtype, const void *base, const uint64_t dims[3],
                    const uint64_t strides[2], const uint32_t box[3], int swizzle_bytes);

// Host: tiled 3-D tensor map over a padded field [nk][nj][nip] of `elem`-byte
// elements, box (bx, by, 1).  Returns 0 or a CUDA driver error code.
int encode_field_map(CUtensorMap *map, const void *base, int elem, int nip, int nj, int nk, int bx,
                     int by);

}  // namespace amcfd
