// fdtd_tma.h — the PTX the TMA/mbarrier step kernels share: shared-memory
// addresses, mbarriers with wall-time-bounded waits, plain 3-D tiled TMA
// loads into the issuing CTA's own shared memory, and the tensor-map acquire;
// and the host encoder of a tensor map over one padded field.
#pragma once

#include "fdtd_internal.h"

#include <cuda.h>

namespace fdtd {

// A 3-D tensor map over one padded field [nx][ny][sz] of 4-byte (float) or
// 2-byte elements, with a (bx, by, 1) box; zero fill outside the field.
cudaError_t encode_field_map(CUtensorMap* m, const void* base, int elem_bytes, const Grid& g, int bx, int by);

namespace {

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// Bounded wait for the phase with the given parity: polls until it completes,
// limit_us of wall time has passed, or kWaitPolls polls were made (whichever
// comes first); false when a bound ran out.  The first 8 polls read no clock
// (most waits end within them, and the clock read costs the march 1 %).
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, unsigned limit_us)
{
    for (int it = 0; it < 8; ++it)
        if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = global_ns(), limit = 1000ull * limit_us;
    for (int it = 0; it < kWaitPolls; ++it) {
        if (mbar_try(bar, parity)) return true;
        if (global_ns() - t0 > limit) return false;
    }
    return false;
}

__device__ __forceinline__ void tma_load3(unsigned dst, const CUtensorMap* map, int x, int y, int z,
                                          unsigned bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];\n"
        ::"r"(dst), "l"(map), "r"(x), "r"(y), "r"(z), "r"(bar) : "memory");
}


// Make the tensor map at `map` (in global memory, rewritten by a host copy since
// it was last used) visible to the TMA unit instead of a cached older copy.
__device__ __forceinline__ void acquire_tensormap(const CUtensorMap* map)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(map) : "memory");
}

}  // namespace
}  // namespace fdtd
