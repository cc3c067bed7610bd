// Shared device helpers: shared-memory staging by bulk async copy (TMA engine,
// cp.async.bulk) completed on an mbarrier, bounded waits, status reporting.
#pragma once

#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "../../include/disco_b200.h"

namespace disco {

// Message returned by disco_b200_last_error() for the calling thread (stored
// in a fixed per-thread buffer; the const char* form never allocates).
void set_last_error(const std::string& msg);
void set_last_error(const char* msg);

// A bounded wait gives up after this many nanoseconds of %globaltimer.  A stage
// copy of a few hundred KB completes in microseconds; the bound only exists so
// that no wait can spin forever.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    return ok != 0;
}

// Waits for phase `parity` of the barrier; false if the bound ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > kWaitLimitNs) return false;
    return true;
}

// One bulk copy global -> shared of `bytes` (multiple of 16, both addresses
// 16-byte aligned), completing `bytes` transactions on `bar`.  Plain (no
// cluster multicast): the source is always this GPU's own memory.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

// Largest single bulk copy issued; a stage is loaded in pieces of this size.
constexpr uint32_t kBulkPiece = 65536;

// Issues the copies of one stage (called by one thread).
__device__ __forceinline__ void stage_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    mbar_arrive_expect_tx(bar, bytes);
    for (uint32_t off = 0; off < bytes; off += kBulkPiece) {
        const uint32_t len = bytes - off < kBulkPiece ? bytes - off : kBulkPiece;
        bulk_load(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, len, bar);
    }
}

// Records the first error of a launch (first writer wins).
__device__ __forceinline__ void report(int* status, int code)
{
    atomicCAS(status, 0, code);
}

} // namespace disco
