// Shared-memory mbarrier and bulk-copy helpers (sm_90+ PTX) used by the
// warp-specialised kernels.  Every wait is bounded: after about a second of
// clock cycles it raises a block-wide abort flag, records an error code and
// returns false, so a kernel whose copies never land ends instead of hanging.
#pragma once

#include <cstdint>

namespace tsb {

constexpr long long MBAR_WAIT_LIMIT = 2000000000LL;   // clock cycles (~1 s)

// The bound a kernel applies to its pipeline waits: `requested` cycles when
// positive (tblis_stra_set_wait_limit), MBAR_WAIT_LIMIT when 0; a negative
// value -c asks every pipeline wait to treat its phase as never completing
// and run out after c cycles (tblis_stra_set_wait_injection: the wait on a
// flag that nothing sets, for failure tests).  Waits that only
// let a CTA's own copies or MMAs land before it exits always use
// MBAR_WAIT_LIMIT, so no CTA leaves with work in flight.
__host__ __device__ __forceinline__ long long wait_cycles(long long requested)
{
    return requested != 0 ? requested : MBAR_WAIT_LIMIT;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" :: "r"(addr), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t addr)
{
    asm volatile("{\n.reg .b64 st;\nmbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" :: "r"(addr) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t addr, uint32_t bytes)
{
    asm volatile("{\n.reg .b64 st;\nmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n"
                 :: "r"(addr), "r"(bytes) : "memory");
}

// Bounded wait (at most `limit` clock cycles) for the phase of the given
// parity; false on timeout or abort.
//
// try_wait may hold a thread inside the instruction until the phase completes
// or a system-dependent time passes, so a bound shorter than that time would
// only be seen to run out when a wait outlasted it.  A bound shorter than the
// default therefore polls with test_wait (which never suspends) in a loop of
// its own, so the default loop keeps its registers.
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity, volatile int* abort_flag,
                                          int* err, int code, long long limit)
{
    const long long start = clock64();
    if (limit < 0)
    {
        // injected: the phase is treated as never completing
        while (clock64() - start <= -limit)
            if (*abort_flag) return false;
        *abort_flag = 1;
        if (err) atomicExch(err, code);
        return false;
    }
    if (limit < MBAR_WAIT_LIMIT)
    {
        while (true)
        {
            uint32_t done;
            asm volatile("{\n.reg .pred p;\nmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                         "selp.u32 %0, 1, 0, p;\n}\n" : "=r"(done) : "r"(addr), "r"(parity) : "memory");
            if (done) return true;
            if (*abort_flag) return false;
            if (clock64() - start > limit)
            {
                *abort_flag = 1;
                if (err) atomicExch(err, code);
                return false;
            }
        }
    }
    while (true)
    {
        uint32_t done;
        asm volatile("{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     "selp.u32 %0, 1, 0, p;\n}\n" : "=r"(done) : "r"(addr), "r"(parity) : "memory");
        if (done) return true;
        if (*abort_flag) return false;
        if (clock64() - start > limit)
        {
            *abort_flag = 1;
            if (err) atomicExch(err, code);
            return false;
        }
    }
}

// 1-D bulk copy global -> shared (both 16-byte aligned, bytes a multiple of
// 16) completing on the mbarrier's transaction count.
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 :: "r"(dst), "l"(src), "r"(bytes), "r"(mbar) : "memory");
}

}  // namespace tsb
