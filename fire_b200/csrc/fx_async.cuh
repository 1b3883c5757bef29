// fx_async.cuh — mbarriers, bulk asynchronous copies and barrier helpers shared by the
// kernels that move data with the Tensor Memory Accelerator (fx_jacobi_zm2t.cuh) or with bulk
// copies issued by a copy warp (fx_jacobi_res.cuh, variant 4). Every wait here is bounded.
#pragma once

#include <cuda.h>

#include "fx_step_math.cuh"

FXD unsigned fx_smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

FXD void fx_mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(fx_smem_u32(bar)), "r"(count) : "memory");
}
// Arrives on bar and adds `bytes` to the transaction count its current phase waits for.
FXD void fx_mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fx_smem_u32(bar)), "r"(bytes)
                 : "memory");
}
FXD void fx_mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(fx_smem_u32(bar)) : "memory");
}
FXD bool fx_mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(fx_smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase with the given parity; false when the limit ran out.
FXD bool fx_mbar_wait(unsigned long long* bar, unsigned parity, unsigned limit) {
    for (unsigned i = 0; i < limit; ++i)
        if (fx_mbar_try_wait(bar, parity)) return true;
    return false;
}
FXD bool fx_mbar_test_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(fx_smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait by polls with back-off (each poll returns at once); false when it ran out.
FXD bool fx_mbar_wait_bounded(unsigned long long* bar, unsigned parity, unsigned limit) {
    unsigned spins = 0;
    while (!fx_mbar_test_wait(bar, parity)) {
        if (++spins > limit) return false;
        if (spins > 64) __nanosleep(32);
    }
    return true;
}
// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from global to this
// CTA's shared memory, completing on bar.
FXD void fx_bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            fx_smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(src)), "r"(bytes), "r"(fx_smem_u32(bar))
        : "memory");
}
// Orders this thread's view of global memory (stores of other CTAs, seen through acquire
// loads) before its following asynchronous-proxy copies from global memory.
FXD void fx_fence_proxy_async_global() { asm volatile("fence.proxy.async.global;\n" ::: "memory"); }
// Named barrier `id` over `count` threads that also ORs a flag over them: every thread gets
// the same answer.
FXD bool fx_bar_or(int id, int count, bool v) {
    unsigned r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}\n"
        : "=r"(r)
        : "r"((unsigned)v), "r"(id), "r"(count)
        : "memory");
    return r != 0;
}
