/* tma_bulk.cuh — one-dimensional TMA bulk copies global -> shared with mbarrier
 * completion (cp.async.bulk, no multicast), and a wait with a time limit (internal). */
#ifndef GSLAM_TMA_BULK_CUH
#define GSLAM_TMA_BULK_CUH

#include <stdint.h>

__device__ __forceinline__ void tma_mbar_init(uint64_t *bar, unsigned count) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void tma_mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool tma_mbar_try_wait(uint64_t *bar, unsigned parity) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0;
}

/* Both addresses 16-byte aligned and bytes a multiple of 16 (the layouts guarantee it:
 * every staged region starts and ends on a 32-slot or 32-row boundary). */
__device__ __forceinline__ void tma_bulk_g2s(void *dst_smem, const void *src, unsigned bytes,
                                             uint64_t *bar) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
        "l"(src), "r"(bytes), "r"(b)
        : "memory");
}

/* Waits for the phase with the given parity; false if `limit` clock cycles pass first. */
__device__ __forceinline__ bool tma_wait(uint64_t *bar, unsigned parity, long long limit) {
    const long long t0 = clock64();
    while (!tma_mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > limit) return false;
    }
    return true;
}

#endif
