// ld_bulk.cuh -- a CTA's tile of global memory into its shared memory by the
// bulk-copy (TMA) engine: one thread posts the expected bytes on an mbarrier
// and issues the copies (16-byte aligned addresses, sizes multiples of 16
// bytes); the other threads do independent set-up meanwhile and then wait
// for the barrier's phase 0.  The wait is bounded in time (the device's
// nanosecond timer) and in rounds: past either limit it returns false and
// the caller reports kDevTimeout instead of spinning.  Every copy is the
// CTA's own, from this GPU's own memory.
#pragma once

namespace ldb {

constexpr unsigned kBulkChunk = 32768;                    // bytes per cp.async.bulk
constexpr unsigned long long kBulkWaitNs = 1000000000ull;  // 1 s; a tile takes microseconds
constexpr long long kBulkWaitRounds = 1LL << 26;          // second bound, should the timer stall

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void bulk_barrier_init(unsigned long long *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// by one thread: the barrier's one arrival, expecting `bytes` of transfers
__device__ __forceinline__ void bulk_expect(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// by one thread: post the byte count and issue the copies
__device__ __forceinline__ void bulk_copy_issue(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    const unsigned b = smem_u32(bar);
    bulk_expect(bar, bytes);
    for (unsigned o = 0; o < bytes; o += kBulkChunk) {
        const unsigned n = bytes - o < kBulkChunk ? bytes - o : kBulkChunk;
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_u32(static_cast<char *>(dst) + o)),
            "l"(static_cast<const char *>(src) + o), "r"(n), "r"(b)
            : "memory");
    }
}
// true once phase 0 of the barrier completed, false when the wait ran out
// (limit_ns of device time or kBulkWaitRounds polls, whichever comes first)
__device__ __forceinline__ bool bulk_copy_wait(unsigned long long *bar, unsigned long long limit_ns = kBulkWaitNs) {
    const unsigned b = smem_u32(bar);
    const unsigned long long t0 = global_ns();
    for (long long k = 0; k < kBulkWaitRounds; ++k) {
        unsigned done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0, %2;\n\tselp.u32 %0, 1, 0, "
            "p;\n\t}"
            : "=r"(done)
            : "r"(b), "r"(20000u)
            : "memory");
        if (done) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
    return false;
}

}  // namespace ldb
