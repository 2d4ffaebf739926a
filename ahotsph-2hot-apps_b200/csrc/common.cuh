// common.cuh -- shared device helpers of libgravcuda: status reporting, the
// TMA bulk-copy / mbarrier primitives (sm_90+ PTX, used here for sm_100a),
// and the FP32 arithmetic building blocks of the interaction kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// ------------------------------------------------------------ host status
namespace gc {

// 0 = print and abort like the reference's Error(); 1 = record and return.
extern int g_error_mode;
int set_status(int code, const char *fmt, ...);
int cuda_status(cudaError_t err, const char *what);

}  // namespace gc

#define GC_CHECK(call)                                              \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess)                                      \
            return gc::cuda_status(_e, #call);                      \
    } while (0)

// Device error word bits (set by kernels, read by the host after a step).
enum : unsigned {
    GC_DEV_WAIT_TIMEOUT = 1u,   // an mbarrier wait gave up
    GC_DEV_BAD_INDEX = 2u,      // a list entry pointed outside its table
    GC_DEV_BAD_COUNT = 4u,      // a body-run checksum did not match
    GC_DEV_BAD_RUNS = 8u,       // a run-packed list did not unpack to its group's length
};

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

// Make mbarrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Arrive once and announce `bytes` of incoming transactions on this phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Non-multicast bulk copy global -> shared, completing `bytes` on `bar`.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void tma_bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                             uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// try_wait with a suspend-time hint: a warp whose data has not landed is
// suspended (up to hint_ns) until the phase completes instead of spinning
// through issue slots the other warps need.
// TMA row gather (sm_100a): four rows of a 2-D tensor map, each one box
// (one row high, the full row wide), selected by row index, land back to
// back at dst (128-byte aligned).  No multicast.
__device__ __forceinline__ void tma_gather4(void *dst, const void *tmap, int r0, int r1, int r2,
                                            int r3, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(dst)),
        "l"(tmap), "r"(0), "r"(r0), "r"(r1), "r"(r2), "r"(r3), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity,
                                              uint32_t hint_ns = 20000) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}

// Bounded wait: gives up after `limit` polls (each suspends for at most the
// hint), sets GC_DEV_WAIT_TIMEOUT and returns false, so a lost transaction
// ends the kernel within about a second instead of hanging the GPU.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  unsigned *err, uint32_t limit = 1u << 16) {
    for (uint32_t i = 0; i < limit; i++)
        if (mbar_try_wait(bar, parity))
            return true;
    atomicOr(err, GC_DEV_WAIT_TIMEOUT);
    return false;
}

// Per-thread asynchronous 16-byte copy global -> shared (cp.async, cached in
// L2 only), grouped by commit_group and completed by wait_group.  Not the
// bulk (TMA) path: each thread copies the bytes it will read itself.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)), "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
// Wait until at most N of this thread's committed groups are still in flight.
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Single MUFU reciprocal square root (approximate, flush-to-zero); the
// reference uses an 11-bit rsqrtps refined by one Newton step
// (nln/do_grav_avx8.c:2188-2201), which this matches in accuracy.
__device__ __forceinline__ float rsqrt_fast(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Knuth two-sum: s + e == a + b exactly.
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
    s = a + b;
    float bp = s - a;
    e = (a - (s - bp)) + (b - bp);
}

// Fold a tile partial sum t into the compensated accumulator (hi, lo).
__device__ __forceinline__ void comp_add(float &hi, float &lo, float t) {
    float s, e;
    two_sum(hi, t, s, e);
    hi = s;
    lo += e;
}
