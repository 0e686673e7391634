// tc.cuh -- thin wrappers over the sm_100a tensor-core instructions used by
// the learned prefilter: TMEM allocation, tcgen05.mma (kind::f16, BF16
// operands, FP32 accumulators), commit to an mbarrier, TMEM loads/stores,
// the fences between them, and shared-memory matrix descriptors for the
// K-major, non-swizzled canonical layout.
//
// Canonical K-major layout of an R x K bf16 tile in shared memory (no
// swizzle): 8-row x 16-byte core matrices, element (r, k) at byte
//   (k / 8) * (R * 16) + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// i.e. core matrices 128 bytes apart along M/N (stride byte offset, SBO)
// and R*16 bytes apart along K (leading byte offset, LBO).  One MMA consumes
// K = 16 (two core-matrix columns); the next MMA's descriptor starts 2*R*16
// bytes further.
//
// Every wait on an mbarrier is bounded: after kSpinLimit polls it records
// an error code in a device flag and returns, so a lost arrival can never
// hang the GPU; the host reads the flag after the launch.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace sbwt {
namespace tc {

using u32 = uint32_t;
using u64 = uint64_t;

constexpr u32 kSpinLimit = 1u << 26;  // ~ seconds of polling at most

__device__ __forceinline__ u32 smem_addr(const void *p) {
    return (u32)__cvta_generic_to_shared(p);
}

// --------------------------------------------------------------- mbarrier

__device__ __forceinline__ void mbar_init(uint64_t *bar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, u32 parity) {
    u32 ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for phase `parity` of the barrier; on timeout sets *err = code and
// returns false (the caller skips the rest of its work).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, u32 parity, int *err, int code) {
    for (u32 i = 0; i < kSpinLimit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    atomicExch(err, code);
    return false;
}

// ------------------------------------------------------------------- TMEM

// One full warp allocates `ncols` (power of two >= 32) TMEM columns and
// writes the base address to *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(u32 *dst, u32 ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(u32 taddr, u32 ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy writes to shared memory -> visible to the tensor cores
__device__ __forceinline__ void fence_smem_to_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16 consecutive 32-bit columns of this thread's TMEM lane (warp w of the
// CTA reaches lanes 32*(w%4) .. +31).
__device__ __forceinline__ void tmem_ld16(u32 taddr, u32 (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_st8(u32 taddr, const u32 (&v)[8]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr), "r"(v[0]),
        "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
        : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Orders the use of v after a preceding tmem_wait_ld (the registers of an
// asynchronous TMEM load are only valid after the wait; this empty volatile
// asm ties them to that point so the compiler cannot use them earlier).
__device__ __forceinline__ void tmem_tie(u32 (&v)[16]) {
    asm volatile(""
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7]),
                   "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]), "+r"(v[14]),
                   "+r"(v[15])
                 :
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// ------------------------------------------------------------- MMA issue

// Shared-memory descriptor of a K-major, non-swizzled canonical tile
// (bits: start>>4 [0,14), LBO>>4 [16,30), SBO>>4 [32,46), version 1 at
// [46,48), base offset 0, layout type 0 = no swizzle).
__device__ __forceinline__ u64 smem_desc(u32 saddr, u32 lbo_bytes, u32 sbo_bytes) {
    u64 d = 0;
    d |= (u64)((saddr >> 4) & 0x3FFFu);
    d |= (u64)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (u64)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (u64)1 << 46;
    return d;
}

// Instruction descriptor: kind::f16 with BF16 A and B (both K-major), FP32
// accumulator, dense, M x N.
__host__ __device__ constexpr u32 idesc_bf16(u32 M, u32 N) {
    return (1u << 4)             // D format F32
           | (1u << 7)           // A format BF16
           | (1u << 10)          // B format BF16
           | ((N >> 3) << 17)    // N / 8
           | ((M >> 4) << 24);   // M / 16
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_ss(u32 d_tmem, u64 a_desc, u64 b_desc, u32 idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"((u32)accumulate)
        : "memory");
}

// D[tmem] (+)= A[tmem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_ts(u32 d_tmem, u32 a_tmem, u64 b_desc, u32 idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"((u32)accumulate)
        : "memory");
}

// Arrives once on the mbarrier when every MMA issued so far by this thread
// has completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
}

// Byte offset of element (r, k) of an R-row K-major canonical tile.
__host__ __device__ constexpr u32 canon_offset(u32 R, u32 r, u32 k) {
    return (k / 8) * (R * 16) + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2;
}

__device__ __forceinline__ u32 pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const u32 *>(&v);
}

}  // namespace tc
}  // namespace sbwt
