// Thin wrappers over the sm_100a tensor-core, tensor-memory, mbarrier and
// bulk-copy instructions used by the tensor-core kernels (inline PTX; no
// library).  Every wait is bounded by the GPU's global timer so that a kernel
// whose partner never arrives returns with an error status instead of
// hanging.
#pragma once

#include <cstdint>

namespace ifgf
{
namespace tc
{

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------------------
// mbarriers (shared::cta)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
// makes initialised barriers visible to the asynchronous proxy (bulk copies,
// tensor-core commits)
__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(bar)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned bar, unsigned bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(bar),
                 "r"(bytes)
                 : "memory");
}
// Tests for the completion of the phase with the given parity; while it is
// incomplete the thread is suspended (not spinning: no issue slots or
// shared-memory bandwidth taken from the working warps) until it completes
// or about suspend_ns nanoseconds have passed.
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity, unsigned suspend_ns)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(bar), "r"(parity), "r"(suspend_ns)
                 : "memory");
    return ok != 0;
}
// Waits for the completion of the phase with the given parity; gives up and
// returns false after limit_ns nanoseconds.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity,
                                          unsigned long long limit_ns)
{
    const unsigned long long t0 = global_ns();
    for (;;)
    {
        if (mbar_try_wait(bar, parity, 1000000u))
            return true;
        if (global_ns() - t0 > limit_ns)
            return false;
    }
}

// ---------------------------------------------------------------------------
// bulk copies global -> shared, completion counted on an mbarrier
// (addresses 16-byte aligned, size a multiple of 16)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes,
                                         unsigned bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], "
                 "%2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// asks for the 128-byte lines covering [src, src + bytes) to be brought into
// L2 (one plain prefetch per line: no completion to wait for, and unlike a
// bulk prefetch no trip through the copy engine)
__device__ __forceinline__ void prefetch_l2(const void* src, unsigned bytes)
{
    const char* p = static_cast<const char*>(src);
    const char* end = p + bytes;
    for (p = reinterpret_cast<const char*>(reinterpret_cast<unsigned long long>(p) & ~127ull);
         p < end; p += 128)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(p) : "memory");
}

// generic-proxy shared-memory writes -> visible to the tensor cores
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---------------------------------------------------------------------------
// tensor memory
// ---------------------------------------------------------------------------
__device__ __forceinline__ void fence_before_sync()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// one full warp; the base address is written to shared memory
__device__ __forceinline__ void tmem_alloc(unsigned dst_smem, unsigned ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}
// 32 lanes (the warp's quarter) x 8 consecutive 32-bit columns
__device__ __forceinline__ void tmem_st8(unsigned taddr, const unsigned (&r)[8])
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(
                     taddr),
                 "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]),
                 "r"(r[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16(unsigned taddr, unsigned (&r)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr)
                 : "memory");
}
// 16 lanes (base lane in the address: 0 or 16 of the warp's quarter) x 8
// columns: thread t holds columns 2 (t % 4), 2 (t % 4) + 1 of lane t / 4 (r[0],
// r[1]) and of lane t / 4 + 8 (r[2], r[3])
__device__ __forceinline__ void tmem_st16x256(unsigned taddr, unsigned r0, unsigned r1, unsigned r2,
                                              unsigned r3)
{
    asm volatile("tcgen05.st.sync.aligned.16x256b.x1.b32 [%0], {%1,%2,%3,%4};" ::"r"(taddr), "r"(r0),
                 "r"(r1), "r"(r2), "r"(r3)
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16x256(unsigned taddr, unsigned (&r)[4])
{
    asm volatile("tcgen05.ld.sync.aligned.16x256b.x1.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr)
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st()
{
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_wait_ld()
{
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ---------------------------------------------------------------------------
// tensor-core MMA, kind::tf32, A from tensor memory, B from shared memory,
// D (FP32) in tensor memory; one thread issues
// ---------------------------------------------------------------------------
// Instruction descriptor: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9 and
// 10-12 = 2), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr unsigned idesc_tf32(int M, int N)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(N >> 3) << 17) |
           ((unsigned)(M >> 4) << 24);
}
// Shared-memory matrix descriptor of a K-major operand without swizzling:
// 8-row x 16-byte core matrices, `lbo` bytes between the two core matrices
// of one K step, `sbo` bytes between consecutive 8-row groups; bits 46-47 =
// 1 (the sm_100 descriptor version).
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr, unsigned lbo, unsigned sbo)
{
    return (unsigned long long)((addr >> 4) & 0x3fffu) |
           ((unsigned long long)((lbo >> 4) & 0x3fffu) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}
__device__ __forceinline__ void mma_tf32_ts(unsigned d_tmem, unsigned a_tmem,
                                            unsigned long long b_desc, unsigned idesc,
                                            unsigned accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
                 "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate)
                 : "memory");
}
// true in exactly one lane of the (converged) calling warp
__device__ __forceinline__ bool elect_one()
{
    unsigned pred = 0;
    asm volatile("{\n\t.reg .pred P;\n\telect.sync _|P, 0xffffffff;\n\tselp.u32 %0, 1, 0, P;\n\t}"
                 : "=r"(pred));
    return pred != 0;
}
// arrive on `bar` once every MMA this thread issued so far has completed
__device__ __forceinline__ void mma_commit(unsigned bar)
{
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
        : "memory");
}

// x rounded to TF32 (10 explicit mantissa bits, nearest, ties away from
// zero) for finite x below FLT_MAX: half a TF32 unit is added to the
// magnitude bits and the 13 low bits dropped (sign-magnitude, so both signs
// round alike).  The tensor core then reads the value exactly.
__device__ __forceinline__ float tf32_round(float x)
{
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xffffe000u);
}

} // namespace tc
} // namespace ifgf
