// skm_tc.cuh -- 5th-generation tensor-core (tcgen05) building blocks for sm_100a.
//
// Used by the tensor-core versions of the phase-table GEMMs (skm_table_tc.cuh):
//   * TMEM allocation / deallocation (one warp), accumulators read back with tcgen05.ld;
//   * shared-memory matrix descriptors for the K-major 128-byte-swizzled canonical layout (the one
//     the tensor cores read at full rate): 8-row x 128-byte atoms, 16-byte chunks XOR-swizzled
//     by the row inside the atom;
//   * tcgen05.mma kind::tf32 issued by one thread, completion through tcgen05.commit to an
//     mbarrier;
//   * FP32-accurate products from TF32 tensor cores: x = hi + lo with hi = x truncated to tf32
//     and lo = x - hi, and  A*B ~= Ahi*Bhi + Ahi*Blo + Alo*Bhi  (relative error ~2^-20).
// Every wait is bounded (2 s of %globaltimer, and a poll count as a backstop): the caller gets
// `false`, records an error and leaves after one more bounded wait for its MMAs in flight.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace skm {
namespace tc {

constexpr unsigned kTcPollLimit = 1u << 28;          // polls of one bounded wait (backstop)
constexpr unsigned long long kTcWaitNs = 2000000000ull; // 2 s of %globaltimer per bounded wait

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor of a K-major operand in the 128-byte-swizzled canonical
// layout (sm100 UMMA descriptor: start [0,14), leading byte offset [16,30), stride byte offset
// [32,46), all in 16-byte units; version 1 at [46,48); layout type 2 = SWIZZLE_128B at [61,64)).
// Rows are 128 bytes (32 tf32 along K), 8-row atoms of 1024 bytes: SBO = 1024 between atoms along
// M/N; LBO is not used by this layout (set to 16 bytes).  The 16-byte chunk index of an address
// (bits 4-6) is XORed with its row within the atom (bits 7-9), so atoms must be 1024-byte aligned;
// a K step inside an atom advances the start address by 32 bytes.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)(16u >> 4) << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)2u << 61;
    return d;
}

// Instruction descriptor of kind::tf32 with F32 accumulation, both operands K-major.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N)
{
    return (1u << 4)                       // D format F32
         | (2u << 7)                       // A format TF32
         | (2u << 10)                      // B format TF32
         | ((uint32_t)(N >> 3) << 17)      // N / 8
         | ((uint32_t)(M >> 4) << 24);     // M / 16
}

// Byte offset of the 16-byte chunk holding elements k..k+3 (k a multiple of 4) of row `row` in
// a K-major 128-byte-swizzled operand of `rows` rows: K blocks of 32 elements, each
// [rows / 8][8][128 bytes], chunk index XOR row-in-atom.
__host__ __device__ __forceinline__ uint32_t sw128_offset(int row, int k, int rows)
{
    return (uint32_t)((k >> 5) * rows * 128 + (row >> 3) * 1024 + (row & 7) * 128 +
                      ((((k & 31) >> 2) ^ (row & 7)) << 4));
}

// x = hi + lo exactly, hi = x with the 13 low mantissa bits cleared (a tf32 value), so both
// parts are read by the tensor core with at most 2^-21 |x| error in lo (ALU ops only).
__device__ __forceinline__ void split_tf32(float x, float &hi, float &lo)
{
    hi = __uint_as_float(__float_as_uint(x) & 0xffffe000u);
    lo = x - hi;
}

// ---- TMEM ----------------------------------------------------------------------------------
// Executed by one full warp; the allocated column base is written to *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_addr(dst)), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- MMA and completion ---------------------------------------------------------------------
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t"
        "}\n"
        :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Same MMA with A read from tensor memory (K-major: lane = row, one 32-bit column per K element).
__device__ __forceinline__ void mma_tf32_tmem_a(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                                uint32_t accumulate)
{
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t"
        "}\n"
        :: "r"(tmem_d), "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// 16 consecutive 32-bit columns of this thread's TMEM lane (warp-collective; the warp's lane
// quarter is warp % 4), then the wait for the warp's stores.
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float *v)
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};"
        :: "r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
           "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
           "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
           "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
           "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
           "r"(__float_as_uint(v[15]))
        : "memory");
}
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const float *v)
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};"
        :: "r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
           "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
           "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Expected transaction bytes on an mbarrier (arrives once) and a bulk global -> shared copy that
// completes them (no multicast).  size: multiple of 16, both addresses 16-byte aligned.
__device__ __forceinline__ void mbar_expect_tx(uint64_t *mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_addr(mbar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *mbar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(mbar)) : "memory");
}

__device__ __forceinline__ void commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_addr(mbar)) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(mbar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbarrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Waits for the completion of the mbarrier phase with the given parity; false when the bound
// runs out first or when *abort becomes nonzero (another role of the CTA gave up).  try_wait
// carries a suspend-time hint: a waiting thread sleeps in hardware until the phase completes (or
// the hint elapses) instead of spinning, so waiting roles leave the issue slots to working ones.
constexpr uint32_t kTcSuspendNs = 20000;
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, const volatile int *abort = nullptr,
                                          unsigned long long limit_ns = kTcWaitNs)
{
    const uint32_t a = smem_addr(mbar);
    unsigned long long t0 = 0;
    for (unsigned i = 0; i < kTcPollLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done) : "r"(a), "r"(parity), "r"(kTcSuspendNs) : "memory");
        if (done) return true;
        if (abort && *abort) return false;
        const unsigned long long t = globaltimer();
        if (i == 0) t0 = t;
        else if (t - t0 > limit_ns) return false;
    }
    return false;
}

// Arrival of the executing thread (release at CTA scope).
__device__ __forceinline__ void mbar_arrive(uint64_t *mbar)
{
    unsigned long long state;
    asm volatile("mbarrier.arrive.shared::cta.b64 %0, [%1];" : "=l"(state) : "r"(smem_addr(mbar)) : "memory");
    (void)state;
}

// Named barrier `id` over `count` threads that also ORs a predicate across them.
__device__ __forceinline__ bool bar_or(int id, int count, bool pred)
{
    uint32_t r;
    asm volatile(
        "{\n\t"
        ".reg .pred ip, op;\n\t"
        "setp.ne.u32 ip, %1, 0;\n\t"
        "bar.red.or.pred op, %2, %3, ip;\n\t"
        "selp.u32 %0, 1, 0, op;\n\t"
        "}\n"
        : "=r"(r) : "r"((uint32_t)pred), "r"(id), "r"(count) : "memory");
    return r != 0;
}

__device__ __forceinline__ void bar_sync(int id, int count)
{
    asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(count) : "memory");
}

// ---- bulk tensor stores (shared -> global, bulk groups of the issuing thread) ------------------
// Generic-proxy writes to shared memory become visible to the bulk copies after this fence (each
// writing thread, before the barrier that precedes the issue).
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// at most N of the thread's bulk groups still read their shared-memory source
template <int N>
__device__ __forceinline__ void bulk_wait_read()
{
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// ---- TMEM -> registers ----------------------------------------------------------------------
// 32 lanes x 32 bits, 16 consecutive columns: thread t of the warp gets row (lane base + t).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 consecutive 32-bit columns of this thread's TMEM lane, one load and one wait.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v)
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace skm
