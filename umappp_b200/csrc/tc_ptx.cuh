// Inline PTX and register helpers shared by the tensor-core kNN kernels
// (knn_tc.cu: TF32 operands; knn_tc16.cu: FP16 operands): mbarriers with
// bounded waits, 2-D TMA loads, tcgen05 fences, commits and TMEM loads, the
// K-major 128-byte-swizzle shared-memory descriptor, and the sorted register
// candidate list.
#pragma once

#include <cuda.h>

#include <cstdint>

#include "common.cuh"

namespace umapb {
namespace tc {

// Polls of a bounded mbarrier wait: the default limit of the role waits (the
// kernels take the limit as an argument, umapb_set_device_wait_limit), and the
// fixed limit of the drain waits at exit, which wait for copies and MMAs
// already issued and must not give up early.
constexpr long long WAIT_LIMIT = 1ll << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait; returns false (and raises the abort flag) on expiry or abort.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int* err,
                                          long long limit) {
    for (long long i = 0; i < limit; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*abort_flag) return false;
        if (i > 64) __nanosleep(32);
    }
    *abort_flag = 1;
    atomicExch(err, DEV_TIMEOUT);
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major, 128-byte swizzled operand: rows of 128 B, 8-row atoms of 1024 B.
__device__ __forceinline__ uint64_t smem_desc(const void* p) {
    const uint64_t addr = smem_u32(p);
    uint64_t d = 0;
    d |= (addr >> 4) & 0x3FFFull;               // start address
    d |= uint64_t(1) << 16;                     // leading byte offset (unused for swizzled K-major)
    d |= uint64_t(1024 >> 4) << 32;             // stride byte offset: 8 rows x 128 B
    d |= uint64_t(1) << 46;                     // descriptor version (sm_100)
    d |= uint64_t(2) << 61;                     // layout: 128-byte swizzle
    return d;
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// After an abort: the MMAs this thread has issued (tcgen05.mma is
// asynchronous) must finish before their shared-memory operands go away and
// before the accumulators are freed.  A commit to 'bar' (fresh, count 1)
// arrives once all of them are done; waited for with the drain limit.
__device__ __forceinline__ void mma_drain(uint64_t* bar) {
    mma_commit(bar);
    for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(bar, 0); ++i) __nanosleep(64);
}

__device__ __forceinline__ void tmem_load32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// tcgen05.ld without the wait: r must not be read before tmem_wait_ld(r).
__device__ __forceinline__ void tmem_load32_async(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}

// Waits for every outstanding tcgen05.ld of the thread; r passes through the
// wait so that no read of it is scheduled before it.
__device__ __forceinline__ void tmem_wait_ld(uint32_t (&r)[32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                   "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                   "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
                 :
                 : "memory");
}

template <int KCAP>
__device__ __forceinline__ void insert_sorted(float (&bd)[KCAP], int (&bi)[KCAP], float cd, int ci) {
#pragma unroll
    for (int i = KCAP - 1; i > 0; --i) {
        if (cd < bd[i - 1]) {
            bd[i] = bd[i - 1];
            bi[i] = bi[i - 1];
        } else if (cd < bd[i]) {
            bd[i] = cd;
            bi[i] = ci;
        }
    }
    if (cd < bd[0]) {
        bd[0] = cd;
        bi[0] = ci;
    }
}

// Register-array element by a run-time index via a 5-level select tree
// (keeps the array in registers; dynamic indexing would spill it).
template <typename V>
__device__ __forceinline__ V select32(const V (&v)[32], int i) {
    V t16[16], t8[8], t4[4], t2[2];
#pragma unroll
    for (int j = 0; j < 16; ++j) t16[j] = (i & 16) ? v[j + 16] : v[j];
#pragma unroll
    for (int j = 0; j < 8; ++j) t8[j] = (i & 8) ? t16[j + 8] : t16[j];
#pragma unroll
    for (int j = 0; j < 4; ++j) t4[j] = (i & 4) ? t8[j + 4] : t8[j];
#pragma unroll
    for (int j = 0; j < 2; ++j) t2[j] = (i & 2) ? t4[j + 2] : t4[j];
    return (i & 1) ? t2[1] : t2[0];
}

// Largest of 32 accumulator values (as floats): the epilogue's screen for a
// whole chunk, one FMNMX per column; only chunks whose maximum passes the
// threshold are examined column by column.
__device__ __forceinline__ float chunk_max32(const uint32_t (&r)[32]) {
    float m[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) m[j] = fmaxf(__uint_as_float(r[j]), __uint_as_float(r[j + 16]));
#pragma unroll
    for (int w = 8; w >= 1; w >>= 1) {
#pragma unroll
        for (int j = 0; j < w; ++j) m[j] = fmaxf(m[j], m[j + w]);
    }
    return m[0];
}

}  // namespace tc
}  // namespace umapb
