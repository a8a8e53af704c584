// Tensor-core candidate search for the exact kNN of float data (sm_100a).
//
// Squared distances are ||q||^2 + ||r||^2 - 2 q.r with the dot products from
// 5th-generation tensor cores (tcgen05.mma, kind::tf32) in split precision:
// every coordinate is split as a = hi + lo with hi = tf32(a) and
// lo = tf32(a - hi), and q.r = hi.hi + hi.lo + lo.hi (the lo.lo term is below
// 2^-22 relative), i.e. "3xTF32", accumulated in FP32 in tensor memory.
//
// One CTA owns 128 queries (the MMA's M) and streams all reference points in
// tiles of 128 (N).  Warp roles:
//   warp 0     TMA producer: the query tile (hi and lo, all K chunks) once,
//              then reference tiles into a 2-stage shared-memory ring;
//   warp 1     MMA issuer (one lane): 3 x 4 x Kc tcgen05.mma per tile into one
//              of two TMEM accumulators (128 lanes x 128 FP32 columns each),
//              tcgen05.commit to the ring's "empty" and the accumulator's
//              "full" mbarriers; it also owns the TMEM allocation;
//   warps 2-9  epilogue: tcgen05.ld of the accumulator rows (one query per
//              thread, each row split between two warps by column halves), a
//              screen of each 32-column chunk by its maximum against the
//              current k-th distance, and sorted register lists of the KCAP best
//              (distance, index) candidates, merged per row at the end.
// Operands are K-major with the 128-byte swizzle (TMA box 128 rows x 32 FP32,
// UMMA shared-memory descriptors with SBO = 1024 B), no cluster multicast.
// Every mbarrier wait is bounded: on expiry the kernel records an error,
// raises a CTA-wide abort flag so the other roles stop waiting, frees TMEM and
// returns.  The candidates are rescored in FP64 by knn.cu.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

#include "stages.cuh"
#include "tc_ptx.cuh"

namespace umapb {

namespace {

using namespace tc;

constexpr int TC_M = 128;         // queries per CTA
constexpr int TC_N = 128;         // references per tile
constexpr int TC_KCHUNK = 32;     // FP32 elements per 128-byte swizzle row
constexpr int TC_STAGES = 2;
constexpr int TC_EPI_WARPS = 8;
constexpr int TC_THREADS = 64 + 32 * TC_EPI_WARPS;   // producer, MMA, 8 epilogue warps
constexpr uint32_t TC_TMEM_COLS = 256;   // two 128-column accumulators

// Instruction descriptor: D = F32, A = B = TF32, both K-major, M = 128, N = TC_N.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(TC_N >> 3) << 17) | (uint32_t(TC_M >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

// ------------------------------------------------------------ prep kernel --

// Operands of the distance GEMM, [n_pad, k_pad] each (zero padded), as TF32
// pairs hi = tf32(v), lo = tf32(v - hi):
//   queries    A = [x, 1]              (column dim holds 1)
//   references B = [x, -|x|^2 / 2]     (column dim holds minus half the norm)
// so that the accumulator is q.r - |r|^2 / 2 and d2 = |q|^2 - 2 acc, with no
// norm look-up in the epilogue.  Padding references carry -1e30 in the norm
// column, so their distance is huge and never qualifies.  norms[i] = |x_i|^2
// (FP64, rounded to FP32; +inf for padding rows).
__device__ __forceinline__ void split_tf32(float a, float& hi, float& lo) {
    uint32_t h, l;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(a));
    const float r = a - __uint_as_float(h);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(r));
    hi = __uint_as_float(h);
    lo = __uint_as_float(l);
}

// pad_src (batched runs) maps operand row i to its data row, or -1 for a
// padding row; without it, rows below n are data rows.
__global__ void prepare_operands_kernel(const float* __restrict__ data, int32_t n, int32_t dim, int32_t n_pad,
                                        int32_t k_pad, float* __restrict__ a_hi, float* __restrict__ a_lo,
                                        float* __restrict__ b_hi, float* __restrict__ b_lo,
                                        float* __restrict__ norms, const int32_t* __restrict__ pad_src) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n_pad; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t src = pad_src ? pad_src[i] : (i < n ? i : -1);
        const bool real = src >= 0;
        double s = 0;
        if (real) {
            for (int d = 0; d < dim; ++d) {
                const double v = data[src * dim + d];
                s += v * v;
            }
        }
        norms[i] = real ? static_cast<float>(s) : CUDART_INF_F;
        const int64_t row = i * k_pad;
        for (int d = 0; d < k_pad; ++d) {
            float v = 0.0f;
            if (real && d < dim) v = data[src * dim + d];
            float h, l;
            split_tf32(v, h, l);
            a_hi[row + d] = h;
            a_lo[row + d] = l;
            if (d == dim) {
                // the norm column: 1 for queries, -|r|^2 / 2 for references
                a_hi[row + d] = real ? 1.0f : 0.0f;
                a_lo[row + d] = 0.0f;
                if (real) {
                    split_tf32(static_cast<float>(-0.5 * s), h, l);
                } else {
                    h = -1e30f;
                    l = 0.0f;
                }
            }
            b_hi[row + d] = h;
            b_lo[row + d] = l;
        }
    }
}

// ----------------------------------------------------------- main kernel --

template <int KC>
struct TcSmem {
    // operand tiles first (1024-byte aligned): A hi/lo then the B ring
    float a_hi[KC][TC_M * TC_KCHUNK];
    float a_lo[KC][TC_M * TC_KCHUNK];
    float b_hi[TC_STAGES][KC][TC_N * TC_KCHUNK];
    float b_lo[TC_STAGES][KC][TC_N * TC_KCHUNK];
    uint64_t full[TC_STAGES];
    uint64_t empty[TC_STAGES];
    uint64_t tmem_full[2];
    uint64_t tmem_empty[2];
    uint64_t a_full;
    uint64_t mma_done;   // drain after an abort (mma_drain)
    uint32_t tmem_base;
    int abort_flag;
};

template <int KC, int KCAP>
__global__ void __launch_bounds__(TC_THREADS, 1) knn_tc_kernel(const __grid_constant__ CUtensorMap map_ahi,
                                                               const __grid_constant__ CUtensorMap map_alo,
                                                               const __grid_constant__ CUtensorMap map_bhi,
                                                               const __grid_constant__ CUtensorMap map_blo,
                                                               const float* __restrict__ norms, int32_t n,
                                                               int32_t n_tiles_all, int32_t ksteps,
                                                               int32_t* __restrict__ cand_idx,
                                                               float* __restrict__ cand_d2, int* __restrict__ err,
                                                               const int4* __restrict__ tasks,
                                                               const int32_t* __restrict__ shifts,
                                                               long long wait_limit) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // the dynamic window is only guaranteed 16-byte aligned: round up to 1024
    TcSmem<KC>& sm = *reinterpret_cast<TcSmem<KC>*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // This CTA's queries are operand rows [q_base, q_base + 128), valid below
    // q_limit; its references are the n_tiles tiles from ref_tile0.  Batched
    // runs give each CTA a task (one instance's query tile against that
    // instance's reference tiles) and the shift from operand rows to data rows.
    int q_base, ref_tile0, n_tiles, q_limit, shift;
    if (tasks) {
        const int4 t = tasks[blockIdx.x];
        q_base = t.x;
        ref_tile0 = t.y;
        n_tiles = t.z;
        q_limit = t.w;
        shift = shifts[blockIdx.x];
    } else {
        q_base = blockIdx.x * TC_M;
        ref_tile0 = 0;
        n_tiles = n_tiles_all;
        q_limit = n;
        shift = 0;
    }
    volatile int* abort_flag = &sm.abort_flag;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&sm.tmem_full[b], 1);
            mbar_init(&sm.tmem_empty[b], 32 * TC_EPI_WARPS);
        }
        mbar_init(&sm.a_full, 1);
        mbar_init(&sm.mma_done, 1);
        sm.abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        // TMEM: two 128-column FP32 accumulators
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem_base)),
                     "r"(TC_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = sm.tmem_base;

    constexpr uint32_t A_BYTES = 2u * KC * TC_M * TC_KCHUNK * 4u;
    constexpr uint32_t B_BYTES = 2u * KC * TC_N * TC_KCHUNK * 4u;
    int issued = 0;   // producer: loads issued (for the drain at exit)

    if (warp == 0) {
        if (lane == 0) {
            mbar_arrive_expect_tx(&sm.a_full, A_BYTES);
            for (int c = 0; c < KC; ++c) {
                tma_load_2d(sm.a_hi[c], &map_ahi, &sm.a_full, c * TC_KCHUNK, q_base);
                tma_load_2d(sm.a_lo[c], &map_alo, &sm.a_full, c * TC_KCHUNK, q_base);
            }
            for (int it = 0; it < n_tiles; ++it) {
                const int s = it % TC_STAGES;
                const uint32_t round = it / TC_STAGES;
                if (!mbar_wait(&sm.empty[s], (round & 1) ^ 1, abort_flag, err, wait_limit)) break;
                mbar_arrive_expect_tx(&sm.full[s], B_BYTES);
                for (int c = 0; c < KC; ++c) {
                    tma_load_2d(sm.b_hi[s][c], &map_bhi, &sm.full[s], c * TC_KCHUNK, (ref_tile0 + it) * TC_N);
                    tma_load_2d(sm.b_lo[s][c], &map_blo, &sm.full[s], c * TC_KCHUNK, (ref_tile0 + it) * TC_N);
                }
                ++issued;
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            if (mbar_wait(&sm.a_full, 0, abort_flag, err, wait_limit)) {
                for (int it = 0; it < n_tiles; ++it) {
                    const int s = it % TC_STAGES;
                    const int buf = it & 1;
                    if (!mbar_wait(&sm.full[s], (it / TC_STAGES) & 1, abort_flag, err, wait_limit)) break;
                    if (!mbar_wait(&sm.tmem_empty[buf], ((it >> 1) & 1) ^ 1, abort_flag, err, wait_limit)) break;
                    tc_fence_after();
                    const uint32_t d = tmem_base + buf * TC_N;
                    uint32_t acc = 0;
#pragma unroll
                    for (int c = 0; c < KC; ++c) {
#pragma unroll
                        for (int kk = 0; kk < TC_KCHUNK / 8; ++kk) {
                            // K-steps past the last non-zero column (data + norm) contribute nothing
                            if (c * (TC_KCHUNK / 8) + kk >= ksteps) break;
                            const int off = kk * 8;   // 8 TF32 = 32 bytes along K inside the swizzle row
                            const uint64_t ah = smem_desc(sm.a_hi[c] + off), al = smem_desc(sm.a_lo[c] + off);
                            const uint64_t bh = smem_desc(sm.b_hi[s][c] + off), bl = smem_desc(sm.b_lo[s][c] + off);
                            mma_tf32(d, al, bh, acc);
                            acc = 1;
                            mma_tf32(d, ah, bl, 1);
                            mma_tf32(d, ah, bh, 1);
                        }
                    }
                    mma_commit(&sm.empty[s]);
                    mma_commit(&sm.tmem_full[buf]);
                }
            }
        }
    } else {
        // Epilogue, 8 warps: warp w reads TMEM lanes 32 * (w % 4) .. + 31 (one
        // query row per thread) and half (w - 2) / 4 of each tile's 128 columns;
        // the two halves of a row keep separate candidate lists, merged at the end.
        const int quarter = warp & 3;
        const int half = (warp - 2) >> 2;
        const int row = quarter * 32 + lane;
        const int q = q_base + row;
        const float qn = (q < q_limit) ? norms[q] : 0.0f;
        float bd[KCAP];
        int bi[KCAP];
#pragma unroll
        for (int i = 0; i < KCAP; ++i) {
            bd[i] = CUDART_INF_F;
            bi[i] = -1;
        }
        float thr = CUDART_INF_F;
        // d2 = qn - 2 acc < thr  <=>  acc > (qn - thr) / 2; rounded down, so the
        // screen admits every column the exact test below would
        float athr = -CUDART_INF_F;
        for (int it = 0; it < n_tiles; ++it) {
            const int buf = it & 1;
            if (!mbar_wait(&sm.tmem_full[buf], (it >> 1) & 1, abort_flag, err, wait_limit)) break;
            tc_fence_after();
            const uint32_t taddr = tmem_base + (uint32_t(quarter * 32) << 16) + buf * TC_N + half * (TC_N / 2);
            const int col0 = (ref_tile0 + it) * TC_N + half * (TC_N / 2);   // operand row of column 0
            const bool diag = (col0 <= q && q < col0 + TC_N / 2);
            // reference columns at or past q_limit are padding (their distances
            // are finite, so they are masked out rather than left to lose)
            const int valid = q_limit - col0;
#pragma unroll 1
            for (int ch = 0; ch < TC_N / 64; ++ch) {
                uint32_t r[32];
                tmem_load32(taddr + ch * 32, r);
                if (chunk_max32(r) > athr) {   // rare after the first tiles
                    uint32_t mask = 0;
#pragma unroll
                    for (int i = 0; i < 32; ++i) mask |= (__uint_as_float(r[i]) > athr ? 1u : 0u) << i;
                    if (diag && (q - col0) / 32 == ch) mask &= ~(1u << ((q - col0) & 31));   // self
                    const int vc = valid - ch * 32;
                    if (vc < 32) mask &= (vc <= 0) ? 0u : ((1u << vc) - 1u);
                    while (mask) {   // rare: candidates better than the current k-th
                        const int i = __ffs(mask) - 1;
                        mask &= mask - 1;
                        const float v = fmaf(-2.0f, __uint_as_float(select32(r, i)), qn);
                        if (v < thr) {
                            insert_sorted<KCAP>(bd, bi, v, col0 + ch * 32 + i + shift);
                            thr = bd[KCAP - 1];
                            athr = __fmul_rd(0.5f, __fsub_rd(qn, thr));
                        }
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(&sm.tmem_empty[buf]);
        }
        // Merge the halves through shared memory (the query tile's space: every
        // MMA has completed once the last accumulator was seen full).
        float* merge_d = &sm.a_hi[0][0];
        int* merge_i = reinterpret_cast<int*>(&sm.a_lo[0][0]);
        const bool ok = (*abort_flag == 0);
        if (half == 1 && ok) {
#pragma unroll
            for (int i = 0; i < KCAP; ++i) {
                merge_d[i * TC_M + row] = bd[i];
                merge_i[i * TC_M + row] = bi[i];
            }
        }
        asm volatile("bar.sync 1, %0;" ::"n"(TC_EPI_WARPS * 32) : "memory");
        if (half == 0 && ok && q < q_limit) {
            for (int i = 0; i < KCAP; ++i) {
                const float v = merge_d[i * TC_M + row];
                if (!(v < thr)) break;   // the partner's list is sorted
                insert_sorted<KCAP>(bd, bi, v, merge_i[i * TC_M + row]);
                thr = bd[KCAP - 1];
            }
            const size_t out_row = static_cast<size_t>(q + shift);   // data row of this query
#pragma unroll
            for (int i = 0; i < KCAP; ++i) {
                cand_idx[out_row * KCAP + i] = bi[i];
                cand_d2[out_row * KCAP + i] = bd[i];
            }
        }
    }

    // drain: loads in flight must land before the CTA's shared memory goes away
    if (warp == 0 && lane == 0 && *abort_flag) {
        for (int it = (issued > TC_STAGES ? issued - TC_STAGES : 0); it < issued; ++it) {
            const int s = it % TC_STAGES;
            for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&sm.full[s], (it / TC_STAGES) & 1); ++i) __nanosleep(64);
        }
        for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&sm.a_full, 0); ++i) __nanosleep(64);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) {
        // after an abort, MMAs issued by lane 0 may still read shared memory and
        // write the accumulators: wait for them before freeing TMEM
        if (lane == 0 && *abort_flag) mma_drain(&sm.mma_done);
        __syncwarp();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TC_TMEM_COLS));
    }
}

// --------------------------------------------------------------- host side --

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess) {
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        }
    });
    require(fn != nullptr, "cuTensorMapEncodeTiled is unavailable", UMAPB_ERR_CUDA);
    return fn;
}

// 2-D FP32 tensor [rows, k_pad] (k_pad contiguous), box 128 rows x 32 columns, 128-byte swizzle.
CUtensorMap make_map(const float* base, int64_t rows, int k_pad) {
    CUtensorMap m;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(k_pad), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(k_pad) * sizeof(float)};
    const cuuint32_t box[2] = {TC_KCHUNK, 128};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = get_encode()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box,
                                    estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    require(r == CUDA_SUCCESS, "cuTensorMapEncodeTiled failed", UMAPB_ERR_CUDA);
    return m;
}

struct Maps {
    CUtensorMap ahi, alo, bhi, blo;
    int ksteps;   // MMA K-steps of 8 columns that hold data or the norm column
};

// One launch: 'ctas' CTAs; with tasks, CTA b runs tasks[b] (see the kernel).
template <int KC, int KCAP>
void launch_tc(const Maps& m, const float* norms, int32_t n, int32_t n_pad, int32_t ctas, const int4* tasks,
               const int32_t* shifts, int32_t* cand_idx, float* cand_d2, int* err, cudaStream_t s) {
    const size_t smem = sizeof(TcSmem<KC>) + 1024;
    static bool configured = false;
    if (!configured) {
        UMAPB_CUDA(cudaFuncSetAttribute(knn_tc_kernel<KC, KCAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(smem)));
        configured = true;
    }
    const int n_tiles = n_pad / TC_N;
    knn_tc_kernel<KC, KCAP><<<ctas, TC_THREADS, smem, s>>>(m.ahi, m.alo, m.bhi, m.blo, norms, n, n_tiles, m.ksteps,
                                                           cand_idx, cand_d2, err, tasks, shifts,
                                                           device_wait_limit());
    UMAPB_LAUNCH_CHECK();
}

template <int KC>
void launch_kcap(int kcap, const Maps& m, const float* norms, int32_t n, int32_t n_pad, int32_t ctas,
                 const int4* tasks, const int32_t* shifts, int32_t* cand_idx, float* cand_d2, int* err,
                 cudaStream_t s) {
    if (kcap == 16) launch_tc<KC, 16>(m, norms, n, n_pad, ctas, tasks, shifts, cand_idx, cand_d2, err, s);
    else if (kcap == 24) launch_tc<KC, 24>(m, norms, n, n_pad, ctas, tasks, shifts, cand_idx, cand_d2, err, s);
    else launch_tc<KC, 32>(m, norms, n, n_pad, ctas, tasks, shifts, cand_idx, cand_d2, err, s);
}

// Shared body: operands over n_pad rows (pad_src maps rows to data rows in
// batched runs), then one launch over 'ctas' CTAs.
void run_candidates(const float* data, int32_t n, int32_t dim, int kcap, int32_t n_pad, const int32_t* pad_src,
                    int32_t ctas, const int4* tasks, const int32_t* shifts, int32_t* cand_idx, float* cand_d2,
                    float* norms_pad, int* d_err, cudaStream_t s) {
    const int kc = (dim + 1 + TC_KCHUNK - 1) / TC_KCHUNK;
    const int k_pad = kc * TC_KCHUNK;
    const size_t elems = static_cast<size_t>(n_pad) * k_pad;
    DevArray<float> ahi(elems, s), alo(elems, s), bhi(elems, s), blo(elems, s);
    prepare_operands_kernel<<<grid_for(n_pad, 256), 256, 0, s>>>(data, n, dim, n_pad, k_pad, ahi.get(), alo.get(),
                                                                  bhi.get(), blo.get(), norms_pad, pad_src);
    UMAPB_LAUNCH_CHECK();
    Maps m;
    m.ahi = make_map(ahi.get(), n_pad, k_pad);
    m.alo = make_map(alo.get(), n_pad, k_pad);
    m.bhi = make_map(bhi.get(), n_pad, k_pad);
    m.blo = make_map(blo.get(), n_pad, k_pad);
    m.ksteps = (dim + 1 + 7) / 8;
    if (kc == 1) launch_kcap<1>(kcap, m, norms_pad, n, n_pad, ctas, tasks, shifts, cand_idx, cand_d2, d_err, s);
    else launch_kcap<2>(kcap, m, norms_pad, n, n_pad, ctas, tasks, shifts, cand_idx, cand_d2, d_err, s);
    // the operand arrays are released stream-ordered, after the kernel
}

// Operand type of the candidate search: FP16 pairs (knn_tc16.cu, default) or
// TF32 pairs (this file); UMAPB_KNN_TC_KIND=tf32 selects the latter.
bool use_f16_operands() {
    const char* e = std::getenv("UMAPB_KNN_TC_KIND");   // read per search: tests switch it
    return !(e && std::strcmp(e, "tf32") == 0);
}

// Tile pruning of the FP16 search (knn_tree.cu); UMAPB_KNN_PRUNE=0 scans
// every tile (operands in data order).
bool prune_enabled() {
    const char* e = std::getenv("UMAPB_KNN_PRUNE");   // read per search: tests switch it
    return !(e && std::strcmp(e, "0") == 0);
}

// Launch-shape tuner of the FP16 search: per (K chunks, size class = log2 of
// the operand tiles) the launch shape whose kernel ran fastest, timed once on
// the first unsharded search of the class in the process; UMAPB_KNN_SHAPE
// (24 or 12) or UMAPB_KNN_QT (2 or 1) forces one where it exists.
struct ShapeTuner {
    std::mutex mu;
    std::map<std::pair<int, int>, int> best;
};
ShapeTuner& shape_tuner() {
    static ShapeTuner t;
    return t;
}

// FP16 search over the (pruned) tile lists of the instances 'inst'.
void run_f16_pruned(const float* data, const std::vector<int32_t>& inst, int32_t dim, int kcap, float scale,
                    int32_t* cand_idx, float* cand_d2, float* norms_by_row, int* d_err, cudaStream_t s,
                    KnnShard shard = KnnShard(), DevArray<int32_t>* shard_rows = nullptr,
                    int32_t* shard_count = nullptr, DevArray<int32_t>* tree_rows = nullptr) {
    const bool prune = prune_enabled();
    KnnTiles tiles;
    knn_tree_order(data, dim, inst, prune, tiles, s);
    if (tree_rows) knn_tree_rows(tiles, inst.back(), *tree_rows, s);
    const std::vector<int> shapes = knn_tc16_shapes(dim);
    int shape = shapes.front();
    bool tune = false;
    std::pair<int, int> key((dim + 1 + 63) / 64, 0);
    while ((int64_t(1) << key.second) < tiles.n_pad / 128) ++key.second;
    int want = 0;
    if (const char* e = std::getenv("UMAPB_KNN_SHAPE")) want = std::atoi(e);
    else if (const char* e = std::getenv("UMAPB_KNN_QT")) want = std::atoi(e) == 1 ? 12 : std::atoi(e) == 2 ? 24 : 0;
    if (want) {
        for (int c : shapes)
            if (c == want) shape = c;
    } else if (shapes.size() > 1 && shard.count == 1) {
        // (a sharded search keeps the default shape: the shards' task lists,
        // and with them the rows each rank computes, must agree across ranks
        // whatever each rank's tuner has seen)
        ShapeTuner& t = shape_tuner();
        std::lock_guard<std::mutex> lock(t.mu);
        auto it = t.best.find(key);
        if (it != t.best.end()) shape = it->second;
        else tune = true;
    }
    if (tune) {
        // every shape computes the same candidate lists: time each, keep the
        // fastest for the class; the last run's lists are the result
        float best_ms = 0.0f;
        int best_shape = shape;
        for (size_t i = 0; i < shapes.size(); ++i) {
            KnnTasks tasks;
            knn_tile_tasks(data, dim, tiles, inst, shapes[i] / 10, kcap, prune, tasks, s, shard);
            knn_tc16_run_tasks(data, dim, kcap, scale, tiles, tasks, cand_idx, cand_d2, norms_by_row, d_err, s,
                               &last_knn_kernel_ms(), shapes[i]);
            last_knn_tiles_scanned() = tasks.total_tiles;
            UMAPB_SYNC(s);
            if (i == 0 || last_knn_kernel_ms() < best_ms) {
                best_ms = last_knn_kernel_ms();
                best_shape = shapes[i];
            }
        }
        ShapeTuner& t = shape_tuner();
        std::lock_guard<std::mutex> lock(t.mu);
        t.best[key] = best_shape;
        return;
    }
    KnnTasks tasks;
    knn_tile_tasks(data, dim, tiles, inst, shape / 10, kcap, prune, tasks, s, shard);
    if (shard_rows) knn_task_rows(tiles, tasks, inst.back(), *shard_rows, *shard_count, s);
    knn_tc16_run_tasks(data, dim, kcap, scale, tiles, tasks, cand_idx, cand_d2, norms_by_row, d_err, s,
                       &last_knn_kernel_ms(), shape);
    last_knn_tiles_scanned() = tasks.total_tiles;
    UMAPB_SYNC(s);   // the tile and task buffers are released below
}

bool tf32_supported(int32_t dim, int kcap) {
    // the norm rides in one extra K column: dim + 1 columns in two 32-wide chunks
    return dim >= 1 && dim + 1 <= 2 * TC_KCHUNK && (kcap == 16 || kcap == 24 || kcap == 32);
}

}  // namespace

bool knn_tc_supported(int32_t dim, int kcap) {
    return tf32_supported(dim, kcap) || (use_f16_operands() && knn_tc16_supported(dim, kcap));
}

// Scale for the FP16 search, or 0 when the TF32 search is to be used.
static float f16_scale_or_zero(const float* data, size_t count, int32_t dim, int kcap, cudaStream_t s) {
    if (!use_f16_operands() || !knn_tc16_supported(dim, kcap)) return 0.0f;
    const float scale = knn_tc16_scale(data, count, s);
    require(scale > 0.0f || tf32_supported(dim, kcap),
            "tensor-core kNN: the data have no finite maximum in [2^-60, 2^60] for the FP16 search");
    return scale;
}

// Candidate lists (KCAP per query, FP32 squared distances, ascending) from the
// tensor-core search; norms_out receives |x|^2 for the certainty bound of the
// FP64 rescoring.
bool knn_tc_candidates(const float* data, int32_t n, int32_t dim, int kcap, int32_t* cand_idx, float* cand_d2,
                       float* norms_out, int* d_err, cudaStream_t s, KnnShard shard, DevArray<int32_t>* shard_rows,
                       int32_t* shard_count, DevArray<int32_t>* tree_rows) {
    require(knn_tc_supported(dim, kcap), "tensor-core kNN: unsupported dimension or candidate count");
    const int32_t n_pad = ((n + TC_M - 1) / TC_M) * TC_M;
    const float scale = f16_scale_or_zero(data, static_cast<size_t>(n) * dim, dim, kcap, s);
    if (scale > 0.0f) {
        run_f16_pruned(data, {0, n}, dim, kcap, scale, cand_idx, cand_d2, norms_out, d_err, s, shard, shard_rows,
                       shard_count, tree_rows);
        return true;
    }
    if (shard.count > 1) return false;   // the TF32 search covers every query: the caller shards by rows instead
    last_knn_tiles_scanned() = static_cast<int64_t>(n_pad / TC_M) * (n_pad / TC_N);
    run_candidates(data, n, dim, kcap, n_pad, nullptr, n_pad / TC_M, nullptr, nullptr, cand_idx, cand_d2, norms_out,
                   d_err, s);
    return true;
}

// Batched: instance i is data rows [inst[i], inst[i + 1]); every query's
// candidates come from its own instance only.  Each instance is placed at a
// 128-row boundary of the operands, so a CTA's query tiles and reference
// tiles all belong to one instance (a CTA's last query tile may run past its
// instance; those rows are masked).  Candidate indices are data rows.
void knn_tc_candidates_batched(const float* data, const std::vector<int32_t>& inst, int32_t dim, int kcap,
                               int32_t* cand_idx, float* cand_d2, int* d_err, cudaStream_t s) {
    require(knn_tc_supported(dim, kcap), "tensor-core kNN: unsupported dimension or candidate count");
    const int ninst = static_cast<int>(inst.size()) - 1;
    const float scale = f16_scale_or_zero(data, static_cast<size_t>(inst[ninst]) * dim, dim, kcap, s);
    if (scale > 0.0f) {
        DevArray<float> norms(inst[ninst], s);
        run_f16_pruned(data, inst, dim, kcap, scale, cand_idx, cand_d2, norms.get(), d_err, s);
        return;
    }
    const int qt = 1;
    std::vector<int32_t> pad_start(ninst + 1, 0);
    for (int i = 0; i < ninst; ++i) {
        const int32_t len = inst[i + 1] - inst[i];
        pad_start[i + 1] = pad_start[i] + ((len + TC_M - 1) / TC_M) * TC_M;
    }
    const int32_t n_pad = std::max(pad_start[ninst], TC_M);
    std::vector<int32_t> src(n_pad, -1);
    std::vector<int4> tasks;
    std::vector<int32_t> shifts;
    for (int i = 0; i < ninst; ++i) {
        const int32_t len = inst[i + 1] - inst[i];
        for (int32_t r = 0; r < len; ++r) src[pad_start[i] + r] = inst[i] + r;
        const int32_t tiles = (len + TC_M - 1) / TC_M;
        for (int32_t t = 0; t < tiles; t += qt) {
            tasks.push_back(make_int4(pad_start[i] + t * TC_M, pad_start[i] / TC_N, tiles, pad_start[i] + len));
            shifts.push_back(inst[i] - pad_start[i]);
        }
    }
    if (tasks.empty()) return;
    DevArray<int32_t> d_src(src.size(), s), d_shift(shifts.size(), s);
    DevArray<int4> d_tasks(tasks.size(), s);
    DevArray<float> norms(n_pad, s);
    UMAPB_CUDA(cudaMemcpyAsync(d_src.get(), src.data(), src.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(d_tasks.get(), tasks.data(), tasks.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(d_shift.get(), shifts.data(), shifts.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    run_candidates(data, inst[ninst], dim, kcap, n_pad, d_src.get(), static_cast<int32_t>(tasks.size()),
                   d_tasks.get(), d_shift.get(), cand_idx, cand_d2, norms.get(), d_err, s);
    UMAPB_SYNC(s);   // the host vectors above are the copies' sources
}

}  // namespace umapb
