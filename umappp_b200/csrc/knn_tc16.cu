// Tensor-core candidate search for the exact kNN of float data, FP16 operands
// (sm_100a, tcgen05.mma kind::f16).
//
// The data are scaled by a power of two s (so every |x s| <= 1; the scaling
// is exact) and every coordinate is split as x s = hi + lo with hi = fp16(x s)
// and lo = fp16(x s - hi); q.r = hi.hi + hi.lo + lo.hi ("3xFP16", the lo.lo
// term is below 2^-22 relative), products exact in FP32 and accumulated in
// FP32 in tensor memory.  This carries the same ~22 significant bits as the
// TF32 split (knn_tc.cu) at twice the tensor rate and half the operand bytes.
// As there, the norm rides in one extra K column: A = [x s, 1],
// B = [x s, -|x s|^2 / 2], so the accumulator is (q.r - |r|^2 / 2) s^2.
//
// One CTA owns QT query tiles of 128 rows (QT = 2 for up to 63 dimensions)
// and streams all reference tiles (N = 128) of its instance through an
// NS-stage shared-memory ring; each reference tile feeds QT MMA groups, one
// per query tile, into double-buffered TMEM accumulators.  Warp roles:
//   warp 0      TMA producer (query tiles once, then the reference ring);
//   warp 1      MMA issuer (one lane) and TMEM owner;
//   warps 2..   epilogue, 4 per query tile: one query row per thread (TMEM
//               lane), all 128 columns of each tile, a screen of each
//               32-column chunk by its maximum against the current k-th
//               distance (columns are compared one by one only in chunks
//               that pass) and a sorted
//               register list of the KCAP best (distance, index) pairs.
// No cluster multicast.  Every mbarrier wait is bounded (tc_ptx.cuh): on
// expiry the kernel records an error, raises a CTA-wide abort flag so the
// other roles stop waiting, waits for its loads and MMAs in flight, frees
// TMEM and returns.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "stages.cuh"
#include "tc_ptx.cuh"

namespace umapb {

namespace {

using namespace tc;

constexpr int H_M = 128;       // rows per query tile (the MMA's M)
constexpr int H_N = 128;       // references per tile (N)
constexpr int H_KCHUNK = 64;   // FP16 elements per 128-byte swizzle row
constexpr int H_KSTEP = 16;    // K of one kind::f16 MMA

// Instruction descriptor: D = F32, A = B = F16, both K-major, M = 128, N = 128.
constexpr uint32_t kIdesc16 = (1u << 4) | (0u << 7) | (0u << 10) | (uint32_t(H_N >> 3) << 17) | (uint32_t(H_M >> 4) << 24);

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(kIdesc16), "r"(accumulate)
        : "memory");
}

// ------------------------------------------------------------ scale ------

// max |x| over the data (as float bits; non-negative floats order like their bits)
__global__ void absmax_kernel(const float* __restrict__ data, size_t count, unsigned int* __restrict__ out) {
    unsigned int m = 0;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x)
        m = max(m, __float_as_uint(fabsf(data[i])));
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__device__ __forceinline__ void split_f16(float v, __half& hi, __half& lo) {
    hi = __float2half_rn(v);
    lo = __float2half_rn(v - __half2float(hi));
}

__global__ void scatter_norms_kernel(const int32_t* __restrict__ row_map, const float* __restrict__ onorm,
                                     int32_t n_pad, float* __restrict__ out) {
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n_pad; r += gridDim.x * blockDim.x)
        if (row_map[r] >= 0) out[row_map[r]] = onorm[r];
}

// Operands [n_pad, k_pad] (FP16 pairs, zero padded):
//   queries    A = [x s, 1]
//   references B = [x s, -|x s|^2 / 2]   (-60000 in the norm column of padding rows)
// norms[i] = |x_i|^2 (FP64 sum rounded to FP32, unscaled; +inf for padding).
// pad_src (batched runs) maps operand row i to its data row, or -1 for a
// padding row; without it, rows below n are data rows.
__global__ void prepare16_kernel(const float* __restrict__ data, int32_t n, int32_t dim, int32_t n_pad, int32_t k_pad,
                                 float s, __half* __restrict__ a_hi, __half* __restrict__ a_lo,
                                 __half* __restrict__ b_hi, __half* __restrict__ b_lo, float* __restrict__ norms,
                                 const int32_t* __restrict__ pad_src) {
    // one warp per operand row: the data row is read and the four operand rows
    // written by consecutive lanes; the FP64 norm is a warp reduction
    const double s2 = static_cast<double>(s) * s;
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n_pad;
         i += warps) {
        const int64_t src = pad_src ? pad_src[i] : (i < n ? i : -1);
        const bool real = src >= 0;   // the same for the whole warp
        double nrm = 0;
        if (real) {
            for (int d = lane; d < dim; d += 32) {
                const double v = data[src * dim + d];
                nrm += v * v;
            }
        }
        for (int o = 16; o > 0; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
        if (lane == 0) norms[i] = real ? static_cast<float>(nrm) : CUDART_INF_F;
        const int64_t row = i * k_pad;
        for (int d = lane; d < k_pad; d += 32) {
            __half h = __float2half_rn(0.0f), l = h;
            if (real && d < dim) split_f16(data[src * dim + d] * s, h, l);
            __half ah = h;
            const __half al = l;
            if (d == dim) {
                if (real) {
                    ah = __float2half_rn(1.0f);
                    split_f16(static_cast<float>(-0.5 * nrm * s2), h, l);
                } else {
                    h = __float2half_rn(-60000.0f);   // padding reference: d2 beyond any candidate
                }
            }
            a_hi[row + d] = ah;
            a_lo[row + d] = al;
            b_hi[row + d] = h;
            b_lo[row + d] = l;
        }
    }
}

// ----------------------------------------------------------- main kernel --

template <int KC, int QT, int NS>
struct H16Smem {
    __half a_hi[QT][KC][H_M * H_KCHUNK];   // 16 KB per [KC] chunk, 1024-byte aligned
    __half a_lo[QT][KC][H_M * H_KCHUNK];
    __half b_hi[NS][KC][H_N * H_KCHUNK];
    __half b_lo[NS][KC][H_N * H_KCHUNK];
    uint64_t full[NS];
    uint64_t empty[NS];
    uint64_t tmem_full[QT][2];
    uint64_t tmem_empty[QT][2];
    uint64_t a_full;
    uint64_t mma_done;   // drain after an abort (mma_drain)
    uint32_t tmem_base;
    int abort_flag;
};

template <int QT>
constexpr int h16_threads() { return 64 + 128 * QT; }
template <int QT>
constexpr uint32_t h16_tmem_cols() { return QT == 2 ? 512u : 256u; }

// One chunk of 32 accumulator columns (chunk ch of the tile whose column 0 is
// operand row col0) against the query's candidate list: the chunk's maximum
// screens it; in a passing chunk each column is compared, and candidates
// nearer than the current k-th enter the list.
template <int KCAP>
__device__ __forceinline__ void scan_chunk(const uint32_t (&r)[32], int ch, int col0, int q, bool diag, int valid,
                                           float qn, int shift, float (&bd)[KCAP], int (&bi)[KCAP], float& thr,
                                           float& athr) {
    if (!(chunk_max32(r) > athr)) return;   // rare after the first tiles
    uint32_t mask = 0;
#pragma unroll
    for (int i = 0; i < 32; ++i) mask |= (__uint_as_float(r[i]) > athr ? 1u : 0u) << i;
    if (diag && (q - col0) / 32 == ch) mask &= ~(1u << ((q - col0) & 31));   // self
    const int vc = valid - ch * 32;
    if (vc < 32) mask &= (vc <= 0) ? 0u : ((1u << vc) - 1u);
    while (mask) {   // candidates better than the current k-th
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

// Merged walk over the (ascending) reference-tile lists of a CTA's query
// tiles: next() yields each tile of the union once, with the mask of the
// query tiles whose lists hold it.
template <int QT>
struct ListWalk {
    const int32_t* list[QT];
    int32_t len[QT];
    int32_t pos[QT];
    __device__ __forceinline__ bool next(int32_t& tile, unsigned& mask) {
        tile = INT32_MAX;
#pragma unroll
        for (int t = 0; t < QT; ++t)
            if (pos[t] < len[t]) tile = min(tile, list[t][pos[t]]);
        if (tile == INT32_MAX) return false;
        mask = 0;
#pragma unroll
        for (int t = 0; t < QT; ++t)
            if (pos[t] < len[t] && list[t][pos[t]] == tile) {
                mask |= 1u << t;
                ++pos[t];
            }
        return true;
    }
};

// One CTA per task {first operand row, first query tile, query tiles, -}:
// query tile t (rows q_base + 128 t ..) scans the reference tiles
// tile_list[qlist_off[qt0 + t] .. + qlist_len[qt0 + t]).  Candidates are kept
// as operand rows and written by data row through row_map (-1: padding row).
template <int KC, int QT, int NS, int KCAP>
__global__ void __launch_bounds__(h16_threads<QT>(), 1)
    knn_tc16_kernel(const __grid_constant__ CUtensorMap map_ahi, const __grid_constant__ CUtensorMap map_alo,
                    const __grid_constant__ CUtensorMap map_bhi, const __grid_constant__ CUtensorMap map_blo,
                    const float* __restrict__ norms, float s2, float inv_s2, int32_t ksteps,
                    int32_t* __restrict__ cand_idx, float* __restrict__ cand_d2, int* __restrict__ err,
                    const int4* __restrict__ tasks, const int64_t* __restrict__ qlist_off,
                    const int32_t* __restrict__ qlist_len, const int32_t* __restrict__ tile_list,
                    const int32_t* __restrict__ row_map, long long wait_limit) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    using Smem = H16Smem<KC, QT, NS>;
    Smem& sm = *reinterpret_cast<Smem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int4 task = tasks[blockIdx.x];
    const int32_t q_base = task.x, qt0 = task.y, nq = task.z;
    ListWalk<QT> walk;
#pragma unroll
    for (int t = 0; t < QT; ++t) {
        walk.list[t] = tile_list + (t < nq ? qlist_off[qt0 + t] : 0);
        walk.len[t] = t < nq ? qlist_len[qt0 + t] : 0;
        walk.pos[t] = 0;
    }
    volatile int* abort_flag = &sm.abort_flag;
    constexpr uint32_t TMEM_COLS = h16_tmem_cols<QT>();

    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], 1);
        }
        for (int t = 0; t < QT; ++t) {
            for (int b = 0; b < 2; ++b) {
                mbar_init(&sm.tmem_full[t][b], 1);
                mbar_init(&sm.tmem_empty[t][b], 128);
            }
        }
        mbar_init(&sm.a_full, 1);
        mbar_init(&sm.mma_done, 1);
        sm.abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem_base)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = sm.tmem_base;

    constexpr uint32_t A_BYTES = 2u * QT * KC * H_M * H_KCHUNK * 2u;
    constexpr uint32_t B_BYTES = 2u * KC * H_N * H_KCHUNK * 2u;
    int issued = 0;

    if (warp == 0) {
        if (lane == 0) {
            mbar_arrive_expect_tx(&sm.a_full, A_BYTES);
            for (int t = 0; t < QT; ++t) {
                for (int c = 0; c < KC; ++c) {
                    tma_load_2d(sm.a_hi[t][c], &map_ahi, &sm.a_full, c * H_KCHUNK, q_base + t * H_M);
                    tma_load_2d(sm.a_lo[t][c], &map_alo, &sm.a_full, c * H_KCHUNK, q_base + t * H_M);
                }
            }
            int32_t tile;
            unsigned mask;
            for (int u = 0; walk.next(tile, mask); ++u) {
                const int s = u % NS;
                if (!mbar_wait(&sm.empty[s], ((u / NS) & 1) ^ 1, abort_flag, err, wait_limit)) break;
                mbar_arrive_expect_tx(&sm.full[s], B_BYTES);
                for (int c = 0; c < KC; ++c) {
                    tma_load_2d(sm.b_hi[s][c], &map_bhi, &sm.full[s], c * H_KCHUNK, tile * H_N);
                    tma_load_2d(sm.b_lo[s][c], &map_blo, &sm.full[s], c * H_KCHUNK, tile * H_N);
                }
                ++issued;
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && mbar_wait(&sm.a_full, 0, abort_flag, err, wait_limit)) {
            bool ok = true;
            int32_t used[QT];   // accumulator rounds of each query tile so far
#pragma unroll
            for (int t = 0; t < QT; ++t) used[t] = 0;
            int32_t tile;
            unsigned mask;
            for (int u = 0; ok && walk.next(tile, mask); ++u) {
                const int s = u % NS;
                if (!mbar_wait(&sm.full[s], (u / NS) & 1, abort_flag, err, wait_limit)) break;
                for (int t = 0; t < QT; ++t) {
                    if (!(mask & (1u << t))) continue;
                    const int c_t = used[t]++;
                    const int buf = c_t & 1;
                    if (!mbar_wait(&sm.tmem_empty[t][buf], ((c_t >> 1) & 1) ^ 1, abort_flag, err, wait_limit)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d = tmem_base + (t * 2 + buf) * H_N;
                    uint32_t acc = 0;
#pragma unroll
                    for (int c = 0; c < KC; ++c) {
#pragma unroll
                        for (int kk = 0; kk < H_KCHUNK / H_KSTEP; ++kk) {
                            // K-steps past the last non-zero column (data + norm) contribute nothing
                            if (c * (H_KCHUNK / H_KSTEP) + kk >= ksteps) break;
                            const int off = kk * H_KSTEP;   // 16 FP16 = 32 bytes along K inside the swizzle row
                            const uint64_t ah = smem_desc(sm.a_hi[t][c] + off), al = smem_desc(sm.a_lo[t][c] + off);
                            const uint64_t bh = smem_desc(sm.b_hi[s][c] + off), bl = smem_desc(sm.b_lo[s][c] + off);
                            mma_f16(d, al, bh, acc);
                            acc = 1;
                            mma_f16(d, ah, bl, 1);
                            mma_f16(d, ah, bh, 1);
                        }
                    }
                    mma_commit(&sm.tmem_full[t][buf]);
                }
                if (ok) mma_commit(&sm.empty[s]);
            }
        }
    } else {
        // epilogue: warps 2 .. 2 + 4 QT - 1; query tile t = (warp - 2) / 4,
        // TMEM lanes 32 * (warp % 4) .. + 31, one query row per thread
        const int t = (warp - 2) >> 2;
        const int quarter = warp & 3;
        const int row = quarter * 32 + lane;
        const int q = q_base + t * H_M + row;
        const int32_t src = (t < nq) ? row_map[q] : -1;   // data row, -1: padding or no tile
        const float qn = (src >= 0) ? norms[q] * s2 : 0.0f;   // |q s|^2
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
        const int32_t* my_list = walk.list[t];
        const int32_t my_len = walk.len[t];
        for (int c_t = 0; c_t < my_len; ++c_t) {
            const int buf = c_t & 1;
            if (!mbar_wait(&sm.tmem_full[t][buf], (c_t >> 1) & 1, abort_flag, err, wait_limit)) break;
            tc_fence_after();
            const uint32_t taddr = tmem_base + (uint32_t(quarter * 32) << 16) + (t * 2 + buf) * H_N;
            const int col0 = my_list[c_t] * H_N;   // operand row of column 0
            const bool diag = (col0 <= q && q < col0 + H_N);
            // Two chunks of 32 columns per TMEM round trip; the accumulator is
            // released to the MMA as soon as its last columns are in registers.
#pragma unroll 1
            for (int pr = 0; pr < H_N / 64; ++pr) {
                uint32_t ra[32], rb[32];
                tmem_load32_async(taddr + pr * 64, ra);
                tmem_load32_async(taddr + pr * 64 + 32, rb);
                tmem_wait_ld(ra);
                tmem_wait_ld(rb);
                if (pr == H_N / 64 - 1) {
                    tc_fence_before();
                    mbar_arrive(&sm.tmem_empty[t][buf]);
                }
                scan_chunk<KCAP>(ra, 2 * pr, col0, q, diag, H_N, qn, 0, bd, bi, thr, athr);
                scan_chunk<KCAP>(rb, 2 * pr + 1, col0, q, diag, H_N, qn, 0, bd, bi, thr, athr);
            }
        }
        if (src >= 0 && *abort_flag == 0) {
            // data rows: through the row map (candidates were collected as operand rows)
            const size_t out_row = static_cast<size_t>(src);
#pragma unroll
            for (int i = 0; i < KCAP; ++i) {
                cand_idx[out_row * KCAP + i] = bi[i] >= 0 ? row_map[bi[i]] : -1;
                cand_d2[out_row * KCAP + i] = bd[i] * inv_s2;   // exact: a power of two
            }
        }
    }

    // drain: loads in flight must land before the CTA's shared memory goes away
    if (warp == 0 && lane == 0 && *abort_flag) {
        for (int it = (issued > NS ? issued - NS : 0); it < issued; ++it) {
            const int s = it % NS;
            for (long long i = 0; i < WAIT_LIMIT && !mbar_try_wait(&sm.full[s], (it / NS) & 1); ++i) __nanosleep(64);
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
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
    }
}

// --------------------------------------------------------------- host side --

PFN_cuTensorMapEncodeTiled_v12000 get_encode16() {
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

// 2-D FP16 tensor [rows, k_pad] (k_pad contiguous), box 128 rows x 64 columns, 128-byte swizzle.
CUtensorMap make_map16(const __half* base, int64_t rows, int k_pad) {
    CUtensorMap m;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(k_pad), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(k_pad) * sizeof(__half)};
    const cuuint32_t box[2] = {H_KCHUNK, 128};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = get_encode16()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<__half*>(base), dims, strides,
                                      box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    require(r == CUDA_SUCCESS, "cuTensorMapEncodeTiled failed", UMAPB_ERR_CUDA);
    return m;
}

struct Maps16 {
    CUtensorMap ahi, alo, bhi, blo;
    int ksteps;
};

template <int KC, int QT, int NS, int KCAP>
void launch16(const Maps16& m, const float* norms, float s2, float inv_s2, int32_t ctas, const KnnTasks& tk,
              const int32_t* row_map, int32_t* cand_idx, float* cand_d2, int* err, cudaStream_t s) {
    const size_t smem = sizeof(H16Smem<KC, QT, NS>) + 1024;
    static_assert(sizeof(H16Smem<KC, QT, NS>) + 1024 <= 227 * 1024, "shared memory budget");
    static std::once_flag once;
    std::call_once(once, [&] {
        UMAPB_CUDA(cudaFuncSetAttribute(knn_tc16_kernel<KC, QT, NS, KCAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(smem)));
    });
    knn_tc16_kernel<KC, QT, NS, KCAP><<<ctas, h16_threads<QT>(), smem, s>>>(
        m.ahi, m.alo, m.bhi, m.blo, norms, s2, inv_s2, m.ksteps, cand_idx, cand_d2, err, tk.tasks.get(),
        tk.qlist_off.get(), tk.qlist_len.get(), tk.tile_list.get(), row_map, device_wait_limit());
    UMAPB_LAUNCH_CHECK();
}

// Launch shapes, coded 10 QT + NS (shared memory: QT * KC * 32 KB of query
// tiles plus NS * KC * 32 KB of reference ring): for KC = 1, 24 = two query
// tiles per CTA with a 4-stage ring (160 KB: one CTA per SM, 512 TMEM
// columns), 12 = one query tile with a 2-stage ring (96 KB: two CTAs per SM,
// 256 columns each, tasks of half the work); KC = 2 takes 12 only.  (One
// query tile with a 4-stage ring and one CTA per SM was measured slower than
// both: 27.6 ms at 1M against 19.5 and 21.2 -- the two CTAs' overlapping
// epilogues matter more than the ring's depth.)
constexpr int qt_for(int kc) { return kc == 1 ? 2 : 1; }

template <int KC, int QT, int NS>
void launch16_shape(int kcap, const Maps16& m, const float* norms, float s2, float inv_s2, int32_t ctas,
                    const KnnTasks& tk, const int32_t* rm, int32_t* ci, float* cd, int* err, cudaStream_t s) {
    if (kcap == 16) launch16<KC, QT, NS, 16>(m, norms, s2, inv_s2, ctas, tk, rm, ci, cd, err, s);
    else if (kcap == 24) launch16<KC, QT, NS, 24>(m, norms, s2, inv_s2, ctas, tk, rm, ci, cd, err, s);
    else launch16<KC, QT, NS, 32>(m, norms, s2, inv_s2, ctas, tk, rm, ci, cd, err, s);
}

}  // namespace

int knn_tc16_query_tiles(int32_t dim) { return qt_for((dim + 1 + H_KCHUNK - 1) / H_KCHUNK); }

std::vector<int> knn_tc16_shapes(int32_t dim) {
    return (dim + 1 + H_KCHUNK - 1) / H_KCHUNK == 1 ? std::vector<int>{24, 12} : std::vector<int>{12};
}

bool knn_tc16_supported(int32_t dim, int kcap) {
    return dim >= 1 && dim + 1 <= 2 * H_KCHUNK && (kcap == 16 || kcap == 24 || kcap == 32);
}

// Power-of-two scale s with max |x s| < 1 (exact scaling), or 0 when the data
// hold no finite non-zero maximum within [2^-60, 2^60] (NaN, inf, all zeros or
// extreme magnitudes), for which the FP16 search is not used.
float knn_tc16_scale(const float* data, size_t count, cudaStream_t s) {
    DevArray<unsigned int> amax(1, s);
    amax.zero(s);
    absmax_kernel<<<grid_for(count, 256, 1024), 256, 0, s>>>(data, count, amax.get());
    UMAPB_LAUNCH_CHECK();
    unsigned int bits = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&bits, amax.get(), sizeof(bits), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    float m = 0;
    std::memcpy(&m, &bits, sizeof(m));
    if (!(m >= 0x1p-60f && m <= 0x1p60f)) return 0.0f;
    int e = 0;
    std::frexp(m, &e);   // m = f 2^e, f in [0.5, 1)
    return std::ldexp(1.0f, -e);
}

// Pruned search (knn_tree.cu): operands in the tiles' row order, one CTA per
// task.  Norms (needed in operand order by the kernel) are scattered to data
// rows for the caller.
void knn_tc16_run_tasks(const float* data, int32_t dim, int kcap, float scale, const KnnTiles& tiles,
                        const KnnTasks& tasks, int32_t* cand_idx, float* cand_d2, float* norms_by_row, int* d_err,
                        cudaStream_t s, float* kernel_ms, int shape) {
    require(knn_tc16_supported(dim, kcap), "tensor-core kNN: unsupported dimension or candidate count");
    require(scale > 0.0f, "tensor-core kNN: no usable scale for the data");
    const int32_t n_pad = tiles.n_pad;
    const int kc = (dim + 1 + H_KCHUNK - 1) / H_KCHUNK;
    const int k_pad = kc * H_KCHUNK;
    const size_t elems = static_cast<size_t>(n_pad) * k_pad;
    DevArray<__half> ahi(elems, s), alo(elems, s), bhi(elems, s), blo(elems, s);
    DevArray<float> onorm(n_pad, s);
    prepare16_kernel<<<grid_for(n_pad, 256 / 32), 256, 0, s>>>(data, 0, dim, n_pad, k_pad, scale, ahi.get(), alo.get(),
                                                           bhi.get(), blo.get(), onorm.get(), tiles.row_map.get());
    UMAPB_LAUNCH_CHECK();
    Maps16 m;
    m.ahi = make_map16(ahi.get(), n_pad, k_pad);
    m.alo = make_map16(alo.get(), n_pad, k_pad);
    m.bhi = make_map16(bhi.get(), n_pad, k_pad);
    m.blo = make_map16(blo.get(), n_pad, k_pad);
    m.ksteps = (dim + 1 + H_KSTEP - 1) / H_KSTEP;
    const float s2 = scale * scale, inv_s2 = 1.0f / s2;
    cudaEvent_t ev0 = event_get(), ev1 = event_get();
    UMAPB_CUDA(cudaEventRecord(ev0, s));
    if (shape <= 0) shape = kc == 1 ? 24 : 12;
    require(kc == 1 ? (shape == 24 || shape == 12) : shape == 12, "tensor-core kNN: unsupported launch shape");
    if (tasks.count > 0) {
        const int32_t* rm = tiles.row_map.get();
        if (kc == 1 && shape == 24)
            launch16_shape<1, 2, 4>(kcap, m, onorm.get(), s2, inv_s2, tasks.count, tasks, rm, cand_idx, cand_d2, d_err, s);
        else if (kc == 1)
            launch16_shape<1, 1, 2>(kcap, m, onorm.get(), s2, inv_s2, tasks.count, tasks, rm, cand_idx, cand_d2, d_err, s);
        else
            launch16_shape<2, 1, 2>(kcap, m, onorm.get(), s2, inv_s2, tasks.count, tasks, rm, cand_idx, cand_d2, d_err, s);
    }
    UMAPB_CUDA(cudaEventRecord(ev1, s));
    scatter_norms_kernel<<<grid_for(n_pad, 256), 256, 0, s>>>(tiles.row_map.get(), onorm.get(), n_pad, norms_by_row);
    UMAPB_LAUNCH_CHECK();
    if (kernel_ms) {
        UMAPB_CUDA(cudaEventSynchronize(ev1));
        UMAPB_CUDA(cudaEventElapsedTime(kernel_ms, ev0, ev1));
    }
    event_put(ev0);
    event_put(ev1);
}

}  // namespace umapb
