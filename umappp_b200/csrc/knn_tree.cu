// Tile pruning for the exact tensor-core kNN: a spatial ordering of the
// points and, per block of queries, the reference tiles that can hold one of
// its neighbours.
//
// Ordering (projection tree): the points of every instance are split
// recursively -- projected on the direction from a random point of the
// segment to the segment's point farthest from it, sorted by the projection,
// cut at a wide gap of the projections if there is one (a hard cut: the two
// sides go to separate padded runs of tiles) and otherwise so that the left
// part is a whole number of 128-row tiles -- until each segment is one tile.
// The farthest point of a segment that spans several clusters lies in
// another cluster than the random one, so the direction separates clusters,
// and clustered data (single-cell profiles, mixtures) come out with tiles that
// each sit in one cluster.
//
// Bounds: every 128-row reference tile T and every query block B (the rows one
// CTA of the search serves) gets a centroid c (FP32) and a radius R (an upper
// bound of |x - c| over its points, FP64 rounded up).  For a query q in B and a
// point r in T the triangle inequality gives
//     |q - r| >= |c_B - c_T| - R_B - R_T =: lb(B, T),
// and the k-th neighbour of every query q of B lies within a radius rho_B of q
// -- the largest over B's queries of the distance to the k-th nearest other
// point of B (computed exactly, rounded up; it needs |B| - 1 >= k), or a bound
// through a nearby tile.  A tile with lb(B, T) > rho_B cannot hold any of
// q's k nearest neighbours: it is left out of B's list.  This is exact (no
// neighbour is lost); for data without cluster structure the lists simply
// cover every tile.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

#include "stages.cuh"

namespace umapb {

namespace {

constexpr int TREE_LEAF = 128;
// A cut goes at the widest gap of a segment's sorted projections (and starts a
// new padded run) when that gap exceeds this many times the typical spacing
// of the middle half; otherwise the cut keeps tiles whole.
constexpr float GAP_FACTOR = 16.0f;

// Order-preserving map of a float to 32 unsigned bits, and its inverse.
__device__ __forceinline__ uint32_t float_order_bits(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float order_bits_float(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// The points of the segments split at a level ("active"), concatenated: item
// i belongs to active segment j = the last with aoff[j] <= i and sits at
// position ast[j] + i - aoff[j] of perm.
__device__ __forceinline__ int active_segment(int64_t i, int32_t nact, const int32_t* __restrict__ aoff) {
    int lo = 0, hi = nact - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (aoff[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// The window of a segment of len points in which a hard cut may fall.
__host__ __device__ __forceinline__ int32_t gap_window_first(int32_t len) { return len / 16 > 1 ? len / 16 : 1; }
__host__ __device__ __forceinline__ int32_t gap_window_last(int32_t len) { return (15 * len) / 16; }

// best[seg] = max(best[seg], key) for every lane of the warp, with one atomic
// per run of lanes that share a segment (seg < 0: nothing).  The lanes' items
// are consecutive, so equal segments form runs: a segmented max down each run
// leaves the run's maximum in its first lane.  All 32 lanes take part.
__device__ __forceinline__ void warp_segment_max(unsigned long long* __restrict__ best, int seg,
                                                 unsigned long long key) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long k2 = __shfl_down_sync(0xffffffffu, key, o);
        const int s2 = __shfl_down_sync(0xffffffffu, seg, o);
        if (lane + o < 32 && s2 == seg && k2 > key) key = k2;
    }
    const int prev = __shfl_up_sync(0xffffffffu, seg, 1);
    if (seg >= 0 && (lane == 0 || prev != seg)) atomicMax(&best[seg], key);
}

// The point of every active segment farthest from its point a (position
// aa[j]; squared FP32 distance): each item folds (distance bits, reversed
// position) into its segment's 64-bit maximum, so that ties go to the
// smallest position.  The loop runs whole warps (warp_segment_max).
__global__ void far_point_kernel(const float* __restrict__ data, int32_t dim, const int32_t* __restrict__ perm,
                                 int32_t nact, const int32_t* __restrict__ aoff, const int32_t* __restrict__ ast,
                                 const int32_t* __restrict__ aa, int64_t total, unsigned long long* __restrict__ best) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31); base < total;
         base += stride) {
        const int64_t i = base + (threadIdx.x & 31);
        int seg = -1;
        unsigned long long key = 0;
        if (i < total) {
            const int j = active_segment(i, nact, aoff);
            const int32_t p = ast[j] + static_cast<int32_t>(i - aoff[j]);
            const float* x = data + static_cast<size_t>(perm[p]) * dim;
            const float* xa = data + static_cast<size_t>(perm[aa[j]]) * dim;
            float d2 = 0.0f;
            for (int d = 0; d < dim; ++d) {
                const float v = x[d] - xa[d];
                d2 = fmaf(v, v, d2);
            }
            seg = j;
            key = (static_cast<unsigned long long>(__float_as_uint(d2)) << 32) |
                  static_cast<unsigned long long>(0xffffffffu - static_cast<uint32_t>(p));
        }
        warp_segment_max(best, seg, key);
    }
}

// Sort key of every active item: its active segment in the high bits, the
// point's projection on x_a - x_b (b: the segment's far point, from
// far_point_kernel) in the low 32 bits; the item's point goes to vals.  One
// radix sort of these keys sorts every active segment at once.
__global__ void rp_keys_kernel(const float* __restrict__ data, int32_t dim, const int32_t* __restrict__ perm,
                               int32_t nact, const int32_t* __restrict__ aoff, const int32_t* __restrict__ ast,
                               const int32_t* __restrict__ aa, const unsigned long long* __restrict__ far,
                               int64_t total, unsigned long long* __restrict__ keys, int32_t* __restrict__ vals) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const int j = active_segment(i, nact, aoff);
        const int32_t p = ast[j] + static_cast<int32_t>(i - aoff[j]);
        const int32_t b = static_cast<int32_t>(0xffffffffu - static_cast<uint32_t>(far[j] & 0xffffffffu));
        const float* x = data + static_cast<size_t>(perm[p]) * dim;
        const float* xa = data + static_cast<size_t>(perm[aa[j]]) * dim;
        const float* xb = data + static_cast<size_t>(perm[b]) * dim;
        float key = 0.0f;
        for (int d = 0; d < dim; ++d) key = fmaf(x[d], xa[d] - xb[d], key);
        keys[i] = (static_cast<unsigned long long>(j) << 32) | float_order_bits(key);
        vals[i] = perm[p];
    }
}

// perm at the active positions from the sorted items.
__global__ void scatter_active_kernel(int32_t nact, const int32_t* __restrict__ aoff, const int32_t* __restrict__ ast,
                                      int64_t total, const int32_t* __restrict__ vals, int32_t* __restrict__ perm) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const int j = active_segment(i, nact, aoff);
        perm[ast[j] + static_cast<int32_t>(i - aoff[j])] = vals[i];
    }
}

__device__ __forceinline__ float sorted_key(const unsigned long long* __restrict__ keys, int64_t p) {
    return order_bits_float(static_cast<uint32_t>(keys[p] & 0xffffffffull));
}

__global__ void iota_kernel(int32_t* __restrict__ v, int32_t n) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

// Widest gap between consecutive sorted keys with the cut in the window
// [start + len/16, start + 15 len/16] of each active segment j: every position
// of every window folds (gap bits, reversed position) into its segment's
// 64-bit maximum, so that ties go to the smallest position.
__global__ void widest_gap_kernel(const unsigned long long* __restrict__ keys, int32_t nact,
                                  const int32_t* __restrict__ seg_start,
                                  const int32_t* __restrict__ seg_end, const int64_t* __restrict__ mid_off,
                                  int64_t total, unsigned long long* __restrict__ best) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31); base < total;
         base += stride) {   // whole warps (warp_segment_max)
        const int64_t i = base + (threadIdx.x & 31);
        int seg = -1;
        unsigned long long key = 0;
        if (i < total) {
            int lo = 0, hi = nact - 1;   // segment of window item i: last offset <= i
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (mid_off[mid] <= i) lo = mid; else hi = mid - 1;
            }
            const int32_t st = seg_start[lo], len = seg_end[lo] - st;
            const int32_t p = st + gap_window_first(len) + static_cast<int32_t>(i - mid_off[lo]);
            const float g = fmaxf(sorted_key(keys, p) - sorted_key(keys, p - 1), 0.0f);
            seg = lo;
            key = (static_cast<unsigned long long>(__float_as_uint(g)) << 32) |
                  static_cast<unsigned long long>(0xffffffffu - static_cast<uint32_t>(p - st));
        }
        warp_segment_max(best, seg, key);
    }
}

// Sorted keys at the ends of each segment's middle half.
__global__ void middle_spread_kernel(const unsigned long long* __restrict__ keys, int32_t nact,
                                     const int32_t* __restrict__ seg_start,
                                     const int32_t* __restrict__ seg_end, float* __restrict__ lo_key,
                                     float* __restrict__ hi_key) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nact; j += gridDim.x * blockDim.x) {
        const int32_t st = seg_start[j], len = seg_end[j] - st;
        lo_key[j] = sorted_key(keys, st + max(1, len / 4));
        hi_key[j] = sorted_key(keys, st + (3 * len) / 4);
    }
}

// row_map[run_dst[r] + i] = perm[run_src[r] + i] for the points of every run.
__global__ void place_runs_kernel(const int32_t* __restrict__ perm, int32_t nrun, const int32_t* __restrict__ run_src,
                                  const int32_t* __restrict__ run_len, const int32_t* __restrict__ run_dst, int32_t n,
                                  int32_t* __restrict__ row_map) {
    for (int32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        int lo = 0, hi = nrun - 1;   // run holding position p: last source start <= p
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (run_src[mid] <= p) lo = mid; else hi = mid - 1;
        }
        row_map[run_dst[lo] + (p - run_src[lo])] = perm[p];
    }
}

// Centroid, radius and real-row count of every group of 'rows' operand rows.
__global__ void group_bounds_kernel(const float* __restrict__ data, int32_t dim, const int32_t* __restrict__ row_map,
                                    int32_t rows, float* __restrict__ centroid, float* __restrict__ radius,
                                    int32_t* __restrict__ count, float* __restrict__ centroid_t, int32_t ngroups) {
    const int32_t g = blockIdx.x;
    const int32_t r0 = g * rows;
    __shared__ double red[256];
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    int c = 0;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) c += (row_map[r0 + r] >= 0);
    atomicAdd(&cnt, c);
    __syncthreads();
    const int m = cnt;
    float* cg = centroid + static_cast<size_t>(g) * dim;
    for (int d = threadIdx.x; d < dim; d += blockDim.x) {
        double s = 0;
        for (int r = 0; r < rows; ++r) {
            const int32_t src = row_map[r0 + r];
            if (src >= 0) s += data[static_cast<size_t>(src) * dim + d];
        }
        cg[d] = m ? static_cast<float>(s / m) : 0.0f;
        if (centroid_t) centroid_t[static_cast<size_t>(d) * ngroups + g] = cg[d];   // [dim][groups] copy
    }
    __syncthreads();
    double worst = 0;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) {
        const int32_t src = row_map[r0 + r];
        if (src < 0) continue;
        double s = 0;
        for (int d = 0; d < dim; ++d) {
            const double v = static_cast<double>(data[static_cast<size_t>(src) * dim + d]) - cg[d];
            s += v * v;
        }
        worst = fmax(worst, s);
    }
    red[threadIdx.x] = worst;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        // rounded up, with a margin for the FP64 sum
        radius[g] = __double2float_ru(sqrt(red[0]) * (1.0 + 1e-9) + 1e-30);
        count[g] = m;
    }
}

constexpr int KTH_MAX = 32;
constexpr float D2_LOW = 1.0f - 1.0e-4f;    // lower-bound factor on FP32 squared distances
constexpr float D2_HIGH = 1.0f + 1.0e-4f;   // upper-bound factor

// For every tile g: a distance within which each of its points has at least k
// other points of the tile -- the largest over the tile's points of the
// distance to the k-th nearest other point (FP32 sums of squares, relative
// error below (dim + 2) 2^-24, rounded up through the D2_HIGH margins) --, or
// infinity when the tile holds k points or fewer or k exceeds KM (<= KTH_MAX).
// One block of TREE_LEAF threads per tile, one thread per row; the tile's
// points are staged in shared memory ([TREE_LEAF][dim]).
template <int KM>
__global__ void __launch_bounds__(TREE_LEAF)
    tile_kth_kernel(const float* __restrict__ data, int32_t dim, const int32_t* __restrict__ row_map,
                    const int32_t* __restrict__ count, int32_t k, float* __restrict__ kth_out) {
    extern __shared__ float pts[];
    __shared__ int valid[TREE_LEAF];
    __shared__ float red[TREE_LEAF / 32];
    const int32_t g = blockIdx.x;
    const int r = threadIdx.x;
    if (k > KM || count[g] < k + 1) {   // uniform over the block
        if (r == 0) kth_out[g] = CUDART_INF_F;
        return;
    }
    const int32_t* rows = row_map + static_cast<size_t>(g) * TREE_LEAF;
    valid[r] = rows[r] >= 0;
    for (int i = r; i < TREE_LEAF * dim; i += TREE_LEAF) {
        const int rr = i / dim;
        const int32_t src = rows[rr];
        pts[i] = src >= 0 ? data[static_cast<size_t>(src) * dim + (i - rr * dim)] : 0.0f;
    }
    __syncthreads();
    float top[KM];   // the KM smallest squared distances so far, ascending (KM >= k)
#pragma unroll
    for (int i = 0; i < KM; ++i) top[i] = CUDART_INF_F;
    float kth2 = 0.0f;
    if (valid[r]) {
        const float* x = pts + r * dim;
        for (int j = 0; j < TREE_LEAF; ++j) {
            if (j == r || !valid[j]) continue;
            const float* y = pts + j * dim;
            float d2 = 0.0f;
            for (int d = 0; d < dim; ++d) {
                const float v = x[d] - y[d];
                d2 = fmaf(v, v, d2);
            }
            if (!(d2 < top[KM - 1])) continue;   // not among the KM nearest so far
#pragma unroll
            for (int i = KM - 1; i > 0; --i) top[i] = d2 < top[i - 1] ? top[i - 1] : fminf(top[i], d2);
            top[0] = fminf(top[0], d2);
        }
#pragma unroll
        for (int i = 0; i < KM; ++i)
            if (i == k - 1) kth2 = top[i];
    }
    for (int o = 16; o > 0; o >>= 1) kth2 = fmaxf(kth2, __shfl_xor_sync(0xffffffffu, kth2, o));
    if ((r & 31) == 0) red[r >> 5] = kth2;
    __syncthreads();
    if (r == 0) {
        float m = red[0];
        for (int w = 1; w < TREE_LEAF / 32; ++w) m = fmaxf(m, red[w]);
        kth_out[g] = sqrtf(m * D2_HIGH) * D2_HIGH;
    }
}

// One warp per LIST_QB consecutive query tiles b (each with tiles
// [t0_b, t0_b + nt_b) of its instance); a centroid read serves all of them.
// Radius rho_b of b's k-neighbourhoods: every query q of b has at least k
// other points within rho_b --
//   kth_b (tile_kth_kernel)              if b holds k + 1 or more points,
//   2 R_b                                likewise (never below kth_b),
//   R_b + |c_b - c_w| + R_w (upper)      for any tile w with k + 1 or more points,
// the smallest of these (infinite if none applies).  Tile t is needed unless
// |c_b - c_t| - R_b - R_t > rho_b.  The needed tiles are written in ascending
// order from lists[slot[b]] (room for nt_b entries), their number to counts[b].
constexpr int LIST_WARPS = 8;
constexpr int LIST_QB = 8;
constexpr int MAX_TREE_DIM = 128;
__global__ void __launch_bounds__(32 * LIST_WARPS)
    tile_lists_kernel(int32_t nq, const int32_t* __restrict__ q_tile0, const int32_t* __restrict__ q_ntiles,
                      const float* __restrict__ ct, int32_t ntiles, const float* __restrict__ tr,
                      const int32_t* __restrict__ tcount, const float* __restrict__ tkth, int32_t dim, int32_t k,
                      bool prune, const int64_t* __restrict__ slot, int32_t* __restrict__ counts,
                      int32_t* __restrict__ lists) {
    __shared__ float cbs[LIST_WARPS][MAX_TREE_DIM][LIST_QB];   // [d][q]: one 32-byte read per d
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int32_t b0 = (blockIdx.x * LIST_WARPS + wib) * LIST_QB;
    if (b0 >= nq) return;   // whole warps
    const int nb = min(LIST_QB, nq - b0);
    float (*cb)[LIST_QB] = cbs[wib];
    for (int e = lane; e < dim * LIST_QB; e += 32) {
        const int d = e / LIST_QB, q = e - d * LIST_QB;
        cb[d][q] = q < nb ? ct[static_cast<size_t>(d) * ntiles + b0 + q] : 0.0f;
    }
    __syncwarp();
    int32_t t0[LIST_QB], t1[LIST_QB];
    float rb[LIST_QB], rho[LIST_QB];
    int32_t lo = INT32_MAX, hi = 0;
#pragma unroll
    for (int q = 0; q < LIST_QB; ++q) {
        const int32_t b = b0 + q;
        t0[q] = q < nb ? q_tile0[b] : 0;
        t1[q] = q < nb ? t0[q] + q_ntiles[b] : 0;
        rb[q] = q < nb ? tr[b] : 0.0f;
        rho[q] = (q < nb && tcount[b] >= k + 1) ? (tkth ? fminf(2.0f * rb[q], tkth[b]) : 2.0f * rb[q]) : CUDART_INF_F;
        if (q < nb) {
            lo = min(lo, t0[q]);
            hi = max(hi, t1[q]);
        }
    }
    // squared centroid distances from every query tile of the group to tile t
    auto dist2 = [&](int32_t t, float (&s)[LIST_QB]) {
#pragma unroll
        for (int q = 0; q < LIST_QB; ++q) s[q] = 0.0f;
        for (int d = 0; d < dim; ++d) {
            const float c = ct[static_cast<size_t>(d) * ntiles + t];
#pragma unroll
            for (int q = 0; q < LIST_QB; ++q) {
                const float v = cb[d][q] - c;
                s[q] = fmaf(v, v, s[q]);
            }
        }
    };
    if (prune) {
        for (int32_t base = lo; base < hi; base += 32) {
            const int32_t w = base + lane;
            if (w < hi && tcount[w] >= k + 1) {
                float s[LIST_QB];
                dist2(w, s);
#pragma unroll
                for (int q = 0; q < LIST_QB; ++q) {
                    if (w >= t0[q] && w < t1[q] && w != b0 + q) {
                        const float dist_up = sqrtf(s[q] * D2_HIGH) * D2_HIGH;
                        rho[q] = fminf(rho[q], __fadd_ru(__fadd_ru(rb[q], dist_up), tr[w]));
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < LIST_QB; ++q)
            for (int o = 16; o > 0; o >>= 1) rho[q] = fminf(rho[q], __shfl_xor_sync(0xffffffffu, rho[q], o));
    }
    int32_t total[LIST_QB];
#pragma unroll
    for (int q = 0; q < LIST_QB; ++q) total[q] = 0;
    for (int32_t base = lo; base < hi; base += 32) {
        const int32_t t = base + lane;
        float s[LIST_QB];
        if (t < hi) dist2(t, s);
        const float rt = t < hi ? tr[t] : 0.0f;
#pragma unroll
        for (int q = 0; q < LIST_QB; ++q) {
            bool need = false;
            if (q < nb && t >= t0[q] && t < t1[q]) {
                // needed unless |c_b - c_t| > rho + R_b + R_t (all non-negative: compare squares)
                const bool all = !prune || !(rho[q] < CUDART_INF_F);
                const float reach = rho[q] + rb[q] + rt;
                need = all || t == b0 + q || s[q] * D2_LOW <= reach * reach * D2_HIGH;
            }
            const unsigned m = __ballot_sync(0xffffffffu, need);
            if (need) lists[slot[b0 + q] + total[q] + __popc(m & ((1u << lane) - 1u))] = t;
            total[q] += __popc(m);
        }
    }
    if (lane < nb) {
#pragma unroll
        for (int q = 0; q < LIST_QB; ++q)
            if (q == lane) counts[b0 + q] = total[q];
    }
}

}  // namespace

void knn_tree_order(const float* data, int32_t dim, const std::vector<int32_t>& inst, bool tree, KnnTiles& out,
                    cudaStream_t s) {
    const int ninst = static_cast<int>(inst.size()) - 1;
    const int32_t n = inst[ninst];
    DevArray<int32_t> perm(n, s);
    DevArray<unsigned long long> keys(n, s), keys2(n, s);
    iota_kernel<<<grid_for(n, 256), 256, 0, s>>>(perm.get(), n);
    UMAPB_LAUNCH_CHECK();

    // Segments over positions of perm, the instances to begin with.  A segment
    // starts at a tile boundary of its run (a stretch of operand rows between
    // two hard cuts, padded to whole tiles); soft cuts keep tile alignment,
    // hard cuts (at a wide gap of the projections, as between two clusters)
    // start a new run, so that no tile spans the gap.
    struct Seg {
        int32_t start, len;
        bool hard_end;
    };
    std::vector<Seg> seg(ninst);
    for (int i = 0; i < ninst; ++i) seg[i] = {inst[i], inst[i + 1] - inst[i], true};
    uint64_t h = 0x9E3779B97F4A7C15ull;
    auto next = [&h]() {   // splitmix64: the choice of the direction's first point
        uint64_t z = (h += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    DevArray<int32_t> vals(n, s), vals2(n, s);
    for (int level = 0; tree && level < 64; ++level) {
        const int nseg = static_cast<int>(seg.size());
        // the segments split at this level, concatenated (active_segment)
        std::vector<int32_t> ast, aoff(1, 0), aa;
        std::vector<int64_t> moff(1, 0);
        for (int g = 0; g < nseg; ++g) {
            if (seg[g].len <= TREE_LEAF) continue;
            ast.push_back(seg[g].start);
            aa.push_back(seg[g].start + static_cast<int32_t>(next() % static_cast<uint64_t>(seg[g].len)));
            aoff.push_back(aoff.back() + seg[g].len);
            moff.push_back(moff.back() + (gap_window_last(seg[g].len) - gap_window_first(seg[g].len) + 1));
        }
        const int nact = static_cast<int>(ast.size());
        if (nact == 0) break;
        const int64_t total = aoff[nact];
        DevArray<int32_t> d_ast(nact, s), d_aoff(nact + 1, s), d_aa(nact, s);
        DevArray<int64_t> d_moff(nact + 1, s);
        DevArray<unsigned long long> d_far(nact, s), d_best(nact, s);
        DevArray<float> d_lo(nact, s), d_hi(nact, s);
        UMAPB_CUDA(cudaMemcpyAsync(d_ast.get(), ast.data(), nact * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(d_aoff.get(), aoff.data(), (nact + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(d_aa.get(), aa.data(), nact * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(d_moff.get(), moff.data(), (nact + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
        // direction: from a to the segment's point farthest from a
        d_far.zero(s);
        far_point_kernel<<<grid_for(static_cast<size_t>(total), 256), 256, 0, s>>>(
            data, dim, perm.get(), nact, d_aoff.get(), d_ast.get(), d_aa.get(), total, d_far.get());
        UMAPB_LAUNCH_CHECK();
        rp_keys_kernel<<<grid_for(static_cast<size_t>(total), 256), 256, 0, s>>>(
            data, dim, perm.get(), nact, d_aoff.get(), d_ast.get(), d_aa.get(), d_far.get(), total, keys.get(),
            vals.get());
        UMAPB_LAUNCH_CHECK();
        int seg_bits = 1;
        while ((1 << seg_bits) < nact) ++seg_bits;
        size_t tb = 0;
        UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.get(), keys2.get(), vals.get(), vals2.get(),
                                                   static_cast<int>(total), 0, 32 + seg_bits, s));
        {
            DevArray<unsigned char> temp(tb, s);
            UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(temp.get(), tb, keys.get(), keys2.get(), vals.get(), vals2.get(),
                                                       static_cast<int>(total), 0, 32 + seg_bits, s));
        }
        scatter_active_kernel<<<grid_for(static_cast<size_t>(total), 256), 256, 0, s>>>(nact, d_aoff.get(), d_ast.get(),
                                                                                      total, vals2.get(), perm.get());
        UMAPB_LAUNCH_CHECK();
        // widest gap of the sorted projections in each active segment's window,
        // on the sorted items (segment j: items [aoff[j], aoff[j + 1]))
        d_best.zero(s);
        widest_gap_kernel<<<grid_for(static_cast<size_t>(moff[nact]), 256), 256, 0, s>>>(
            keys2.get(), nact, d_aoff.get(), d_aoff.get() + 1, d_moff.get(), moff[nact], d_best.get());
        UMAPB_LAUNCH_CHECK();
        middle_spread_kernel<<<grid_for(nact, 128), 128, 0, s>>>(keys2.get(), nact, d_aoff.get(), d_aoff.get() + 1,
                                                                 d_lo.get(), d_hi.get());
        UMAPB_LAUNCH_CHECK();
        std::vector<unsigned long long> best(nact);
        std::vector<float> klo(nact), khi(nact), spread(nact);
        UMAPB_CUDA(cudaMemcpyAsync(best.data(), d_best.get(), nact * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaMemcpyAsync(klo.data(), d_lo.get(), nact * sizeof(float), cudaMemcpyDeviceToHost, s));
        UMAPB_CUDA(cudaMemcpyAsync(khi.data(), d_hi.get(), nact * sizeof(float), cudaMemcpyDeviceToHost, s));
        UMAPB_SYNC(s);   // also: the host tables above are the copies' sources
        std::vector<int32_t> gpos(nact);
        std::vector<float> gap(nact);
        for (int j = 0; j < nact; ++j) {
            const uint32_t gbits = static_cast<uint32_t>(best[j] >> 32);
            std::memcpy(&gap[j], &gbits, sizeof(float));
            gpos[j] = static_cast<int32_t>(0xffffffffu - static_cast<uint32_t>(best[j] & 0xffffffffu));
            spread[j] = khi[j] - klo[j];
        }
        std::vector<Seg> nseg2;
        nseg2.reserve(2 * nseg);
        int j = 0;
        for (int g = 0; g < nseg; ++g) {
            const Seg x = seg[g];
            if (x.len <= TREE_LEAF) {
                nseg2.push_back(x);
                continue;
            }
            // a gap far wider than the typical spacing of the middle half
            const float typical = spread[j] / (0.5f * x.len);
            const bool hard = x.len >= 2 * TREE_LEAF && gpos[j] > 0 && gap[j] > GAP_FACTOR * typical &&
                              gap[j] > 0.0f;
            if (hard) {
                const int32_t left = gpos[j];
                nseg2.push_back({x.start, left, true});
                nseg2.push_back({x.start + left, x.len - left, x.hard_end});
            } else {
                const int32_t tiles = (x.len + TREE_LEAF - 1) / TREE_LEAF;
                const int32_t left = (tiles + 1) / 2 * TREE_LEAF;
                nseg2.push_back({x.start, left, false});
                nseg2.push_back({x.start + left, x.len - left, x.hard_end});
            }
            ++j;
        }
        seg.swap(nseg2);
    }

    // runs (segments up to a hard end) laid out one after another, each padded to whole tiles
    std::vector<int32_t> run_src, run_len, run_dst;
    out.pad_start.assign(ninst + 1, 0);
    int32_t pos = 0, inst_i = 0;
    {
        int32_t rs = -1, rl = 0;
        for (const Seg& x : seg) {
            if (rs < 0) rs = x.start;
            rl += x.len;
            if (x.hard_end) {
                while (inst_i < ninst && inst[inst_i] == rs) out.pad_start[inst_i++] = pos;   // an instance's first run
                run_src.push_back(rs);
                run_len.push_back(rl);
                run_dst.push_back(pos);
                pos += ((rl + TREE_LEAF - 1) / TREE_LEAF) * TREE_LEAF;
                rs = -1;
                rl = 0;
            }
        }
    }
    out.pad_start[ninst] = pos;
    out.n_pad = std::max(pos, TREE_LEAF);
    const int nrun = static_cast<int>(run_src.size());
    DevArray<int32_t> d_rs(nrun, s), d_rl(nrun, s), d_rd(nrun, s);
    UMAPB_CUDA(cudaMemcpyAsync(d_rs.get(), run_src.data(), nrun * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(d_rl.get(), run_len.data(), nrun * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(d_rd.get(), run_dst.data(), nrun * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    out.row_map.allocate(out.n_pad, s);
    UMAPB_CUDA(cudaMemsetAsync(out.row_map.get(), 0xff, out.n_pad * sizeof(int32_t), s));   // -1: padding
    place_runs_kernel<<<grid_for(n, 256), 256, 0, s>>>(perm.get(), nrun, d_rs.get(), d_rl.get(), d_rd.get(), n,
                                                       out.row_map.get());
    UMAPB_LAUNCH_CHECK();
    UMAPB_SYNC(s);   // host vectors above
}

void knn_tile_tasks(const float* data, int32_t dim, const KnnTiles& t, const std::vector<int32_t>& inst, int qt,
                    int32_t k, bool prune, KnnTasks& out, cudaStream_t s, KnnShard shard) {
    const int ninst = static_cast<int>(inst.size()) - 1;
    const int32_t ntiles = t.n_pad / TREE_LEAF;
    // every tile's instance tile range; CTAs of qt tiles within an instance
    std::vector<int32_t> tile0(ntiles, 0), ntl(ntiles, 0);
    std::vector<int4> tasks;
    for (int i = 0; i < ninst; ++i) {
        const int32_t a = t.pad_start[i] / TREE_LEAF, b = t.pad_start[i + 1] / TREE_LEAF;
        for (int32_t x = a; x < b; ++x) {
            tile0[x] = a;
            ntl[x] = b - a;
        }
        for (int32_t x = a; x < b; x += qt) tasks.push_back(make_int4(x * TREE_LEAF, x, std::min(qt, b - x), 0));
    }
    require(dim <= MAX_TREE_DIM, "tile pruning supports up to 128 dimensions");
    DevArray<float> tcen(static_cast<size_t>(ntiles) * dim, s), tcen_t(static_cast<size_t>(ntiles) * dim, s),
        trad(ntiles, s);
    DevArray<int32_t> tcnt(ntiles, s);
    group_bounds_kernel<<<ntiles, 128, 0, s>>>(data, dim, t.row_map.get(), TREE_LEAF, tcen.get(), trad.get(), tcnt.get(),
                                               tcen_t.get(), ntiles);
    UMAPB_LAUNCH_CHECK();
    DevArray<int32_t> d_tile0(ntiles, s), d_ntl(ntiles, s);
    out.qlist_len.allocate(ntiles, s);
    out.qlist_off.allocate(ntiles, s);
    // list slots: every query tile has room for all tiles of its instance
    std::vector<int64_t> ho(ntiles + 1, 0);
    for (int32_t x = 0; x < ntiles; ++x) ho[x + 1] = ho[x] + ntl[x];
    out.tile_list.allocate(std::max<int64_t>(ho[ntiles], 1), s);
    UMAPB_CUDA(cudaMemcpyAsync(d_tile0.get(), tile0.data(), ntiles * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(d_ntl.get(), ntl.data(), ntiles * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(out.qlist_off.get(), ho.data(), ntiles * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    const unsigned warps_grid = static_cast<unsigned>((ntiles + LIST_WARPS * LIST_QB - 1) / (LIST_WARPS * LIST_QB));
    DevArray<float> tkth;
    if (prune && k <= KTH_MAX) {
        tkth.allocate(ntiles, s);
        const size_t smem = sizeof(float) * TREE_LEAF * dim;   // dim <= MAX_TREE_DIM: 64 KB at most
        // the insertion list as short as k allows
        auto launch = [&](auto km) {
            constexpr int KM = decltype(km)::value;
            static std::once_flag once;
            std::call_once(once, [] {
                UMAPB_CUDA(cudaFuncSetAttribute(tile_kth_kernel<KM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                static_cast<int>(sizeof(float) * TREE_LEAF * MAX_TREE_DIM)));
            });
            tile_kth_kernel<KM><<<ntiles, TREE_LEAF, smem, s>>>(data, dim, t.row_map.get(), tcnt.get(), k, tkth.get());
        };
        if (k <= 16) launch(std::integral_constant<int, 16>());
        else if (k <= 24) launch(std::integral_constant<int, 24>());
        else launch(std::integral_constant<int, KTH_MAX>());
        UMAPB_LAUNCH_CHECK();
    }
    tile_lists_kernel<<<warps_grid, 32 * LIST_WARPS, 0, s>>>(ntiles, d_tile0.get(), d_ntl.get(), tcen_t.get(), ntiles,
                                                             trad.get(), tcnt.get(), tkth.get(), dim, k, prune,
                                                             out.qlist_off.get(), out.qlist_len.get(),
                                                             out.tile_list.get());
    UMAPB_LAUNCH_CHECK();
    std::vector<int32_t> hc(ntiles);
    UMAPB_CUDA(cudaMemcpyAsync(hc.data(), out.qlist_len.get(), ntiles * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    out.total_tiles = 0;
    for (int32_t x = 0; x < ntiles; ++x) out.total_tiles += hc[x];
    // CTAs with the most reference tiles first (they are scheduled first and finish together)
    std::vector<int64_t> work(tasks.size());
    for (size_t j = 0; j < tasks.size(); ++j) {
        int64_t w = 0;
        for (int x = 0; x < tasks[j].z; ++x) w += hc[tasks[j].y + x];
        work[j] = w;
    }
    if (shard.count > 1) {
        // this shard's tasks: a contiguous range (tree order) holding an equal
        // share of the work, cut where the running total crosses index / count
        int64_t total = 0;
        for (int64_t w : work) total += w;
        std::vector<int4> kept;
        std::vector<int64_t> kept_work;
        int64_t run = 0;
        for (size_t j = 0; j < tasks.size(); ++j) {
            const int64_t mid = run + work[j] / 2;   // the task belongs to the shard its midpoint falls in
            const int32_t owner = total > 0 ? static_cast<int32_t>(std::min<int64_t>(shard.count - 1, mid * shard.count / total))
                                            : static_cast<int32_t>(j * shard.count / std::max<size_t>(tasks.size(), 1));
            run += work[j];
            if (owner == shard.index) {
                kept.push_back(tasks[j]);
                kept_work.push_back(work[j]);
            }
        }
        tasks.swap(kept);
        work.swap(kept_work);
        out.total_tiles = 0;
        for (int64_t w : work) out.total_tiles += w;
    }
    std::vector<int32_t> order(tasks.size());
    for (size_t j = 0; j < order.size(); ++j) order[j] = static_cast<int32_t>(j);
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return work[x] > work[y]; });
    std::vector<int4> sorted(tasks.size());
    for (size_t j = 0; j < order.size(); ++j) sorted[j] = tasks[order[j]];
    out.count = static_cast<int32_t>(sorted.size());
    out.host_tasks = sorted;
    out.tasks.allocate(std::max<size_t>(sorted.size(), 1), s);
    UMAPB_CUDA(cudaMemcpyAsync(out.tasks.get(), sorted.data(), sorted.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
    UMAPB_SYNC(s);   // host vectors above
}

namespace {
__global__ void task_rows_flag_kernel(const int4* __restrict__ tasks, const int32_t* __restrict__ row_map,
                                      int32_t n_pad, uint8_t* __restrict__ flag) {
    const int4 tk = tasks[blockIdx.x];
    const int32_t end = min(n_pad, tk.x + TREE_LEAF * tk.z);
    for (int32_t r = tk.x + threadIdx.x; r < end; r += blockDim.x) {
        const int32_t d = row_map[r];
        if (d >= 0) flag[d] = 1;
    }
}
}  // namespace

namespace {
struct IsRow {
    __device__ __forceinline__ bool operator()(int32_t r) const { return r >= 0; }
};
}  // namespace

void knn_tree_rows(const KnnTiles& t, int32_t n, DevArray<int32_t>& rows, cudaStream_t s) {
    rows.allocate(std::max<int32_t>(n, 1), s);
    DevArray<int32_t> d_count(1, s);
    size_t tb = 0;
    UMAPB_CUDA(cub::DeviceSelect::If(nullptr, tb, t.row_map.get(), rows.get(), d_count.get(), t.n_pad, IsRow(), s));
    DevArray<unsigned char> temp(tb, s);
    UMAPB_CUDA(cub::DeviceSelect::If(temp.get(), tb, t.row_map.get(), rows.get(), d_count.get(), t.n_pad, IsRow(), s));
}

void knn_task_rows(const KnnTiles& t, const KnnTasks& tk, int32_t n, DevArray<int32_t>& rows, int32_t& count,
                   cudaStream_t s) {
    DevArray<uint8_t> flag(n, s);
    UMAPB_CUDA(cudaMemsetAsync(flag.get(), 0, static_cast<size_t>(n), s));
    if (tk.count > 0) {
        task_rows_flag_kernel<<<static_cast<unsigned>(tk.count), 128, 0, s>>>(tk.tasks.get(), t.row_map.get(), t.n_pad,
                                                                             flag.get());
        UMAPB_LAUNCH_CHECK();
    }
    rows.allocate(std::max<int32_t>(n, 1), s);
    DevArray<int32_t> d_count(1, s);
    thrust::counting_iterator<int32_t> it(0);
    size_t tb = 0;
    UMAPB_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, it, flag.get(), rows.get(), d_count.get(), n, s));
    DevArray<unsigned char> temp(tb, s);
    UMAPB_CUDA(cub::DeviceSelect::Flagged(temp.get(), tb, it, flag.get(), rows.get(), d_count.get(), n, s));
    UMAPB_CUDA(cudaMemcpyAsync(&count, d_count.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
}

}  // namespace umapb
