// optimize_layout on the device (include/umappp/optimize_layout.hpp:116-185).
//
// Schedule.  Which edges fire in an epoch, and how many negative samples each
// draws, depends only on the per-edge schedule (epochs_per_sample and the two
// running epoch_of_next_* values), never on the layout.  So the schedule is
// advanced by itself, in the reference's exact Float_ arithmetic (this file is
// compiled with -fmad=false), and its firing events are written out for a
// window of epochs as compact per-epoch lists of (head, tail, #negatives) in
// the edges' CSR order.  Two passes over the edges build a window: one counts
// events per (epoch, block), an exclusive scan places them, the second
// writes them.  The window is sized to a device-memory budget (the whole run
// fits at a million observations on a 180 GB part).
//
// Epoch kernel.  One thread per firing event: the attractive step moves the
// head (in registers) and the tail (vector atomic add); then the head takes
// its negative samples in sequence, as the reference does, and its total
// displacement is added atomically.  Negative samples come from Philox4x32-10
// keyed by the seed with counter (head, tail, epoch, block), so they do not
// depend on the launch shape or on how epochs are split across run() calls.
// Updates of different events race (Hogwild-style), as in any parallel SGD of
// this kind; per-event arithmetic follows optimize_layout.hpp:145-179.
#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <cstdlib>
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

#include "stages.cuh"

namespace umapb {

namespace {

constexpr int SCHED_BLOCK = 256;
constexpr int MAX_WINDOW = 512;
// Default cap on a window's event buffers (events, negative counts, segment
// starts): 4 GiB, or 1/16 of the device's memory if that is less.  Every
// window re-reads the whole edge state (count and write passes), so fewer,
// larger windows cost less -- a million-point run needs ~18 B x 7.2M events
// per epoch, 32 epochs to a 4 GiB window, 7 windows for 200 epochs -- while
// one buffer for the whole run (~26 GB) would crowd the data.  The buffers are
// kept from window to window and, through the workspace cache, across runs.
size_t window_bytes() {
    static const size_t v = [] {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            cudaGetLastError();
            total_b = 0;
        }
        const size_t cap = size_t(4) << 30;
        return total_b ? std::min(cap, total_b / 16) : (size_t(1) << 30);
    }();
    return v;
}
// UMAPB_SGD_WINDOW_BYTES caps the window buffers (read at every build; 0 or
// unset: window_bytes()).
size_t window_bytes_override() {
    const char* e = std::getenv("UMAPB_SGD_WINDOW_BYTES");
    return e ? static_cast<size_t>(std::strtoull(e, nullptr, 10)) : 0;
}
constexpr int MAX_GENERIC_DIM = 64;

template <typename T>
struct FloatLimits;
template <>
struct FloatLimits<float> {
    static __device__ __forceinline__ float epsilon() { return FLT_EPSILON; }
};
template <>
struct FloatLimits<double> {
    static __device__ __forceinline__ double epsilon() { return DBL_EPSILON; }
};

// One schedule step of edge j at 'epoch' (optimize_layout.hpp:141-143,160-161,178-179).
template <typename T>
__device__ __forceinline__ bool schedule_step(T epoch, T eps, T epns, T& enext, T& enneg, int& nneg) {
    if (enext > epoch) return false;
    nneg = static_cast<int>((epoch - enneg) / epns);
    enext += eps;
    enneg += static_cast<T>(nneg) * epns;
    return true;
}

template <typename T>
__global__ void __launch_bounds__(SCHED_BLOCK) sched_count_kernel(int64_t nnz, const T* __restrict__ eps,
                                                                  const T* __restrict__ enext_in,
                                                                  const T* __restrict__ enneg_in, T rate, int e0, int W,
                                                                  int64_t* __restrict__ counts) {
    const int64_t j = static_cast<int64_t>(blockIdx.x) * SCHED_BLOCK + threadIdx.x;
    const bool valid = j < nnz;
    const T ep = valid ? eps[j] : T(1);
    const T epns = ep / rate;
    T en = valid ? enext_in[j] : T(0);
    T enn = valid ? enneg_in[j] : T(0);
    for (int w = 0; w < W; ++w) {
        int nn = 0;
        const bool fire = valid && schedule_step<T>(static_cast<T>(e0 + w), ep, epns, en, enn, nn);
        const int c = __syncthreads_count(fire);
        if (threadIdx.x == 0) counts[static_cast<int64_t>(w) * gridDim.x + blockIdx.x] = c;
    }
}

template <typename T>
__global__ void __launch_bounds__(SCHED_BLOCK) sched_write_kernel(int64_t nnz, const int32_t* __restrict__ heads,
                                                                  const int32_t* __restrict__ targets,
                                                                  const T* __restrict__ eps, T* __restrict__ enext_st,
                                                                  T* __restrict__ enneg_st, T rate, int e0, int W,
                                                                  const int64_t* __restrict__ offsets,
                                                                  int2* __restrict__ ht, uint16_t* __restrict__ nneg_out,
                                                                  int* __restrict__ status) {
    __shared__ int warp_counts[SCHED_BLOCK / 32];
    const int64_t j = static_cast<int64_t>(blockIdx.x) * SCHED_BLOCK + threadIdx.x;
    const bool valid = j < nnz;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const T ep = valid ? eps[j] : T(1);
    const T epns = ep / rate;
    T en = valid ? enext_st[j] : T(0);
    T enn = valid ? enneg_st[j] : T(0);
    const int2 pair = valid ? make_int2(heads[j], targets[j]) : make_int2(0, 0);
    for (int w = 0; w < W; ++w) {
        int nn = 0;
        const bool fire = valid && schedule_step<T>(static_cast<T>(e0 + w), ep, epns, en, enn, nn);
        const unsigned mask = __ballot_sync(0xffffffffu, fire);
        if (lane == 0) warp_counts[warp] = __popc(mask);
        __syncthreads();
        if (fire) {
            int before = 0;
            for (int q = 0; q < warp; ++q) before += warp_counts[q];
            const int64_t pos = offsets[static_cast<int64_t>(w) * gridDim.x + blockIdx.x] + before +
                                __popc(mask & ((1u << lane) - 1u));
            ht[pos] = pair;
            if (nn < 0) nn = 0;   // a negative count draws nothing, as in the reference's loop
            if (nn > 65535) {
                atomicExch(status, DEV_BAD_INPUT);
                nn = 65535;
            }
            nneg_out[pos] = static_cast<uint16_t>(nn);
        }
        __syncthreads();
    }
    if (valid) {
        enext_st[j] = en;
        enneg_st[j] = enn;
    }
}

// Advances the schedule state by W epochs without recording events.
template <typename T>
__global__ void sched_advance_kernel(int64_t nnz, const T* __restrict__ eps, T* __restrict__ enext, T* __restrict__ enneg,
                                     T rate, int e0, int W) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < nnz; j += int64_t(gridDim.x) * blockDim.x) {
        const T ep = eps[j];
        const T epns = ep / rate;
        T en = enext[j], enn = enneg[j];
        for (int w = 0; w < W; ++w) {
            int nn;
            schedule_step<T>(static_cast<T>(e0 + w), ep, epns, en, enn, nn);
        }
        enext[j] = en;
        enneg[j] = enn;
    }
}

// Per-epoch totals of firing edges and negative samples.
template <typename T>
__global__ void __launch_bounds__(SCHED_BLOCK) sched_totals_kernel(int64_t nnz, const T* __restrict__ eps,
                                                                   T* __restrict__ enext, T* __restrict__ enneg, T rate,
                                                                   int e0, int W,
                                                                   unsigned long long* __restrict__ totals) {
    typedef cub::BlockReduce<unsigned long long, SCHED_BLOCK> Reduce;
    __shared__ typename Reduce::TempStorage tmp;
    const int64_t j = static_cast<int64_t>(blockIdx.x) * SCHED_BLOCK + threadIdx.x;
    const bool valid = j < nnz;
    const T ep = valid ? eps[j] : T(1);
    const T epns = ep / rate;
    T en = valid ? enext[j] : T(0);
    T enn = valid ? enneg[j] : T(0);
    for (int w = 0; w < W; ++w) {
        int nn = 0;
        const bool fire = valid && schedule_step<T>(static_cast<T>(e0 + w), ep, epns, en, enn, nn);
        const int c = __syncthreads_count(fire);
        const unsigned long long negs = Reduce(tmp).Sum(fire && nn > 0 ? static_cast<unsigned long long>(nn) : 0ull);
        if (threadIdx.x == 0) {
            atomicAdd(&totals[2 * w], static_cast<unsigned long long>(c));
            atomicAdd(&totals[2 * w + 1], negs);
        }
        __syncthreads();
    }
    if (valid) {
        enext[j] = en;
        enneg[j] = enn;
    }
}

__global__ void gather_epoch_starts_kernel(const int64_t* __restrict__ offsets, int64_t nblocks, int W,
                                           int64_t total_last, int64_t* __restrict__ starts) {
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w <= W; w += gridDim.x * blockDim.x) {
        starts[w] = (w < W) ? offsets[static_cast<int64_t>(w) * nblocks] : total_last;
    }
}

// ---------------------------------------------------------- epoch kernel --

template <typename T>
struct SgdParams {
    T a, b;
    T neg2ab;      // -2ab
    T gamma2b;     // 2 gamma b
    T alpha;
    uint32_t k0, k1;
    uint32_t epoch;
    int32_t n;
    // Independent instances laid out one after another (batched runs):
    // instance i owns observations [inst_start[i], inst_start[i + 1]) and
    // draws its negative samples there.  num_inst <= 1: one instance of n.
    const int32_t* inst_start;
    int32_t num_inst;
};

// Observation range [base, base + size) of the instance that owns h.
template <typename T>
__device__ __forceinline__ void instance_range(int32_t h, const SgdParams<T>& p, int32_t& base, uint32_t& size) {
    if (p.num_inst <= 1) {
        base = 0;
        size = static_cast<uint32_t>(p.n);
        return;
    }
    int lo = 0, hi = p.num_inst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (p.inst_start[mid] <= h) lo = mid; else hi = mid - 1;
    }
    base = p.inst_start[lo];
    size = static_cast<uint32_t>(p.inst_start[lo + 1] - base);
}


// Counter-based negative-sample stream of one event.
struct NegStream {
    uint32_t c0, c1, c2, c3, k0, k1;
    Philox4 buf;
    int used;
    __device__ __forceinline__ NegStream(uint32_t h, uint32_t t, uint32_t epoch, uint32_t key0, uint32_t key1)
        : c0(h), c1(t), c2(epoch), c3(0), k0(key0), k1(key1), used(4) {}
    __device__ __forceinline__ uint32_t next() {
        if (used == 4) {
            buf = philox4x32_10(c0, c1, c2, c3++, k0, k1);
            used = 0;
        }
        return buf.v[used++];
    }
    // Exactly uniform integer in [0, n) (Lemire, "Fast random integer generation
    // in an interval", ACM TOMACS 2019): multiply-shift with rejection.
    __device__ __forceinline__ int32_t bounded(uint32_t n) {
        uint64_t m = static_cast<uint64_t>(next()) * n;
        uint32_t l = static_cast<uint32_t>(m);
        if (l < n) {
            const uint32_t thr = (0u - n) % n;
            while (l < thr) {
                m = static_cast<uint64_t>(next()) * n;
                l = static_cast<uint32_t>(m);
            }
        }
        return static_cast<int32_t>(m >> 32);
    }
};

template <typename T>
__device__ __forceinline__ T clamp4(T g) {
    g = (g < T(-4)) ? T(-4) : g;
    return (T(4) < g) ? T(4) : g;
}

// FP32 layouts use the hardware-approximated power (__powf, an exp2 of b log2 x
// in the special-function unit): the step is stochastic and clamped, and a
// few-ulp error in d^(2b) is far below the noise of negative sampling.
__device__ __forceinline__ float pow_b(float x, float b) { return __powf(x, b); }
__device__ __forceinline__ double pow_b(double x, double b) { return pow(x, b); }

// Attractive coefficient, optimize_layout.hpp:147-149.
template <typename T>
__device__ __forceinline__ T attract_coef(T d2, const SgdParams<T>& p) {
    const T pd2b = pow_b(d2, p.b);
    return (p.neg2ab * pd2b) / (d2 * (p.a * pd2b + T(1)));
}

// Repulsive coefficient, optimize_layout.hpp:170-171.
template <typename T>
__device__ __forceinline__ T repulse_coef(T d2, const SgdParams<T>& p) {
    return p.gamma2b / ((T(0.001) + d2) * (p.a * pow_b(d2, p.b) + T(1)));
}

// FP32 coefficients for the 2-d kernel with fused multiply-adds and the
// approximate divide (__fdividef, 2 ulp): the step is stochastic and
// clamped, and the per-event dependency chain is what bounds the kernel.
__device__ __forceinline__ float attract_coef_fast(float d2, const SgdParams<float>& p) {
    const float pd2b = pow_b(d2, p.b);
    return __fdividef(p.neg2ab * pd2b, d2 * __fmaf_rn(p.a, pd2b, 1.0f));
}

__device__ __forceinline__ float repulse_coef_fast(float d2, const SgdParams<float>& p) {
    return __fdividef(p.gamma2b, (0.001f + d2) * __fmaf_rn(p.a, pow_b(d2, p.b), 1.0f));
}

// The same coefficients with libm's powf and IEEE division (a kernel variant
// that measures what the approximations above cost in layout quality).
__device__ __forceinline__ float attract_coef_precise(float d2, const SgdParams<float>& p) {
    const float pd2b = powf(d2, p.b);
    return (p.neg2ab * pd2b) / (d2 * (p.a * pd2b + 1.0f));
}
__device__ __forceinline__ float repulse_coef_precise(float d2, const SgdParams<float>& p) {
    return p.gamma2b / ((0.001f + d2) * (p.a * powf(d2, p.b) + 1.0f));
}

template <typename T>
__device__ __forceinline__ T floor_eps(T d2) {
    const T e = FloatLimits<T>::epsilon();
    return (e < d2) ? d2 : e;
}

// Segments: the firing events of one head in one epoch are contiguous in the
// event list (it follows the edges' CSR order).  A segment is a run of at most
// seg_max events of one head: a head's run is cut every seg_max events from
// its first, which bounds the longest sequential chain (hub heads have
// hundreds of edges), and at the boundaries of the 2048-event ranges that the
// segment passes work on.  Segments partition the window's events in order:
// seg_pos[s] is the first event of segment s, seg_pos[S] = the event total,
// and the segments of epoch w are [seg_first[w], seg_first[w + 1]).  Built
// without atomics by a count / scan / write over fixed event ranges, so the
// list is deterministic.  Counting the cuts from the run's own start (rather
// than from fixed positions of the epoch) leaves a head with up to seg_max
// events in one segment: at 1M points that is ~1.1 segments per firing head
// instead of ~1.75, and the epochs run ~20 % faster.
//
// seg_max: the segments of one head run concurrently from the same starting
// position, so a split hub takes its steps from a stale copy of itself.  When
// an epoch holds fewer events than the epoch kernel keeps threads resident,
// every segment is in flight at once and splitting buys no parallelism, so
// heads are cut only every SEG_MAX_FEW events (at 2,000 points this lifts the
// mean trustworthiness by about 0.002, to that of the serial order).  Larger
// epochs use SEG_MAX, which keeps the kernel's rounds balanced (at 1M points,
// 64-event segments made the SGD about 1.6x slower and moved the edge
// cross-entropy further from the reference's).
constexpr int SEG_MAX = 8;
constexpr int SEG_MAX_FEW = 64;
constexpr int SEG_BLOCK = 256;
constexpr int SEG_ITEMS = 8;    // events per thread in the segment passes

// Segment flags of the events [base + SEG_ITEMS t, + SEG_ITEMS) of one block
// (blocked: each thread takes consecutive events): a run starts at the block's
// first event, at an epoch's first event and where the head changes; the
// block-wide maximum scan of run starts gives each event its run's first
// event, and an event starts a segment when its distance to that is a
// multiple of seg_max.
template <class Scan>
__device__ __forceinline__ void segment_flags(int64_t base, int64_t total, const int2* __restrict__ ht,
                                              const int64_t* __restrict__ starts, int W, int seg_max,
                                              typename Scan::TempStorage& tmp, int (&flag)[SEG_ITEMS]) {
    int run[SEG_ITEMS];
#pragma unroll
    for (int i = 0; i < SEG_ITEMS; ++i) {
        const int local = threadIdx.x * SEG_ITEMS + i;
        const int64_t e = base + local;
        bool first = local == 0;
        if (!first && e < total) {
            first = ht[e - 1].x != ht[e].x;
            if (!first) {
                int lo = 0, hi = W - 1;   // epoch of e: the last w with starts[w] <= e
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (starts[mid] <= e) lo = mid; else hi = mid - 1;
                }
                first = starts[lo] == e;
            }
        }
        run[i] = first ? local : 0;
    }
    Scan(tmp).InclusiveScan(run, run, cub::Max());
#pragma unroll
    for (int i = 0; i < SEG_ITEMS; ++i) {
        const int local = threadIdx.x * SEG_ITEMS + i;
        flag[i] = (base + local < total && (local - run[i]) % seg_max == 0) ? 1 : 0;
    }
}

__global__ void __launch_bounds__(SEG_BLOCK) seg_count_kernel(int64_t total, const int2* __restrict__ ht,
                                                              const int64_t* __restrict__ starts, int W, int seg_max,
                                                              int64_t* __restrict__ block_counts) {
    typedef cub::BlockScan<int, SEG_BLOCK> Scan;
    typedef cub::BlockReduce<int, SEG_BLOCK> Reduce;
    __shared__ union {
        typename Scan::TempStorage scan;
        typename Reduce::TempStorage reduce;
    } tmp;
    const int64_t base = static_cast<int64_t>(blockIdx.x) * SEG_BLOCK * SEG_ITEMS;
    int flag[SEG_ITEMS];
    segment_flags<Scan>(base, total, ht, starts, W, seg_max, tmp.scan, flag);
    int c = 0;
#pragma unroll
    for (int i = 0; i < SEG_ITEMS; ++i) c += flag[i];
    __syncthreads();   // the scan's storage is reused
    const int sum = Reduce(tmp.reduce).Sum(c);
    if (threadIdx.x == 0) block_counts[blockIdx.x] = sum;
}

// Writes segment starts in event order: block b covers events
// [b * SEG_BLOCK * SEG_ITEMS, ...).
__global__ void __launch_bounds__(SEG_BLOCK) seg_write_kernel(int64_t total, const int2* __restrict__ ht,
                                                              const int64_t* __restrict__ starts, int W, int seg_max,
                                                              const int64_t* __restrict__ block_offsets,
                                                              int64_t* __restrict__ seg_pos) {
    typedef cub::BlockScan<int, SEG_BLOCK> Scan;
    __shared__ typename Scan::TempStorage tmp;
    const int64_t base = static_cast<int64_t>(blockIdx.x) * SEG_BLOCK * SEG_ITEMS;
    int flag[SEG_ITEMS], prefix[SEG_ITEMS];
    segment_flags<Scan>(base, total, ht, starts, W, seg_max, tmp, flag);
    __syncthreads();   // the scan's storage is reused
    int sum = 0;
    Scan(tmp).ExclusiveSum(flag, prefix, sum);
    const int64_t out = block_offsets[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SEG_ITEMS; ++i)
        if (flag[i]) seg_pos[out + prefix[i]] = base + threadIdx.x * SEG_ITEMS + i;
}

// Head slices: within every epoch the segments are ordered by the slice of
// their head -- slice b of P holds the heads [base + b size / P, base + (b+1)
// size / P) of each instance [base, base + size) -- so that launches over
// consecutive slot ranges take the slices in order.  seg_bucket_* count and
// scatter each segment to order[seg_first[w] + rank] (rank among its epoch's
// segments by slice; within a slice in no particular order).
__device__ __forceinline__ void segment_slice(int64_t s, const int64_t* __restrict__ seg_pos,
                                              const int2* __restrict__ ht, const int64_t* __restrict__ seg_first, int W,
                                              const int32_t* __restrict__ inst_start, int32_t num_inst, int32_t n,
                                              int P, int& w, int& b) {
    int lo = 0, hi = W - 1;   // epoch: last w with seg_first[w] <= s
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (seg_first[mid] <= s) lo = mid; else hi = mid - 1;
    }
    w = lo;
    const int32_t h = ht[seg_pos[s]].x;
    int32_t base = 0, size = n;
    if (num_inst > 1) {
        int a = 0, c = num_inst - 1;
        while (a < c) {
            const int mid = (a + c + 1) >> 1;
            if (inst_start[mid] <= h) a = mid; else c = mid - 1;
        }
        base = inst_start[a];
        size = inst_start[a + 1] - base;
    }
    b = static_cast<int>((static_cast<int64_t>(h - base) * P) / size);
}

// One instance: the slices of an epoch are consecutive segment ranges (heads
// ascend within an epoch); off[w][b] = first segment whose head is at least
// b n / P (binary search), off[w][P] = the epoch's end.
__global__ void slice_bounds_kernel(const int64_t* __restrict__ seg_pos, const int2* __restrict__ ht,
                                    const int64_t* __restrict__ seg_first, int W, int32_t n, int P,
                                    int64_t* __restrict__ off) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * (P + 1)) return;
    const int w = i / (P + 1), b = i % (P + 1);
    int64_t lo = seg_first[w], hi = seg_first[w + 1];
    if (b == P) {
        off[i] = hi;
        return;
    }
    const int64_t key = (static_cast<int64_t>(b) * n + P - 1) / P;   // ceil(b n / P)
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (ht[seg_pos[mid]].x < key) lo = mid + 1; else hi = mid;
    }
    off[i] = lo;
}

// Several instances: block-local histograms of (epoch, slice), one global
// atomic per block and bin to reserve ranks, then the block's segments are
// scattered within their reservations.
constexpr int SLICE_BLOCK = 256;
constexpr int SLICE_MAX_BINS = 4096;
__global__ void __launch_bounds__(SLICE_BLOCK)
    seg_bucket_kernel(int64_t nseg, const int64_t* __restrict__ seg_pos, const int2* __restrict__ ht,
                      const int64_t* __restrict__ seg_first, int W, const int32_t* __restrict__ inst_start,
                      int32_t num_inst, int32_t n, int P, int* __restrict__ counts, int* __restrict__ cursor,
                      int32_t* __restrict__ order) {
    __shared__ int bins[SLICE_MAX_BINS];
    const int nb = W * P;
    for (int i = threadIdx.x; i < nb; i += SLICE_BLOCK) bins[i] = 0;
    __syncthreads();
    const int64_t s = blockIdx.x * int64_t(SLICE_BLOCK) + threadIdx.x;
    int w = 0, b = 0, local = -1;
    if (s < nseg) {
        segment_slice(s, seg_pos, ht, seg_first, W, inst_start, num_inst, n, P, w, b);
        local = atomicAdd(&bins[w * P + b], 1);
    }
    __syncthreads();
    if (!order) {   // counting pass
        for (int i = threadIdx.x; i < nb; i += SLICE_BLOCK)
            if (bins[i]) atomicAdd(&counts[i], bins[i]);
        return;
    }
    for (int i = threadIdx.x; i < nb; i += SLICE_BLOCK)
        if (bins[i]) bins[i] = atomicAdd(&cursor[i], bins[i]);   // base of this block's ranks in bin i
    __syncthreads();
    if (s < nseg) order[seg_first[w] + bins[w * P + b] + local] = static_cast<int32_t>(s - seg_first[w]);
}

// seg_first[w] = index of the first segment of epoch w (lower bound of starts[w] in seg_pos).
__global__ void seg_first_kernel(const int64_t* __restrict__ seg_pos, int64_t nseg, const int64_t* __restrict__ starts,
                                 int W, int64_t* __restrict__ seg_first) {
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w <= W; w += gridDim.x * blockDim.x) {
        const int64_t key = starts[w];
        int64_t lo = 0, hi = nseg;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (seg_pos[mid] < key) lo = mid + 1; else hi = mid;
        }
        seg_first[w] = lo;
    }
}

// Negative samples are gathered NB at a time: their indices do not depend on
// the layout, so all loads of a batch (and the tail's) are in flight together,
// and the head then takes the updates in sequence.  NB and the minimum number
// of resident 256-thread blocks (which caps the registers per thread) trade
// gathers in flight per thread against resident threads; the variants are
// listed in SGD_2D_VARIANTS.

// One thread per segment: the head's firing edges are processed in CSR order
// with the head kept in registers, each edge's attractive step (head and tail)
// followed by its negative samples -- the per-row sequence of
// optimize_layout.hpp:136-180.  The tail moves by a vector atomic; the head's
// total displacement is added once at the end.
// Head publication modes of the 2-d kernel: HEAD_AT_END adds the head's total
// displacement once at the segment's end; HEAD_PER_EVENT adds each event's
// displacement as soon as it is computed; HEAD_FRESH also re-reads the head
// at the start of every event (seeing the pulls of other threads' attractive
// steps, which move it as a tail), so no event works from a copy of the head
// older than one event.
enum HeadMode { HEAD_AT_END = 0, HEAD_PER_EVENT = 1, HEAD_FRESH = 2 };
// PAIR: an undirected edge fires in both directions in the same epochs (the
// union gives both directions the same weight, hence the same schedule); the
// event whose head is the smaller index takes both attractive steps, the
// second one (head and tail exchanged) from the positions the first one left,
// and the event of the larger head takes only its negative samples.

// Coherent device-scope load: ordered after this thread's own earlier atomic
// adds to the same address.
__device__ __forceinline__ float2 ld_relaxed_f2(const float2* p) {
    float2 v;
    asm volatile("ld.relaxed.gpu.global.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p) : "memory");
    return v;
}

template <int NB, int MINB, bool PRECISE = false, int MODE = HEAD_AT_END, bool PAIR = false>
__global__ void __launch_bounds__(256, MINB) sgd_epoch_2d_f32(const int32_t* __restrict__ order, int64_t base,
                                                        int64_t slot0, int64_t slot1,
                                                        const int64_t* __restrict__ seg_pos,
                                                        const int2* __restrict__ ht, const uint16_t* __restrict__ nneg,
                                                        float2* __restrict__ Y, SgdParams<float> p) {
    for (int64_t slot = slot0 + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; slot < slot1;
         slot += int64_t(gridDim.x) * blockDim.x) {
        const int64_t s = order ? base + order[slot] : slot;
        const int64_t e0 = seg_pos[s], e1 = seg_pos[s + 1];
        const int32_t h = ht[e0].x;
        int32_t nbase;
        uint32_t nsize;
        instance_range(h, p, nbase, nsize);
        const float2 y0 = MODE == HEAD_FRESH ? ld_relaxed_f2(&Y[h]) : __ldcg(&Y[h]);
        float hx = y0.x, hy = y0.y;
        for (int64_t e = e0; e < e1; ++e) {
            const int2 pr = ht[e];
            int remaining = nneg[e];
            const float2 yt = __ldcg(&Y[pr.y]);
            if (MODE == HEAD_FRESH && e != e0) {
                const float2 yh = ld_relaxed_f2(&Y[h]);
                hx = yh.x;
                hy = yh.y;
            }
            const float ex = hx, ey = hy;   // head at the event's start
            NegStream rng(static_cast<uint32_t>(h), static_cast<uint32_t>(pr.y), p.epoch, p.k0, p.k1);
            bool attract = true;
            do {
                // issue this batch's gathers, then apply the updates in order
                const int m = remaining < NB ? remaining : NB;
                int32_t ks[NB];
                float2 yk[NB];
#pragma unroll
                for (int i = 0; i < NB; ++i) {
                    if (i < m) {
                        ks[i] = nbase + rng.bounded(nsize);
                        yk[i] = __ldcg(&Y[ks[i]]);
                    }
                }
                if (attract && (!PAIR || pr.y > h)) {
                    const float dx = hx - yt.x, dy = hy - yt.y;
                    const float d2 = floor_eps(__fmaf_rn(dx, dx, dy * dy));
                    const float cf = PRECISE ? attract_coef_precise(d2, p) : attract_coef_fast(d2, p);
                    float gx = p.alpha * clamp4(cf * dx);
                    float gy = p.alpha * clamp4(cf * dy);
                    hx += gx;
                    hy += gy;
                    if (PAIR) {   // the reverse edge's step: head = tail, from the moved positions
                        const float tx = yt.x - gx, ty = yt.y - gy;
                        const float ex2 = tx - hx, ey2 = ty - hy;
                        const float e2 = floor_eps(__fmaf_rn(ex2, ex2, ey2 * ey2));
                        const float cf2 = PRECISE ? attract_coef_precise(e2, p) : attract_coef_fast(e2, p);
                        const float g2x = p.alpha * clamp4(cf2 * ex2);
                        const float g2y = p.alpha * clamp4(cf2 * ey2);
                        hx -= g2x;
                        hy -= g2y;
                        gx -= g2x;   // the tail's total move is -(g - g2)
                        gy -= g2y;
                    }
                    atomicAdd(&Y[pr.y], make_float2(-gx, -gy));
                }
                attract = false;
#pragma unroll
                for (int i = 0; i < NB; ++i) {
                    if (i < m && ks[i] != h) {
                        const float dx = hx - yk[i].x, dy = hy - yk[i].y;
                        const float d2 = floor_eps(__fmaf_rn(dx, dx, dy * dy));
                        const float cf = PRECISE ? repulse_coef_precise(d2, p) : repulse_coef_fast(d2, p);
                        hx = __fmaf_rn(p.alpha, clamp4(cf * dx), hx);
                        hy = __fmaf_rn(p.alpha, clamp4(cf * dy), hy);
                    }
                }
                remaining -= m;
            } while (remaining > 0);
            if (MODE != HEAD_AT_END) atomicAdd(&Y[h], make_float2(hx - ex, hy - ey));
        }
        if (MODE == HEAD_AT_END) atomicAdd(&Y[h], make_float2(hx - y0.x, hy - y0.y));
    }
}

struct Sgd2dVariant {
    void (*kernel)(const int32_t*, int64_t, int64_t, int64_t, const int64_t*, const int2*, const uint16_t*, float2*,
                   SgdParams<float>);
    int neg_batch, min_blocks;
};
const Sgd2dVariant SGD_2D_VARIANTS[] = {
    {sgd_epoch_2d_f32<12, 1>, 12, 1},   // 80 registers: 3 blocks of 256 per SM
    {sgd_epoch_2d_f32<12, 4>, 12, 4},   // 64 registers
    {sgd_epoch_2d_f32<8, 4>, 8, 4},     // default
    {sgd_epoch_2d_f32<6, 6>, 6, 6},     // 40 registers
    {sgd_epoch_2d_f32<8, 4, true>, 8, 4},   // libm powf and IEEE division (precision check)
    {sgd_epoch_2d_f32<8, 4, false, HEAD_PER_EVENT>, 8, 4},
    {sgd_epoch_2d_f32<8, 4, false, HEAD_FRESH>, 8, 4},
    {sgd_epoch_2d_f32<8, 4, false, HEAD_AT_END, true>, 8, 4},   // 7: PAIR
    {sgd_epoch_2d_f32<8, 4, false, HEAD_FRESH, true>, 8, 4},    // 8: PAIR, fresh head
};
constexpr int NUM_SGD_2D_VARIANTS = sizeof(SGD_2D_VARIANTS) / sizeof(SGD_2D_VARIANTS[0]);
constexpr int NUM_TUNED_VARIANTS = 4;   // the tuner picks among launch shapes of one arithmetic

// Resident blocks per SM of variant v at 'block' threads (occupancy query, cached).
int sgd_2d_resident(int v, int block) {
    static int cache[NUM_SGD_2D_VARIANTS][2] = {};
    const int bi = block == 128 ? 0 : 1;
    if (cache[v][bi] == 0) {
        int r = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, SGD_2D_VARIANTS[v].kernel, block, 0) != cudaSuccess || r < 1) {
            cudaGetLastError();
            r = 1;
        }
        cache[v][bi] = r;
    }
    return cache[v][bi];
}

// Any dimension (up to MAX_GENERIC_DIM) and either precision; same per-segment order.
template <typename T>
__global__ void __launch_bounds__(128) sgd_epoch_generic(const int32_t* __restrict__ order, int64_t base,
                                                         int64_t slot0, int64_t slot1,
                                                         const int64_t* __restrict__ seg_pos,
                                                         const int2* __restrict__ ht, const uint16_t* __restrict__ nneg,
                                                         T* __restrict__ Y, int dim, SgdParams<T> p) {
    T head[MAX_GENERIC_DIM], orig[MAX_GENERIC_DIM];
    for (int64_t slot = slot0 + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; slot < slot1;
         slot += int64_t(gridDim.x) * blockDim.x) {
        const int64_t s = order ? base + order[slot] : slot;
        const int64_t e0 = seg_pos[s], e1 = seg_pos[s + 1];
        const int32_t h = ht[e0].x;
        int32_t nbase;
        uint32_t nsize;
        instance_range(h, p, nbase, nsize);
        T* yh = Y + static_cast<size_t>(h) * dim;
        for (int d = 0; d < dim; ++d) head[d] = orig[d] = __ldcg(yh + d);
        for (int64_t e = e0; e < e1; ++e) {
            const int2 pr = ht[e];
            const int nn = nneg[e];
            T* yt = Y + static_cast<size_t>(pr.y) * dim;
            T d2 = 0;
            for (int d = 0; d < dim; ++d) {
                const T diff = head[d] - __ldcg(yt + d);
                d2 += diff * diff;
            }
            {
                const T c = attract_coef(floor_eps(d2), p);
                for (int d = 0; d < dim; ++d) {
                    const T g = p.alpha * clamp4(c * (head[d] - __ldcg(yt + d)));
                    head[d] += g;
                    atomicAdd(yt + d, -g);
                }
            }
            if (nn > 0) {
                NegStream rng(static_cast<uint32_t>(h), static_cast<uint32_t>(pr.y), p.epoch, p.k0, p.k1);
                for (int q = 0; q < nn; ++q) {
                    const int32_t k = nbase + rng.bounded(nsize);
                    if (k == h) continue;
                    const T* yk = Y + static_cast<size_t>(k) * dim;
                    T dd2 = 0;
                    for (int d = 0; d < dim; ++d) {
                        const T diff = head[d] - __ldcg(yk + d);
                        dd2 += diff * diff;
                    }
                    const T c = repulse_coef(floor_eps(dd2), p);
                    for (int d = 0; d < dim; ++d) head[d] += p.alpha * clamp4(c * (head[d] - __ldcg(yk + d)));
                }
            }
        }
        for (int d = 0; d < dim; ++d) atomicAdd(yh + d, head[d] - orig[d]);
    }
}

// UMAPB_CHECK_SCHEDULE=1: verify every event window (SgdEngine::verify_window).
bool check_schedule() {
    const char* e = std::getenv("UMAPB_CHECK_SCHEDULE");
    return e && *e && *e != '0';
}

// Grid size as a multiple of the resident blocks (UMAPB_SGD_GRID_MULTIPLE, default 1).
int grid_multiple() {
    static const int v = [] {
        const char* e = std::getenv("UMAPB_SGD_GRID_MULTIPLE");
        const int x = e ? std::atoi(e) : 0;
        return (x >= 1 && x <= 64) ? x : 1;
    }();
    return v;
}

int sm_count() {
    static int count = 0;
    if (count == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        if (count <= 0) count = 148;
    }
    return count;
}

}  // namespace

template <typename T>
void SgdEngine<T>::setup(const DeviceEpochs<T>* ep, cudaStream_t s, int base_epoch) {
    ep_ = ep;
    base_epoch_ = base_epoch;
    require(static_cast<double>(ep->negative_sample_rate) <= 30000.0,
            "negative_sample_rate above 30000 is not supported");
    enext_.allocate(ep->nnz, s);
    enneg_.allocate(ep->nnz, s);
    if (ep->nnz) {
        UMAPB_CUDA(cudaMemcpyAsync(enext_.get(), ep->enext0.get(), ep->nnz * sizeof(T), cudaMemcpyDeviceToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(enneg_.get(), ep->enneg0.get(), ep->nnz * sizeof(T), cudaMemcpyDeviceToDevice, s));
    }
    state_epoch_ = base_epoch_;
    for (Window& w : win_) {
        w.begin = w.end = base_epoch_;
        w.ht.release();
        w.nneg.release();
        w.epoch_offsets.release();
        w.host_epoch_offsets.clear();
    }
}

template <typename T>
void SgdEngine<T>::state_at(int epoch, T* enext, T* enneg, cudaStream_t s) {
    const int64_t nnz = ep_->nnz;
    if (nnz == 0) return;
    require(epoch >= base_epoch_, "schedule state requested before its starting epoch");
    UMAPB_CUDA(cudaMemcpyAsync(enext, ep_->enext0.get(), nnz * sizeof(T), cudaMemcpyDeviceToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(enneg, ep_->enneg0.get(), nnz * sizeof(T), cudaMemcpyDeviceToDevice, s));
    if (epoch > base_epoch_) {
        sched_advance_kernel<T><<<grid_for(nnz, 256), 256, 0, s>>>(nnz, ep_->eps.get(), enext, enneg,
                                                                   ep_->negative_sample_rate, base_epoch_,
                                                                   epoch - base_epoch_);
        UMAPB_LAUNCH_CHECK();
    }
}

template <typename T>
void SgdEngine<T>::build_window(Window& win, int first, int last_wanted, cudaStream_t s) {
    const int64_t nnz = ep_->nnz;
    win.begin = win.end = first;   // empty until complete
    // bring the state to 'first'
    if (state_epoch_ != first) {
        if (state_epoch_ > first) {
            state_at(first, enext_.get(), enneg_.get(), s);
        } else if (nnz) {
            sched_advance_kernel<T><<<grid_for(nnz, 256), 256, 0, s>>>(nnz, ep_->eps.get(), enext_.get(), enneg_.get(),
                                                                       ep_->negative_sample_rate, state_epoch_,
                                                                       first - state_epoch_);
            UMAPB_LAUNCH_CHECK();
        }
        state_epoch_ = first;
    }
    const int W = std::min(last_wanted - first, MAX_WINDOW);
    const int64_t nblocks = std::max<int64_t>((nnz + SCHED_BLOCK - 1) / SCHED_BLOCK, 1);
    require(nblocks <= INT32_MAX, "too many edges", UMAPB_ERR_OVERFLOW);
    const int64_t ncount = nblocks * W;
    DevArray<int64_t> counts(ncount, s), offsets(ncount, s);
    if (nnz) {
        sched_count_kernel<T><<<static_cast<unsigned>(nblocks), SCHED_BLOCK, 0, s>>>(
            nnz, ep_->eps.get(), enext_.get(), enneg_.get(), ep_->negative_sample_rate, first, W, counts.get());
        UMAPB_LAUNCH_CHECK();
    } else {
        counts.zero(s);
    }
    {
        size_t tb = 0;
        UMAPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, counts.get(), offsets.get(), ncount, s));
        DevArray<unsigned char> temp(tb, s);
        UMAPB_CUDA(cub::DeviceScan::ExclusiveSum(temp.get(), tb, counts.get(), offsets.get(), ncount, s));
    }
    int64_t last_off = 0, last_cnt = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&last_off, offsets.get() + ncount - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaMemcpyAsync(&last_cnt, counts.get() + ncount - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    DevArray<int64_t> starts(W + 1, s);
    gather_epoch_starts_kernel<<<grid_for(W + 1, 128), 128, 0, s>>>(offsets.get(), nblocks, W, last_off + last_cnt,
                                                                     starts.get());
    UMAPB_LAUNCH_CHECK();
    std::vector<int64_t> h(W + 1);
    UMAPB_CUDA(cudaMemcpyAsync(h.data(), starts.get(), (W + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);

    // fit the window to the memory budget
    const size_t env_budget = window_bytes_override();
    const size_t budget = event_budget_bytes ? event_budget_bytes : env_budget ? env_budget : window_bytes();
    // event record + (at most) one segment start per event
    const size_t per_event = sizeof(int2) + sizeof(uint16_t) + sizeof(int64_t) + sizeof(int32_t);
    int Wk = W;
    while (Wk > 1 && static_cast<size_t>(h[Wk]) * per_event > budget) --Wk;
    const int64_t events = h[Wk];

    // the window buffers are kept across windows (and runs) and only grow
    win.ht.reserve(events, s);
    win.nneg.reserve(events, s);
    DevArray<int> status(1, s);
    status.zero(s);
    if (nnz) {
        sched_write_kernel<T><<<static_cast<unsigned>(nblocks), SCHED_BLOCK, 0, s>>>(
            nnz, ep_->heads.get(), ep_->targets.get(), ep_->eps.get(), enext_.get(), enneg_.get(),
            ep_->negative_sample_rate, first, Wk, offsets.get(), win.ht.get(), win.nneg.get(), status.get());
        UMAPB_LAUNCH_CHECK();
    }
    win.epoch_offsets.allocate(Wk + 1, s);
    UMAPB_CUDA(cudaMemcpyAsync(win.epoch_offsets.get(), h.data(), (Wk + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));

    // head segments of every epoch in the window (count, scan, write, per-epoch first segment)
    const int64_t resident_threads =
        static_cast<int64_t>(sm_count()) * sgd_2d_resident(variant_, block_) * block_;
    int seg_max = events < resident_threads * Wk ? SEG_MAX_FEW : SEG_MAX;
    if (const char* e = std::getenv("UMAPB_SGD_SEG_MAX")) {   // override of the segment cap
        const int x = std::atoi(e);
        if (x >= 1 && x <= 4096) seg_max = x;
    }
    win.seg_max = seg_max;
    const int64_t seg_blocks = std::max<int64_t>((events + SEG_BLOCK * SEG_ITEMS - 1) / (SEG_BLOCK * SEG_ITEMS), 1);
    DevArray<int64_t> bcount(seg_blocks + 1, s), boff(seg_blocks + 1, s);
    bcount.zero(s);
    if (events > 0) {
        seg_count_kernel<<<static_cast<unsigned>(seg_blocks), SEG_BLOCK, 0, s>>>(events, win.ht.get(), win.epoch_offsets.get(),
                                                                               Wk, seg_max, bcount.get());
        UMAPB_LAUNCH_CHECK();
    }
    {
        size_t tb = 0;
        UMAPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, bcount.get(), boff.get(), seg_blocks + 1, s));
        DevArray<unsigned char> temp(tb, s);
        UMAPB_CUDA(cub::DeviceScan::ExclusiveSum(temp.get(), tb, bcount.get(), boff.get(), seg_blocks + 1, s));
    }
    int64_t nseg = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&nseg, boff.get() + seg_blocks, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    win.seg_pos.reserve(nseg + 1, s);
    UMAPB_CUDA(cudaMemcpyAsync(win.seg_pos.get() + nseg, &events, sizeof(int64_t), cudaMemcpyHostToDevice, s));
    if (events > 0) {
        seg_write_kernel<<<static_cast<unsigned>(seg_blocks), SEG_BLOCK, 0, s>>>(events, win.ht.get(), win.epoch_offsets.get(),
                                                                               Wk, seg_max, boff.get(), win.seg_pos.get());
        UMAPB_LAUNCH_CHECK();
    }
    win.seg_first.allocate(Wk + 1, s);
    seg_first_kernel<<<grid_for(Wk + 1, 128), 128, 0, s>>>(win.seg_pos.get(), nseg, win.epoch_offsets.get(), Wk,
                                                            win.seg_first.get());
    UMAPB_LAUNCH_CHECK();
    win.host_seg_first.resize(Wk + 1);
    UMAPB_CUDA(cudaMemcpyAsync(win.host_seg_first.data(), win.seg_first.get(), (Wk + 1) * sizeof(int64_t),
                               cudaMemcpyDeviceToHost, s));

    win.host_epoch_offsets.assign(h.begin(), h.begin() + Wk + 1);
    build_slices(win, nseg, Wk, s);
    int st = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&st, status.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    require(st == DEV_OK, "a negative-sample count exceeded 65535");
    if (check_schedule()) verify_window(win, first, Wk, s);
    win.begin = first;
    win.end = first + Wk;
    state_epoch_ = win.end;
}

// Autotuner: times the 2-d epoch kernel with each candidate launch shape on a
// scratch copy of the layout (one epoch of the current window), keeps the
// fastest, and remembers it per size class (log2 of the epoch's events).
template <typename T>
template <class Launch>
void SgdEngine<T>::tune(T* Y, int num_dim, int first, int stop, const Window& win, Launch& launch, cudaStream_t s) {
    static std::mutex mu;
    static std::map<int, std::pair<int, int>> cache;   // size class -> (block, variant)
    int w = -1;
    for (int e = (first + stop) / 2; e < stop && w < 0; ++e) {
        const int ww = e - win.begin;
        if (win.host_seg_first[ww + 1] > win.host_seg_first[ww]) w = ww;
    }
    if (w < 0) return;
    const int64_t events = win.host_epoch_offsets[w + 1] - win.host_epoch_offsets[w];
    int key = 0;
    while ((int64_t(1) << key) < events) ++key;
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            block_ = it->second.first;
            variant_ = it->second.second;
            return;
        }
    }
    const size_t total = static_cast<size_t>(ep_->n) * num_dim;
    DevArray<T> scratch(total, s);
    cudaEvent_t a = event_get(), b = event_get();
    float best = 1e30f;
    for (int v = 0; v < NUM_TUNED_VARIANTS; ++v) {
        for (int blk : {128, 256}) {
            UMAPB_CUDA(cudaMemcpyAsync(scratch.get(), Y, total * sizeof(T), cudaMemcpyDeviceToDevice, s));
            UMAPB_CUDA(cudaEventRecord(a, s));
            launch(scratch.get(), win, win.begin + w, w, blk, v);
            UMAPB_CUDA(cudaEventRecord(b, s));
            UMAPB_CUDA(cudaEventSynchronize(b));
            float t = 0;
            UMAPB_CUDA(cudaEventElapsedTime(&t, a, b));
            if (t < best) {
                best = t;
                block_ = blk;
                variant_ = v;
            }
        }
    }
    event_put(a);
    event_put(b);
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = std::make_pair(block_, variant_);
}

template <typename T>
void SgdEngine<T>::run(T* Y, int num_dim, int first, int last, double a, double b, double gamma, double learning_rate,
                       uint64_t seed, cudaStream_t caller, float* ms_schedule, float* ms_sgd) {
    if (ms_schedule) *ms_schedule = 0;
    if (ms_sgd) *ms_sgd = 0;
    if (last <= first) return;
    require(num_dim >= 1 && num_dim <= MAX_GENERIC_DIM, "num_dim must be between 1 and 64");
    const int total = ep_->total_epochs;
    SgdParams<T> p;
    p.a = static_cast<T>(a);
    p.b = static_cast<T>(b);
    p.neg2ab = T(-2) * p.a * p.b;
    p.gamma2b = T(2) * static_cast<T>(gamma) * p.b;
    p.k0 = static_cast<uint32_t>(seed) ^ RNG_NEGATIVE;
    p.k1 = static_cast<uint32_t>(seed >> 32);
    p.n = ep_->n;
    p.inst_start = inst_start_;
    p.num_inst = num_inst_;
    const T lr = static_cast<T>(learning_rate);
    const int blocks_gen = sm_count() * 8;
    cudaStream_t s = nullptr;   // the epochs' stream (below)

    // One epoch launch of window slot w on Yp, with the 2-d kernel's block size and variant.
    auto launch = [&](T* Yp, const Window& win, int e_abs, int w, int block, int variant) {
        const T epoch_t = static_cast<T>(e_abs);
        // alpha = lr * (1 - epoch / num_epochs) in the reference's types (optimize_layout.hpp:132-133)
        p.alpha = static_cast<T>(static_cast<double>(lr) * (1.0 - static_cast<double>(epoch_t / static_cast<T>(total))));
        p.epoch = static_cast<uint32_t>(e_abs);
        const int64_t nsegs = win.host_seg_first[w + 1] - win.host_seg_first[w];
        if (nsegs == 0) return;
        const bool use_2d = std::is_same<T, float>::value && num_dim == 2;
        const int blk = use_2d ? block : 128;
        const int resident = use_2d ? sm_count() * sgd_2d_resident(variant, block) : blocks_gen;
        unsigned cap_blocks = static_cast<unsigned>(resident * grid_multiple());
        if (const char* e = std::getenv("UMAPB_SGD_MAX_BLOCKS")) {   // cap on the blocks in flight
            const int x = std::atoi(e);
            if (x >= 1) cap_blocks = std::min<unsigned>(cap_blocks, static_cast<unsigned>(x));
        }
        const unsigned g = grid_for(nsegs, blk, cap_blocks);
        // Parallel updates read positions that the serial order would already
        // have moved; when every event of an epoch is in flight at once the
        // layouts come out measurably tighter (lower edge cross-entropy) than
        // the reference's.  The epoch's segments are therefore ordered by head
        // slice (P = min_phases slices of each instance, build_window), and
        // taken in that order: by the grid-stride loop's rounds when the epoch
        // holds several rounds of segments, and by consecutive launches over
        // slot ranges (L of them, slices split evenly) to make up the rest.
        const int P = win.buckets;
        const int64_t threads = static_cast<int64_t>(std::min<int64_t>(g, resident)) * blk;
        const int64_t rounds = (nsegs + threads - 1) / threads;
        int L = static_cast<int>(std::min<int64_t>(P, std::max<int64_t>(1, (P + rounds - 1) / rounds)));
        if (const char* he = std::getenv("UMAPB_SGD_HARD_SLICES")) {   // one launch per slice
            if (*he && *he != '0') L = P;
        }
        const int64_t* off = win.host_bucket_off.data() + static_cast<size_t>(w) * (P + 1);
        const int32_t* order = win.ordered ? win.seg_order.get() : nullptr;
        for (int l = 0; l < L; ++l) {
            const int64_t slot0 = off[(P * l) / L], slot1 = off[(P * (l + 1)) / L];
            if (slot1 <= slot0) continue;
            const unsigned gl = grid_for(slot1 - slot0, blk, cap_blocks);
            if (use_2d) {
                if constexpr (std::is_same<T, float>::value) {
                    SGD_2D_VARIANTS[variant].kernel<<<gl, blk, 0, s>>>(order, win.host_seg_first[w], slot0, slot1,
                                                                       win.seg_pos.get(), win.ht.get(), win.nneg.get(),
                                                                       reinterpret_cast<float2*>(Yp), p);
                }
            } else {
                sgd_epoch_generic<T><<<gl, 128, 0, s>>>(order, win.host_seg_first[w], slot0, slot1, win.seg_pos.get(),
                                                        win.ht.get(), win.nneg.get(), Yp, num_dim, p);
            }
            UMAPB_LAUNCH_CHECK();
        }
    };

    // The epochs run on a high-priority stream s and windows are built on a
    // default-priority stream s2 while the epochs of the previous window run:
    // the host enqueues a window's epochs, then builds the next window (the
    // build synchronises only its own stream), so the GPU runs both at once,
    // the block scheduler giving the epochs first claim on the SMs.  A window
    // buffer is rebuilt only after the epochs that read it have finished (host
    // wait on its 'done' event), which also orders the release of any buffer
    // the rebuild grows.  Both streams start after the caller's work on
    // 'caller' (layout, schedule state); the host waits for the last epoch.
    s = stream_get(true);
    cudaStream_t s2 = stream_get();
    cudaEvent_t start = event_get(), finish = event_get();
    cudaEvent_t done[2] = {event_get(), event_get()};
    bool pending[2] = {false, false};
    std::vector<cudaEvent_t> marks;            // per window: SGD begin, SGD end (on s)
    std::vector<cudaGraphExec_t> execs;
    auto cleanup = [&] {
        for (auto x : execs) cudaGraphExecDestroy(x);
        for (auto x : marks) event_put(x);
        event_put(start);
        event_put(finish);
        event_put(done[0]);
        event_put(done[1]);
        stream_put(s2);
        stream_put(s);
    };
    try {
        UMAPB_CUDA(cudaEventRecord(start, caller));
        UMAPB_CUDA(cudaStreamWaitEvent(s, start, 0));
        UMAPB_CUDA(cudaStreamWaitEvent(s2, start, 0));
        auto find = [&](int e) {
            for (int i = 0; i < 2; ++i)
                if (win_[i].begin <= e && e < win_[i].end) return i;
            return -1;
        };
        auto build_into = [&](int i, int e) {
            if (pending[i]) {
                UMAPB_CUDA(cudaEventSynchronize(done[i]));
                pending[i] = false;
            }
            build_window(win_[i], e, last, s2);
        };
        int e = first;
        int cur = find(e);
        if (cur < 0) build_into(cur = 0, e);
        while (true) {
            const Window& win = win_[cur];
            const int stop = std::min(last, win.end);
            if (autotune && std::is_same<T, float>::value && num_dim == 2) tune(Y, num_dim, e, stop, win, launch, s);
            marks.push_back(event_get());
            marks.push_back(event_get());
            UMAPB_CUDA(cudaEventRecord(marks[marks.size() - 2], s));
            if (use_graphs) {
                // this window's epoch launches as one CUDA graph
                cudaGraph_t graph = nullptr;
                UMAPB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                for (int x = e; x < stop; ++x) launch(Y, win, x, x - win.begin, block_, variant_);
                UMAPB_CUDA(cudaStreamEndCapture(s, &graph));
                cudaGraphExec_t exec = nullptr;
                const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
                cudaGraphDestroy(graph);
                if (ie != cudaSuccess) cuda_fail(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
                execs.push_back(exec);
                UMAPB_CUDA(cudaGraphLaunch(exec, s));
            } else {
                for (int x = e; x < stop; ++x) launch(Y, win, x, x - win.begin, block_, variant_);
            }
            UMAPB_CUDA(cudaEventRecord(marks.back(), s));
            UMAPB_CUDA(cudaEventRecord(done[cur], s));
            pending[cur] = true;
            e = stop;
            if (e >= last) break;
            int next = find(e);
            if (next < 0) build_into(next = 1 - cur, e);
            cur = next;
        }
        UMAPB_CUDA(cudaEventRecord(finish, s));
        UMAPB_CUDA(cudaEventSynchronize(finish));
        // SGD: the windows' epoch spans on s; schedule: the rest of the span
        // from the start to the last epoch (the first build and any wait for
        // a build that the epochs did not hide)
        float sgd_ms = 0, all_ms = 0;
        for (size_t i = 0; i < marks.size(); i += 2) {
            float t = 0;
            UMAPB_CUDA(cudaEventElapsedTime(&t, marks[i], marks[i + 1]));
            sgd_ms += t;
        }
        UMAPB_CUDA(cudaEventElapsedTime(&all_ms, start, finish));
        if (ms_schedule) *ms_schedule = std::max(0.0f, all_ms - sgd_ms);
        if (ms_sgd) *ms_sgd = sgd_ms;
    } catch (...) {
        // an error inside a graph capture leaves s capturing: end and drop it
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(s, &g);
            if (g) cudaGraphDestroy(g);
        }
        cudaGetLastError();
        cudaStreamSynchronize(s);
        cudaStreamSynchronize(s2);
        cleanup();
        throw;
    }
    cleanup();
}
// Orders every epoch's segments of the window by head slice (see the epoch
// kernels): counts per (epoch, slice), slot offsets on the host, scatter.
template <typename T>
void SgdEngine<T>::build_slices(Window& win, int64_t nseg, int W, cudaStream_t s) {
    const int P = win.buckets = std::max(1, std::min(min_phases, 64));
    UMAPB_SYNC(s);   // win.host_seg_first (copied by the caller) is read below
    win.host_bucket_off.assign(static_cast<size_t>(W) * (P + 1), 0);
    if (num_inst_ <= 1 || W * P > SLICE_MAX_BINS) {
        // slices are consecutive segment ranges: identity order (with several
        // instances and too many bins for one block, slices of the whole row range)
        win.ordered = false;
        DevArray<int64_t> off(static_cast<size_t>(W) * (P + 1), s);
        slice_bounds_kernel<<<grid_for(static_cast<size_t>(W) * (P + 1), 128), 128, 0, s>>>(
            win.seg_pos.get(), win.ht.get(), win.seg_first.get(), W, ep_->n, P, off.get());
        UMAPB_LAUNCH_CHECK();
        UMAPB_CUDA(cudaMemcpyAsync(win.host_bucket_off.data(), off.get(), win.host_bucket_off.size() * sizeof(int64_t),
                                   cudaMemcpyDeviceToHost, s));
        UMAPB_SYNC(s);
        return;
    }
    win.ordered = true;
    win.seg_order.reserve(std::max<int64_t>(nseg, 1), s);
    DevArray<int> counts(static_cast<size_t>(W) * P, s);
    counts.zero(s);
    const unsigned blocks = static_cast<unsigned>((nseg + SLICE_BLOCK - 1) / SLICE_BLOCK);
    if (nseg > 0) {
        seg_bucket_kernel<<<blocks, SLICE_BLOCK, 0, s>>>(nseg, win.seg_pos.get(), win.ht.get(), win.seg_first.get(), W,
                                                         inst_start_, num_inst_, ep_->n, P, counts.get(), nullptr,
                                                         nullptr);
        UMAPB_LAUNCH_CHECK();
    }
    std::vector<int> hc(static_cast<size_t>(W) * P);
    UMAPB_CUDA(cudaMemcpyAsync(hc.data(), counts.get(), hc.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    std::vector<int> cursor(static_cast<size_t>(W) * P);
    for (int w = 0; w < W; ++w) {
        int64_t acc = win.host_seg_first[w];
        for (int b = 0; b < P; ++b) {
            win.host_bucket_off[static_cast<size_t>(w) * (P + 1) + b] = acc;
            cursor[static_cast<size_t>(w) * P + b] = static_cast<int>(acc - win.host_seg_first[w]);
            acc += hc[static_cast<size_t>(w) * P + b];
        }
        win.host_bucket_off[static_cast<size_t>(w) * (P + 1) + P] = acc;
    }
    if (nseg > 0) {
        DevArray<int> d_cursor(cursor.size(), s);
        UMAPB_CUDA(cudaMemcpyAsync(d_cursor.get(), cursor.data(), cursor.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        seg_bucket_kernel<<<blocks, SLICE_BLOCK, 0, s>>>(nseg, win.seg_pos.get(), win.ht.get(), win.seg_first.get(), W,
                                                         inst_start_, num_inst_, ep_->n, P, nullptr, d_cursor.get(),
                                                         win.seg_order.get());
        UMAPB_LAUNCH_CHECK();
        UMAPB_SYNC(s);   // the cursor vector is the copy's source
    }
}

// Self-check of the event windows (UMAPB_CHECK_SCHEDULE=1, used by the tests):
// per epoch, the window's events and negative samples must equal the totals of
// the schedule recomputed from the initial state, and the events of an epoch
// must come in head order.

__global__ void window_stats_kernel(const int2* __restrict__ ht, const uint16_t* __restrict__ nneg,
                                    const int64_t* __restrict__ starts, unsigned long long* __restrict__ negs,
                                    unsigned long long* __restrict__ disorder) {
    const int w = blockIdx.x;
    const int64_t a = starts[w], b = starts[w + 1];
    unsigned long long sn = 0, bad = 0;
    for (int64_t e = a + threadIdx.x; e < b; e += blockDim.x) {
        sn += nneg[e];
        if (e > a && ht[e - 1].x > ht[e].x) ++bad;
    }
    atomicAdd(&negs[w], sn);
    atomicAdd(&disorder[w], bad);
}

// Segments of epoch w: increasing, each inside one head's run and at most
// seg_max long, the first starting at the epoch's first event; bad counts
// the segments that break a rule.
__global__ void window_segments_kernel(const int2* __restrict__ ht, const int64_t* __restrict__ starts,
                                       const int64_t* __restrict__ seg_pos, const int64_t* __restrict__ seg_first,
                                       int seg_max, unsigned long long* __restrict__ bad) {
    const int w = blockIdx.x;
    const int64_t s0 = seg_first[w], s1 = seg_first[w + 1];
    unsigned long long nb = 0;
    if (threadIdx.x == 0 && s1 > s0 && seg_pos[s0] != starts[w]) ++nb;
    if (threadIdx.x == 0 && s1 == s0 && starts[w + 1] != starts[w]) ++nb;
    for (int64_t x = s0 + threadIdx.x; x < s1; x += blockDim.x) {
        const int64_t a = seg_pos[x], b = seg_pos[x + 1];
        if (!(a < b) || b - a > seg_max || ht[a].x != ht[b - 1].x || b > starts[w + 1]) ++nb;
    }
    atomicAdd(&bad[w], nb);
}

template <typename T>
void SgdEngine<T>::verify_window(const Window& win, int first, int W, cudaStream_t s) {
    const int64_t nnz = ep_->nnz;
    DevArray<T> en(nnz, s), enn(nnz, s);
    state_at(first, en.get(), enn.get(), s);
    DevArray<unsigned long long> totals(2 * static_cast<size_t>(W), s), negs(W, s), disorder(W, s);
    totals.zero(s);
    negs.zero(s);
    disorder.zero(s);
    if (nnz) {
        const int64_t nblocks = (nnz + SCHED_BLOCK - 1) / SCHED_BLOCK;
        sched_totals_kernel<T><<<static_cast<unsigned>(nblocks), SCHED_BLOCK, 0, s>>>(
            nnz, ep_->eps.get(), en.get(), enn.get(), ep_->negative_sample_rate, first, W, totals.get());
        UMAPB_LAUNCH_CHECK();
    }
    window_stats_kernel<<<W, 256, 0, s>>>(win.ht.get(), win.nneg.get(), win.epoch_offsets.get(), negs.get(), disorder.get());
    UMAPB_LAUNCH_CHECK();
    window_segments_kernel<<<W, 256, 0, s>>>(win.ht.get(), win.epoch_offsets.get(), win.seg_pos.get(),
                                             win.seg_first.get(), win.seg_max, disorder.get());
    UMAPB_LAUNCH_CHECK();
    std::vector<unsigned long long> ht_tot(2 * static_cast<size_t>(W)), hn(W), hd(W);
    UMAPB_CUDA(cudaMemcpyAsync(ht_tot.data(), totals.get(), ht_tot.size() * sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaMemcpyAsync(hn.data(), negs.get(), W * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaMemcpyAsync(hd.data(), disorder.get(), W * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    for (int w = 0; w < W; ++w) {
        const unsigned long long ev = static_cast<unsigned long long>(win.host_epoch_offsets[w + 1] - win.host_epoch_offsets[w]);
        require(ev == ht_tot[2 * w] && hn[w] == ht_tot[2 * w + 1] && hd[w] == 0,
                "schedule window self-check failed at epoch " + std::to_string(first + w), UMAPB_ERR_CUDA);
    }
}

template <typename T>
void SgdEngine<T>::counts(int first, int last, int64_t* out, cudaStream_t s) {
    const int64_t nnz = ep_->nnz;
    const int W = last - first;
    if (W <= 0) return;
    DevArray<T> en(nnz, s), enn(nnz, s);
    state_at(first, en.get(), enn.get(), s);
    DevArray<unsigned long long> totals(2 * static_cast<size_t>(W), s);
    totals.zero(s);
    if (nnz) {
        const int64_t nblocks = (nnz + SCHED_BLOCK - 1) / SCHED_BLOCK;
        sched_totals_kernel<T><<<static_cast<unsigned>(nblocks), SCHED_BLOCK, 0, s>>>(
            nnz, ep_->eps.get(), en.get(), enn.get(), ep_->negative_sample_rate, first, W, totals.get());
        UMAPB_LAUNCH_CHECK();
    }
    std::vector<unsigned long long> h(2 * static_cast<size_t>(W));
    UMAPB_CUDA(cudaMemcpyAsync(h.data(), totals.get(), h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    for (size_t i = 0; i < h.size(); ++i) out[i] = static_cast<int64_t>(h[i]);
}

// 8 ordered slices: measured on 2,000- and 100,000-point layouts, an epoch in
// one launch ends about 2-3 % below the serial reference's edge
// cross-entropy, 4 slices about 1.4 % below, 8 slices within about 0.6 %.
// UMAPB_SGD_PHASES overrides it (1 = every event of an epoch in one launch).
template <typename T>
int SgdEngine<T>::default_min_phases() {
    const char* e = std::getenv("UMAPB_SGD_PHASES");
    const int x = e ? std::atoi(e) : 0;
    return (x >= 1 && x <= 64) ? x : 8;
}

// UMAPB_SGD_VARIANT selects the 2-d kernel variant (index into
// SGD_2D_VARIANTS) when the launch shape is not tuned.
template <typename T>
int SgdEngine<T>::default_variant() {
    static const int v = [] {
        const char* e = std::getenv("UMAPB_SGD_VARIANT");
        const int x = e ? std::atoi(e) : -1;
        return (x >= 0 && x < NUM_SGD_2D_VARIANTS) ? x : 2;   // measured fastest at 100k and 1M points
    }();
    return v;
}

template class SgdEngine<float>;
template class SgdEngine<double>;

}  // namespace umapb
