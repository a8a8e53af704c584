// optimize_layout on the device (include/umappp/optimize_layout.hpp:116-185).
//
// Rows.  The reference walks the heads in order and, for each head, its
// firing edges in CSR order: an attractive step that moves head and tail,
// then that edge's negative samples, which move the head only.  Here one
// thread takes one head's whole row, in the same per-row order: it evaluates
// the schedule of each edge of the row in the reference's exact Float_
// arithmetic (this file is compiled with -fmad=false), and for each firing
// edge takes the attractive step and the negative samples.  No event lists
// are built: the schedule state (epoch_of_next_sample and
// epoch_of_next_negative_sample) is advanced in place, edge by edge, by the
// thread that owns the edge's row.
//
// Concurrency.  All rows of an epoch run at once (one launch per epoch);
// warps claim chunks of 32 rows from a per-epoch counter, in an order fixed
// per run: rows by descending firing rate (sum of 1 / epochs_per_sample), so
// that the hubs -- heads with hundreds of firing edges per epoch at a million
// points, whose rows are the longest sequential chains -- start first.  A
// row's head is kept in registers and its displacement is added to the
// embedding (vector atomic add) after every 'publish_every' firing edges and
// at the end of the row; tails move by vector atomic adds.  Measured on a
// 1,000,000-point mixture against the serial reference's edge cross-entropy:
// splitting a hub's row into concurrently processed pieces, or publishing the
// head's move only at the end of a long row, leaves the layout about 1-1.5 %
// tighter than the reference's; whole rows with the head published after each
// firing edge come within about 0.3 %.
//
// Negative samples come from Philox4x32-10 keyed by the seed with counter
// (head, tail, epoch, block), so they do not depend on the launch shape or on
// how epochs are split across run() calls.
#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

#include "stages.cuh"
#include "umap_grad.cuh"

namespace umapb {

namespace {

constexpr int SCHED_BLOCK = 256;
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

// One schedule step of an edge at 'epoch' (optimize_layout.hpp:141-143,160-161,178-179).
template <typename T>
__device__ __forceinline__ bool schedule_step(T epoch, T eps, T epns, T& enext, T& enneg, int& nneg) {
    if (enext > epoch) return false;
    nneg = static_cast<int>((epoch - enneg) / epns);
    enext += eps;
    enneg += static_cast<T>(nneg) * epns;
    return true;
}

// Advances the schedule state by W epochs without any layout update.
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

// Per-epoch totals of firing edges and negative samples drawn, from the schedule alone.
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

// ------------------------------------------------------------ row order --

// Hub rows: expected to fire at least HUB_RATE edges per epoch.
constexpr int HUB_RATE = 128;
// Rows per group of the claim order (row_order_key_kernel).
constexpr int ORDER_GROUP = 4096;

// Order key of each row, sorted ascending: hub rows (firing rate -- the sum
// of 1 / epochs_per_sample over the row, the expected number of firing edges
// per epoch -- at least hub_rate) first, heaviest first; then the other rows
// in groups of 'group' consecutive indices, in index order of the groups and
// by descending rate within a group.  Rows in flight together then come from
// a narrow index range (the concurrency the layout's quality depends on),
// while the 32 rows a warp takes at once have similar lengths.
template <typename T>
__global__ void row_order_key_kernel(int32_t n, const int64_t* __restrict__ ptr, const T* __restrict__ eps,
                                     float hub_rate, int32_t group, uint64_t* __restrict__ key,
                                     int32_t* __restrict__ row, int* __restrict__ nhub) {
    int hubs = 0;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float r = 0.0f;
        for (int64_t j = ptr[i]; j < ptr[i + 1]; ++j) r += 1.0f / static_cast<float>(eps[j]);
        const bool hub = r >= hub_rate;
        hubs += hub;
        const uint64_t g = hub ? 0ull : 1ull + static_cast<uint64_t>(i / group);
        key[i] = (g << 32) | static_cast<uint64_t>(~__float_as_uint(r));   // r >= 0: bits order as values
        row[i] = i;
    }
    for (int o = 16; o > 0; o >>= 1) hubs += __shfl_xor_sync(0xffffffffu, hubs, o);
    if ((threadIdx.x & 31) == 0 && hubs) atomicAdd(nhub, hubs);
}

// The non-hub rows of one epoch in claim order: every chunk of ORDER_GROUP
// consecutive positions of the run's order (hub rows left out) sorted by
// descending number of edges that fire in this epoch -- counted by the
// previous epoch's kernel while it scanned the rows (RowArgs::next_count) --,
// equal counts (and counts of 255 or more) in the run's order (a stable sort).  A chunk keeps its
// positions, so the rows in flight together still come from one index range,
// while the 32 rows a warp takes fire the same number of edges (and rows that
// fire none come last).
constexpr int EPOCH_ORDER_THREADS = 512;
constexpr int EPOCH_ORDER_ITEMS = ORDER_GROUP / EPOCH_ORDER_THREADS;
__global__ void __launch_bounds__(EPOCH_ORDER_THREADS)
    epoch_bulk_order_kernel(const int32_t* __restrict__ run_order, int32_t nbulk, const uint16_t* __restrict__ count,
                            int32_t* __restrict__ bulk) {
    using Sort = cub::BlockRadixSort<uint32_t, EPOCH_ORDER_THREADS, EPOCH_ORDER_ITEMS, int32_t>;
    __shared__ typename Sort::TempStorage tmp;
    const int64_t first = static_cast<int64_t>(blockIdx.x) * ORDER_GROUP + threadIdx.x * EPOCH_ORDER_ITEMS;
    uint32_t key[EPOCH_ORDER_ITEMS];
    int32_t row[EPOCH_ORDER_ITEMS];
#pragma unroll
    for (int i = 0; i < EPOCH_ORDER_ITEMS; ++i) {   // blocked: item rank = position in the chunk
        const int64_t pos = first + i;
        row[i] = pos < nbulk ? run_order[pos] : -1;
        // descending count, capped at 255 (non-hub rows fire fewer edges than
        // that), in 8 bits; past the end: 256, last
        key[i] = pos < nbulk ? 255u - min(static_cast<uint32_t>(count[row[i]]), 255u) : 256u;
    }
    Sort(tmp).Sort(key, row, 0, 9);
#pragma unroll
    for (int i = 0; i < EPOCH_ORDER_ITEMS; ++i)
        if (first + i < nbulk) bulk[first + i] = row[i];
}

// ---------------------------------------------------------- epoch kernels --

template <typename T>
struct SgdParams {
    T a, b;
    T neg2ab;      // -2ab
    T gamma2b;     // 2 gamma b
    T alpha;
    T rate;        // negative_sample_rate in Float_
    T epoch;       // the epoch as Float_
    uint32_t k0, k1;
    uint32_t epoch_u;
    int32_t n;
    int32_t publish_every;
    // Independent instances laid out one after another (batched runs):
    // instance i owns observations [inst_start[i], inst_start[i + 1]) and
    // draws its negative samples there.  num_inst <= 1: one instance of n.
    const int32_t* inst_start;
    int32_t num_inst;
};

// The rows of one epoch and where they are claimed from.
template <typename T>
struct RowArgs {
    const int32_t* order;      // rows in processing order
    int32_t nrows;
    const int64_t* ptr;
    const int32_t* targets;
    const T* eps;
    T* enext;
    T* enneg;
    int* counter;              // claims so far in this epoch: [0] hub rows (or row groups), [1] other rows
    unsigned long long* totals;   // optional: [firing edges, negative samples drawn] of this epoch
    int32_t nhub;              // 2-d kernel: order[0, nhub) are hub rows, one warp each
    const int32_t* bulk;       // 2-d kernel: the other rows in this epoch's claim order (null: order + nhub)
    uint16_t* next_count;      // 2-d kernel, optional: receives each non-hub row's firing edges in the next epoch
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

// Counter-based negative-sample stream of one firing edge (Philox4x32-7).
struct NegStream {
    uint32_t c0, c1, c2, c3, k0, k1;
    Philox4 buf;
    int used;
    __device__ __forceinline__ NegStream(uint32_t h, uint32_t t, uint32_t epoch, uint32_t key0, uint32_t key1)
        : c0(h), c1(t), c2(epoch), c3(0), k0(key0), k1(key1), used(4) {}
    __device__ __forceinline__ uint32_t next() {
        if (used == 4) {
            // 7 rounds: the fewest for which Salmon et al. found Philox4x32
            // free of BigCrush failures; negative samples only need uniform,
            // independent indices, and the rounds are a tenth of an edge's work
            buf = philox4x32<7>(c0, c1, c2, c3++, k0, k1);
            used = 0;
        }
        // a select chain rather than buf.v[used]: a dynamically indexed array would live in local memory
        const uint32_t v = used == 0 ? buf.v[0] : used == 1 ? buf.v[1] : used == 2 ? buf.v[2] : buf.v[3];
        ++used;
        return v;
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

// The step coefficients, optimize_layout.hpp:147-149 (attractive) and
// :170-171 (repulsive), from the edge derivatives shared with the adjoint
// (umap_grad.cuh): attractive = -2 dA/dd2, repulsive = -2 gamma dR/dd2 with
// eps = 0.001.  FP32 layouts use the hardware-approximated power (__powf, an
// exp2 of b log2 x in the special-function unit) and divide (__fdividef): the
// step is stochastic and clamped, and the layout's cross-entropy was measured
// unchanged with libm's powf and IEEE division at a million points.
template <typename T>
__device__ __forceinline__ T attract_coef(T d2, const SgdParams<T>& p) {
    return attract_dd2<std::is_same<T, float>::value>(d2, p.a, p.b, p.neg2ab);
}

template <typename T>
__device__ __forceinline__ T repulse_coef(T d2, const SgdParams<T>& p) {
    return repulse_dd2<std::is_same<T, float>::value>(d2, p.a, p.b, p.gamma2b, T(0.001));
}

__device__ __forceinline__ float attract_coef_fast(float d2, const SgdParams<float>& p) { return attract_coef(d2, p); }
__device__ __forceinline__ float repulse_coef_fast(float d2, const SgdParams<float>& p) { return repulse_coef(d2, p); }

template <typename T>
__device__ __forceinline__ T floor_eps(T d2) {
    const T e = FloatLimits<T>::epsilon();
    return (e < d2) ? d2 : e;
}

// Next firing edge of a row at or after j (r1: none).
template <typename T>
__device__ __forceinline__ int64_t next_firing(const T* __restrict__ enext, int64_t j, int64_t r1, T epoch) {
    while (j < r1 && enext[j] > epoch) ++j;
    return j;
}

// The warp's next chunk of 32 rows (all lanes get the same base).
__device__ __forceinline__ int32_t claim_rows(int* counter) {
    int32_t base = 0;
    if ((threadIdx.x & 31) == 0) base = atomicAdd(counter, 32);
    return __shfl_sync(0xffffffffu, base, 0);
}

__device__ __forceinline__ void add_totals(unsigned long long* totals, unsigned long long fired,
                                           unsigned long long drawn) {
    if (!totals) return;
    for (int o = 16; o > 0; o >>= 1) {
        fired += __shfl_xor_sync(0xffffffffu, fired, o);
        drawn += __shfl_xor_sync(0xffffffffu, drawn, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&totals[0], fired);
        atomicAdd(&totals[1], drawn);
    }
}

// Coherent device-scope load: ordered after this thread's own earlier atomic
// adds to the same address (per-location coherence), so a head re-read after
// its own publication sees it, plus whatever other threads have added.
__device__ __forceinline__ float2 ld_relaxed_f2(const float2* q) {
    float2 v;
    asm volatile("ld.relaxed.gpu.global.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(q) : "memory");
    return v;
}

// 2-d FP32 rows.  Work units, claimed by warps in order: first the hub rows
// (one row per warp), then the other rows, 32 per warp (one per lane).
constexpr int BULK_CHUNK = 8;    // edges of a row whose schedule state a lane loads at once

// A row's schedule state, read BULK_CHUNK edges at a time into registers
// (the next window's loads in flight while the current one is used), and the
// row's firing edges found in it in order.
__device__ __forceinline__ void cp_async4(float* dst_shared, const float* src, bool valid) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst_shared));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// A lane's scan of its row's epoch_of_next_sample, BULK_CHUNK edges at a
// time, through two windows in shared memory (the lane's column of its warp's
// slab, [buffer][edge][lane]: conflict-free): the next window is copied
// asynchronously (cp.async) while the current one is used.
struct RowScan {
    int64_t cb, nb, r1;        // current window's first edge, next window's first edge, row end
    float* w;                  // this lane's column: w[(buffer * BULK_CHUNK + q) * 32]
    unsigned cm;               // firing edges of the current window not yet taken
    int cur;                   // buffer of the current window
    int n1;                    // edges seen so far that fire at the next epoch (their new state counted
                               // by lane_row_step for the ones that fire now)
    __device__ __forceinline__ void load(int buf, const float* __restrict__ enext, int64_t b) {
#pragma unroll
        for (int q = 0; q < BULK_CHUNK; ++q) {
            const bool ok = b + q < r1;
            cp_async4(&w[(buf * BULK_CHUNK + q) * 32], ok ? enext + b + q : enext, ok);
        }
        cp_async_commit();
    }
    __device__ __forceinline__ unsigned fire_mask(int buf, int64_t b, float ef) {
        // b < r1 here; edges past the row's end are masked off
        unsigned m = 0, m1 = 0;
        const float ef1 = ef + 1.0f;   // the next epoch (an integer: exact)
#pragma unroll
        for (int q = 0; q < BULK_CHUNK; ++q) {
            const float v = w[(buf * BULK_CHUNK + q) * 32];
            m |= (v <= ef ? 1u : 0u) << q;
            m1 |= (v <= ef1 ? 1u : 0u) << q;
        }
        const int64_t left = r1 - b;
        const unsigned valid = left >= BULK_CHUNK ? (1u << BULK_CHUNK) - 1u : (1u << static_cast<int>(left)) - 1u;
        m &= valid;
        n1 += __popc(m1 & valid) - __popc(m);   // fire at the next epoch, not at this one
        return m;
    }
    __device__ __forceinline__ void start(float* column, const float* __restrict__ enext, int64_t j0, int64_t end,
                                          float ef) {
        // the lane's previous row may have left a window copy in flight into
        // these buffers: let it land before they are refilled
        cp_async_wait<0>();
        w = column;
        r1 = end;
        cb = j0;
        nb = j0 + BULK_CHUNK;
        cur = 0;
        n1 = 0;
        load(0, enext, cb);
        load(1, enext, nb);
        cp_async_wait<1>();
        cm = fire_mask(0, cb, ef);
    }
    // Next firing edge (false: none left); en = its epoch_of_next_sample.
    __device__ __forceinline__ bool next(const float* __restrict__ enext, float ef, int64_t& j, float& en) {
        while (cm == 0) {
            if (nb >= r1) return false;
            cb = nb;
            cur ^= 1;
            cp_async_wait<0>();
            cm = fire_mask(cur, cb, ef);
            nb += BULK_CHUNK;
            load(cur ^ 1, enext, nb);
        }
        const int q = __ffs(cm) - 1;
        cm &= cm - 1;
        j = cb + q;
        en = w[(cur * BULK_CHUNK + q) * 32];
        return true;
    }
};

// One firing edge of a lane's row, with its target and schedule state.
struct RowEdge {
    int64_t j;
    float en, ep, enn;
    int32_t t;
};

// A lane's current row: its scan, the firing edge at hand (cur: state loaded
// two steps ago), the one after it (nxt: state loads in flight) and its
// instance's range for negative samples.
struct LaneRow {
    int32_t h;       // -1: none
    float hx, hy;    // the head, when it is not re-read (FRESH = false)
    int32_t nbase;
    uint32_t nsize;
    bool has_nxt;
    RowEdge cur, nxt;
    RowScan sc;
};

// Finds the row's next firing edge and issues its state loads.
__device__ __forceinline__ bool lane_row_fetch(LaneRow& L, RowEdge& e, const RowArgs<float>& r, float ef) {
    if (!L.sc.next(r.enext, ef, e.j, e.en)) return false;
    e.t = r.targets[e.j];
    e.ep = r.eps[e.j];
    e.enn = r.enneg[e.j];
    return true;
}

// Starts row h on a lane: false when the row fires no edge this epoch.
template <typename P>
__device__ __forceinline__ bool lane_row_start(LaneRow& L, int32_t h, const RowArgs<float>& r, const float2* Y,
                                               const P& p, float* column) {
    const float ef = p.epoch;
    const int64_t j0 = r.ptr[h], r1 = r.ptr[h + 1];
    if (j0 >= r1) {
        if (r.next_count) r.next_count[h] = 0;
        return false;
    }
    L.sc.start(column, r.enext, j0, r1, ef);
    if (!lane_row_fetch(L, L.cur, r, ef)) {   // the whole row scanned: nothing fires now
        if (r.next_count) r.next_count[h] = static_cast<uint16_t>(min(L.sc.n1, 65535));
        return false;
    }
    L.has_nxt = lane_row_fetch(L, L.nxt, r, ef);
    L.h = h;
    const float2 y0 = __ldcg(&Y[h]);
    L.hx = y0.x;
    L.hy = y0.y;
    instance_range(h, p, L.nbase, L.nsize);
    return true;
}

// One firing edge of a lane's row.  The head (re-read: it sees the pulls of
// other rows' attractive steps), the tail and the first NB negative samples
// are gathered together -- the negative-sample indices do not depend on the
// layout; while they are in flight the schedule step is written and the
// state loads of the firing edge after the next one are issued (so an edge's
// gathers never wait for its own state); then the updates are applied in the
// reference's order and the head's move is published.  Returns false when
// the row has no firing edge left.
template <int NB, bool FRESH>
__device__ __forceinline__ bool lane_row_step(LaneRow& L, const RowArgs<float>& r, float2* __restrict__ Y,
                                              const SgdParams<float>& p, unsigned long long& fired,
                                              unsigned long long& drawn) {
    const float ef = p.epoch;
    const int32_t h = L.h, t = L.cur.t;
    const float2 yh = FRESH ? ld_relaxed_f2(&Y[h]) : make_float2(L.hx, L.hy);
    const float2 yt = __ldcg(&Y[t]);
    const float epns = L.cur.ep / p.rate;   // optimize_layout.hpp:160-161
    const int nn = static_cast<int>((ef - L.cur.enn) / epns);
    int remaining = nn > 0 ? nn : 0;         // a negative count draws nothing, as in the reference's loop
    NegStream rng(static_cast<uint32_t>(h), static_cast<uint32_t>(t), p.epoch_u, p.k0, p.k1);
    int m = remaining < NB ? remaining : NB;
    int32_t ks[NB];
    float2 yk[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        if (b < m) {
            ks[b] = L.nbase + rng.bounded(L.nsize);
            yk[b] = __ldcg(&Y[ks[b]]);
        }
    }
    const float en_new = L.cur.en + L.cur.ep;                 // :178-179
    r.enext[L.cur.j] = en_new;
    r.enneg[L.cur.j] = L.cur.enn + static_cast<float>(nn) * epns;
    L.sc.n1 += en_new <= ef + 1.0f ? 1 : 0;
    ++fired;
    drawn += remaining;
    // rotate: nxt becomes cur; fetch the one after
    const bool more = L.has_nxt;
    if (more) {
        L.cur = L.nxt;
        L.has_nxt = lane_row_fetch(L, L.nxt, r, ef);
    }
    float hx = yh.x, hy = yh.y;
    {   // attractive step (:145-155)
        const float dx = hx - yt.x, dy = hy - yt.y;
        const float d2 = floor_eps(__fmaf_rn(dx, dx, dy * dy));
        const float cf = attract_coef_fast(d2, p);
        const float gx = p.alpha * clamp4(cf * dx);
        const float gy = p.alpha * clamp4(cf * dy);
        hx += gx;
        hy += gy;
        atomicAdd(&Y[t], make_float2(-gx, -gy));
    }
    while (true) {   // negative samples (:157-176)
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            if (b < m && ks[b] != h) {
                const float dx = hx - yk[b].x, dy = hy - yk[b].y;
                const float d2 = floor_eps(__fmaf_rn(dx, dx, dy * dy));
                const float cf = repulse_coef_fast(d2, p);
                hx = __fmaf_rn(p.alpha, clamp4(cf * dx), hx);
                hy = __fmaf_rn(p.alpha, clamp4(cf * dy), hy);
            }
        }
        remaining -= m;
        if (remaining <= 0) break;
        m = remaining < NB ? remaining : NB;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            if (b < m) {
                ks[b] = L.nbase + rng.bounded(L.nsize);
                yk[b] = __ldcg(&Y[ks[b]]);
            }
        }
    }
    atomicAdd(&Y[h], make_float2(hx - yh.x, hy - yh.y));
    L.hx = hx;
    L.hy = hy;
    // the row's last firing edge: every window has been scanned
    if (!more && r.next_count) r.next_count[h] = static_cast<uint16_t>(min(L.sc.n1, 65535));
    return more;
}

// Gathered operands of one firing edge of a hub row (shared memory).
template <int NB>
struct HubEvent {
    float2 yt;
    float2 yk[NB];
    int32_t ks[NB];
    int32_t t;
    int32_t nn;
};

// A hub row, by a whole warp: the lanes take 32 edges at a time -- schedule
// step, tail and first NB negative samples gathered into shared memory, all
// in parallel -- and lane 0 then applies the chunk's firing edges in order,
// publishing the head's move after each edge.  Lane 0 re-reads the head at
// the start of every chunk (the value arrives while the chunk is gathered) and
// at the chunk's end takes it, plus the chunk's own moves, as the head: the
// pulls of other rows' attractive steps on the hub are seen a chunk late.
template <int NB>
__device__ __forceinline__ void hub_row(int32_t h, const RowArgs<float>& r, float2* __restrict__ Y,
                                        const SgdParams<float>& p, HubEvent<NB>* __restrict__ ev,
                                        unsigned long long& fired, unsigned long long& drawn) {
    const int lane = threadIdx.x & 31;
    const float ef = p.epoch;
    const int64_t j0 = r.ptr[h], r1 = r.ptr[h + 1];
    int32_t nbase;
    uint32_t nsize;
    instance_range(h, p, nbase, nsize);
    float hx = 0.0f, hy = 0.0f;   // lane 0: the head
    bool have = false;
    for (int64_t c = j0; c < r1; c += 32) {
        float2 seen = make_float2(0.0f, 0.0f);
        const bool resync = lane == 0 && have;
        if (resync) seen = ld_relaxed_f2(&Y[h]);   // includes this lane's earlier publications
        const float cx = hx, cy = hy;                          // lane 0: the head at the chunk's start
        const int64_t j = c + lane;
        bool fire = false;
        if (j < r1) {
            const float en = r.enext[j];
            fire = en <= ef;
            if (fire) {
                const float ep = r.eps[j], enn = r.enneg[j];
                const int32_t t = r.targets[j];
                const float epns = ep / p.rate;
                const int nn = static_cast<int>((ef - enn) / epns);
                r.enext[j] = en + ep;
                r.enneg[j] = enn + static_cast<float>(nn) * epns;
                const int draws = nn > 0 ? nn : 0;
                ++fired;
                drawn += draws;
                HubEvent<NB>& e = ev[lane];
                e.t = t;
                e.nn = draws;
                e.yt = __ldcg(&Y[t]);
                NegStream rng(static_cast<uint32_t>(h), static_cast<uint32_t>(t), p.epoch_u, p.k0, p.k1);
                const int m = draws < NB ? draws : NB;
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    if (b < m) {
                        const int32_t k = nbase + rng.bounded(nsize);
                        e.ks[b] = k;
                        e.yk[b] = __ldcg(&Y[k]);
                    }
                }
            }
        }
        unsigned mask = __ballot_sync(0xffffffffu, fire);
        __syncwarp();
        if (lane == 0) {
            if (mask && !have) {
                const float2 y0 = ld_relaxed_f2(&Y[h]);
                hx = y0.x;
                hy = y0.y;
                have = true;
            }
            while (mask) {
                const int q = __ffs(mask) - 1;
                mask &= mask - 1;
                const HubEvent<NB>& e = ev[q];
                const float sx = hx, sy = hy;
                {
                    const float dx = hx - e.yt.x, dy = hy - e.yt.y;
                    const float d2 = floor_eps(__fmaf_rn(dx, dx, dy * dy));
                    const float cf = attract_coef_fast(d2, p);
                    const float gx = p.alpha * clamp4(cf * dx);
                    const float gy = p.alpha * clamp4(cf * dy);
                    hx += gx;
                    hy += gy;
                    atomicAdd(&Y[e.t], make_float2(-gx, -gy));
                }
                const int nn = e.nn;
                const int m = nn < NB ? nn : NB;
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    if (b < m && e.ks[b] != h) {
                        const float dx = hx - e.yk[b].x, dy = hy - e.yk[b].y;
                        const float d2 = floor_eps(__fmaf_rn(dx, dx, dy * dy));
                        const float cf = repulse_coef_fast(d2, p);
                        hx = __fmaf_rn(p.alpha, clamp4(cf * dx), hx);
                        hy = __fmaf_rn(p.alpha, clamp4(cf * dy), hy);
                    }
                }
                if (nn > NB) {   // rare: the rest of this edge's negative samples, from the same stream
                    NegStream rng(static_cast<uint32_t>(h), static_cast<uint32_t>(e.t), p.epoch_u, p.k0, p.k1);
                    for (int b = 0; b < nn; ++b) {
                        const int32_t k = nbase + rng.bounded(nsize);
                        if (b < NB || k == h) continue;
                        const float2 y = __ldcg(&Y[k]);
                        const float dx = hx - y.x, dy = hy - y.y;
                        const float d2 = floor_eps(__fmaf_rn(dx, dx, dy * dy));
                        const float cf = repulse_coef_fast(d2, p);
                        hx = __fmaf_rn(p.alpha, clamp4(cf * dx), hx);
                        hy = __fmaf_rn(p.alpha, clamp4(cf * dy), hy);
                    }
                }
                atomicAdd(&Y[h], make_float2(hx - sx, hy - sy));
            }
            if (resync) {   // a read was issued at this chunk's start
                hx = seen.x + (hx - cx);
                hy = seen.y + (hy - cy);
            }
        }
        __syncwarp();
    }
}

// The epoch: warps first take the hub rows, one per warp, from counter[0];
// then the other rows 32 at a time from counter[1], one per lane, each loop
// iteration applying one firing edge of every lane's row (the rows a warp
// takes have similar lengths: row_order_key_kernel, and per epoch
// epoch_bulk_order_kernel).
template <int NB, int MINB, bool FRESH>
__global__ void __launch_bounds__(256, MINB) sgd_rows_2d_f32(RowArgs<float> r, float2* __restrict__ Y,
                                                             SgdParams<float> p) {
    __shared__ HubEvent<NB> hub_ev[256 / 32][32];
    __shared__ float scan_win[256 / 32][2 * BULK_CHUNK * 32];
    unsigned long long fired = 0, drawn = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    while (true) {
        int32_t u = 0;
        if (lane == 0) u = atomicAdd(&r.counter[0], 1);
        u = __shfl_sync(0xffffffffu, u, 0);
        if (u >= r.nhub) break;
        hub_row<NB>(r.order[u], r, Y, p, hub_ev[warp], fired, drawn);
        __syncwarp();
    }
    const int32_t nbulk = r.nrows - r.nhub;
    const int32_t* bulk = r.bulk ? r.bulk : r.order + r.nhub;
    while (true) {
        int32_t base = 0;
        if (lane == 0) base = atomicAdd(&r.counter[1], 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= nbulk) break;
        LaneRow L;
        L.h = -1;
        const int32_t idx = base + lane;
        if (idx < nbulk && !lane_row_start(L, bulk[idx], r, Y, p, &scan_win[warp][lane])) L.h = -1;
        while (__any_sync(0xffffffffu, L.h >= 0)) {
            if (L.h >= 0 && !lane_row_step<NB, FRESH>(L, r, Y, p, fired, drawn)) L.h = -1;
        }
    }
    add_totals(r.totals, fired, drawn);
}

struct Sgd2dVariant {
    void (*kernel)(RowArgs<float>, float2*, SgdParams<float>);
    int neg_batch, min_blocks;
};
const Sgd2dVariant SGD_2D_VARIANTS[] = {
    // default: head kept in registers, published per firing edge, negative
    // samples gathered 5 at a time (most firing edges draw 5; measured at
    // 1M: 180 ms against 185 for 6, 186 for 4, 189 for 8)
    {sgd_rows_2d_f32<5, 2, false>, 5, 2},
    {sgd_rows_2d_f32<6, 2, false>, 6, 2},
    {sgd_rows_2d_f32<6, 3, false>, 6, 3},
    {sgd_rows_2d_f32<8, 2, false>, 8, 2},
    {sgd_rows_2d_f32<6, 2, true>, 6, 2},     // head re-read before every firing edge
    {sgd_rows_2d_f32<4, 2, false>, 4, 2},
};
constexpr int NUM_SGD_2D_VARIANTS = sizeof(SGD_2D_VARIANTS) / sizeof(SGD_2D_VARIANTS[0]);

// Any dimension (up to MAX_GENERIC_DIM) and either precision; same per-row order.
template <typename T>
__global__ void __launch_bounds__(128) sgd_rows_generic(RowArgs<T> r, T* __restrict__ Y, int dim, SgdParams<T> p) {
    T head[MAX_GENERIC_DIM], pub[MAX_GENERIC_DIM];
    unsigned long long fired = 0, drawn = 0;
    const T ef = p.epoch;
    while (true) {
        const int32_t base = claim_rows(r.counter);
        if (base >= r.nrows) break;
        const int32_t i = base + (threadIdx.x & 31);
        if (i < r.nrows) {
            const int32_t h = r.order[i];
            const int64_t r1 = r.ptr[h + 1];
            int64_t j = next_firing(r.enext, r.ptr[h], r1, ef);
            if (j < r1) {
                int32_t nbase;
                uint32_t nsize;
                instance_range(h, p, nbase, nsize);
                T* yh = Y + static_cast<size_t>(h) * dim;
                for (int d = 0; d < dim; ++d) head[d] = pub[d] = __ldcg(yh + d);
                int since = 0;
                do {
                    const T ep = r.eps[j];
                    const T epns = ep / p.rate;
                    const T enn = r.enneg[j];
                    const int nn = static_cast<int>((ef - enn) / epns);
                    r.enext[j] = r.enext[j] + ep;
                    r.enneg[j] = enn + static_cast<T>(nn) * epns;
                    const int32_t t = r.targets[j];
                    ++fired;
                    drawn += nn > 0 ? nn : 0;
                    T* yt = Y + static_cast<size_t>(t) * dim;
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
                        NegStream rng(static_cast<uint32_t>(h), static_cast<uint32_t>(t), p.epoch_u, p.k0, p.k1);
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
                    j = next_firing(r.enext, j + 1, r1, ef);
                    if (++since >= p.publish_every || j >= r1) {
                        for (int d = 0; d < dim; ++d) {
                            atomicAdd(yh + d, head[d] - pub[d]);
                            pub[d] = head[d];
                        }
                        since = 0;
                    }
                } while (j < r1);
            }
        }
        __syncwarp();
    }
    add_totals(r.totals, fired, drawn);
}

// ------------------------------------------------------------ transform --
// Out-of-sample embedding (no counterpart in the reference: optimize_layout
// applied to points added to a finished layout).  Row i of the transform
// graph holds new point i's nearest reference points with their smoothed
// similarities; it is optimised like a row of optimize_layout
// (optimize_layout.hpp:136-180: schedule, attractive step, negative samples,
// the same arithmetic as sgd_rows_generic) except that only the new point
// moves: the reference points it is pulled to and the negative samples,
// drawn among the reference points, stay fixed.  Rows then share nothing that
// changes, so one thread takes one row through all epochs in one launch and
// the result does not depend on the launch shape.

// Initial position of every new point: the mean of its neighbours' reference
// positions weighted by the similarities (FP64 sums in edge order; plain mean
// if the weights sum to zero).
template <typename T>
__global__ void transform_init_kernel(int32_t nq, int dim, const int64_t* __restrict__ ptr,
                                      const int32_t* __restrict__ idx, const T* __restrict__ w,
                                      const T* __restrict__ Yref, T* __restrict__ Ynew) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) {
        const int64_t r0 = ptr[i], r1 = ptr[i + 1];
        double ws = 0;
        for (int64_t j = r0; j < r1; ++j) ws += static_cast<double>(w[j]);
        const bool weighted = ws > 0;
        const double den = weighted ? ws : static_cast<double>(r1 - r0);
        for (int d = 0; d < dim; ++d) {
            double acc = 0;
            for (int64_t j = r0; j < r1; ++j) {
                const double wj = weighted ? static_cast<double>(w[j]) : 1.0;
                acc += wj * static_cast<double>(Yref[static_cast<size_t>(idx[j]) * dim + d]);
            }
            Ynew[static_cast<size_t>(i) * dim + d] = static_cast<T>(den > 0 ? acc / den : 0.0);
        }
    }
}

// All epochs of every new point's row (thread i: row i).  head0 + i is the
// point's index in the negative-sample stream's counter; lr is the learning
// rate in the layout's type.
template <typename T>
__global__ void __launch_bounds__(128)
    transform_sgd_kernel(int32_t nq, int dim, const int64_t* __restrict__ ptr, const int32_t* __restrict__ targets,
                         const T* __restrict__ eps, T* __restrict__ enext, T* __restrict__ enneg,
                         const T* __restrict__ Yref, int32_t nref, T* __restrict__ Ynew, int32_t head0, int num_epochs,
                         T lr, SgdParams<T> p) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    T head[MAX_GENERIC_DIM];
    T* yh = Ynew + static_cast<size_t>(i) * dim;
    for (int d = 0; d < dim; ++d) head[d] = yh[d];
    const int64_t r0 = ptr[i], r1 = ptr[i + 1];
    const uint32_t hid = static_cast<uint32_t>(head0 + i);
    for (int e = 0; e < num_epochs; ++e) {
        const T ef = static_cast<T>(e);
        // alpha as in the layout's epochs (optimize_layout.hpp:132-133)
        const T alpha = static_cast<T>(static_cast<double>(lr) *
                                       (1.0 - static_cast<double>(ef / static_cast<T>(num_epochs))));
        for (int64_t j = r0; j < r1; ++j) {
            if (!(enext[j] <= ef)) continue;
            const T ep = eps[j];
            const T epns = ep / p.rate;
            const T enn = enneg[j];
            const int nn = static_cast<int>((ef - enn) / epns);
            enext[j] = enext[j] + ep;
            enneg[j] = enn + static_cast<T>(nn) * epns;
            const int32_t t = targets[j];
            const T* yt = Yref + static_cast<size_t>(t) * dim;
            T d2 = 0;
            for (int d = 0; d < dim; ++d) {
                const T diff = head[d] - yt[d];
                d2 += diff * diff;
            }
            {
                const T c = attract_coef(floor_eps(d2), p);
                for (int d = 0; d < dim; ++d) head[d] += alpha * clamp4(c * (head[d] - yt[d]));
            }
            if (nn > 0) {
                NegStream rng(hid, static_cast<uint32_t>(t), static_cast<uint32_t>(e), p.k0, p.k1);
                for (int q = 0; q < nn; ++q) {
                    const T* yk = Yref + static_cast<size_t>(rng.bounded(static_cast<uint32_t>(nref))) * dim;
                    T dd2 = 0;
                    for (int d = 0; d < dim; ++d) {
                        const T diff = head[d] - yk[d];
                        dd2 += diff * diff;
                    }
                    const T c = repulse_coef(floor_eps(dd2), p);
                    for (int d = 0; d < dim; ++d) head[d] += alpha * clamp4(c * (head[d] - yk[d]));
                }
            }
        }
    }
    for (int d = 0; d < dim; ++d) yh[d] = head[d];
}

// UMAPB_CHECK_SCHEDULE=1: the epoch kernels count the firing edges and
// negative samples they process, and every run compares the counts with the
// schedule's own totals (sched_totals_kernel).
bool check_schedule() {
    const char* e = std::getenv("UMAPB_CHECK_SCHEDULE");
    return e && *e && *e != '0';
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

// Resident blocks per SM of 2-d variant v at 'block' threads (occupancy query, cached).
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

int generic_resident() {
    static int r = 0;
    if (r == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, sgd_rows_generic<double>, 128, 0) != cudaSuccess || r < 1) {
            cudaGetLastError();
            r = 1;
        }
    }
    return r;
}

}  // namespace

template <typename T>
void SgdEngine<T>::setup(const DeviceEpochs<T>* ep, cudaStream_t s, int base_epoch) {
    ep_ = ep;
    base_epoch_ = base_epoch;
    const int64_t nnz = ep->nnz;
    const int32_t n = ep->n;
    enext_.allocate(nnz, s);
    enneg_.allocate(nnz, s);
    if (nnz) {
        UMAPB_CUDA(cudaMemcpyAsync(enext_.get(), ep->enext0.get(), nnz * sizeof(T), cudaMemcpyDeviceToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(enneg_.get(), ep->enneg0.get(), nnz * sizeof(T), cudaMemcpyDeviceToDevice, s));
    }
    state_epoch_ = base_epoch_;
    // rows by descending firing rate
    order_.allocate(n, s);
    if (n > 0) {
        DevArray<uint64_t> key(n, s), key_sorted(n, s);
        DevArray<int32_t> row(n, s);
        DevArray<int> cnt(1, s);
        cnt.zero(s);
        float hub_rate = static_cast<float>(HUB_RATE);   // UMAPB_SGD_HUB_RATE overrides it
        if (const char* e = std::getenv("UMAPB_SGD_HUB_RATE")) hub_rate = static_cast<float>(std::atof(e));
        int32_t group = ORDER_GROUP;                       // UMAPB_SGD_ORDER_GROUP overrides it
        if (const char* e = std::getenv("UMAPB_SGD_ORDER_GROUP")) group = std::max(1, std::atoi(e));
        row_order_key_kernel<T><<<grid_for(n, 256), 256, 0, s>>>(n, ep->ptr.get(), ep->eps.get(), hub_rate, group,
                                                                key.get(), row.get(), cnt.get());
        UMAPB_LAUNCH_CHECK();
        int end_bit = 33;
        while (end_bit < 64 && (int64_t(1) << (end_bit - 32)) <= int64_t(n) / group + 1) ++end_bit;
        size_t tb = 0;
        UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.get(), key_sorted.get(), row.get(), order_.get(), n,
                                                   0, end_bit, s));
        DevArray<unsigned char> temp(tb, s);
        UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(temp.get(), tb, key.get(), key_sorted.get(), row.get(), order_.get(),
                                                   n, 0, end_bit, s));
        UMAPB_CUDA(cudaMemcpyAsync(&nhub_, cnt.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        UMAPB_SYNC(s);
    } else {
        nhub_ = 0;
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

// Autotuner: times one epoch with each candidate launch shape on scratch
// copies of the layout and of the schedule state, keeps the fastest, and
// remembers it per size class (log2 of the edge count).
template <typename T>
template <class Launch>
void SgdEngine<T>::tune(T* Y, int num_dim, int epoch, Launch& launch, cudaStream_t s) {
    static std::mutex mu;
    static std::map<int, std::pair<int, int>> cache;   // size class -> (block, variant)
    const int64_t nnz = ep_->nnz;
    int key = 0;
    while ((int64_t(1) << key) < nnz) ++key;
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
    DevArray<T> yscr(total, s), en(nnz, s), enn(nnz, s);
    DevArray<int> counter(2, s);
    cudaEvent_t a = event_get(), b = event_get();
    float best = 1e30f;
    for (int v = 0; v < NUM_SGD_2D_VARIANTS; ++v) {
        for (int blk : {128, 256}) {
            UMAPB_CUDA(cudaMemcpyAsync(yscr.get(), Y, total * sizeof(T), cudaMemcpyDeviceToDevice, s));
            UMAPB_CUDA(cudaMemcpyAsync(en.get(), enext_.get(), nnz * sizeof(T), cudaMemcpyDeviceToDevice, s));
            UMAPB_CUDA(cudaMemcpyAsync(enn.get(), enneg_.get(), nnz * sizeof(T), cudaMemcpyDeviceToDevice, s));
            counter.zero(s);
            UMAPB_CUDA(cudaEventRecord(a, s));
            launch(yscr.get(), en.get(), enn.get(), counter.get(), nullptr, epoch, blk, v);
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
    p.rate = ep_->negative_sample_rate;
    p.k0 = static_cast<uint32_t>(seed) ^ RNG_NEGATIVE;
    p.k1 = static_cast<uint32_t>(seed >> 32);
    p.n = ep_->n;
    p.publish_every = std::max(1, publish_every);
    p.inst_start = inst_start_;
    p.num_inst = num_inst_;
    const T lr = static_cast<T>(learning_rate);
    const bool use_2d = std::is_same<T, float>::value && num_dim == 2;
    const bool check = check_schedule();
    cudaStream_t s = caller;
    // Rows in flight at once: at most n / window_div (a sliding window over
    // the claim order), so that few rows run beside their neighbours with
    // positions read before those neighbours' updates; at a million points
    // that is still enough rows to keep L2 saturated.
    // UMAPB_SGD_MAX_BLOCKS overrides the block count (0: from the window).
    int max_blocks = 0;
    if (const char* e = std::getenv("UMAPB_SGD_MAX_BLOCKS")) max_blocks = std::max(0, std::atoi(e));
    const int64_t window_rows = window_div > 0
        ? std::max<int64_t>(1, std::max<int64_t>(ep_->n / window_div, std::min<int64_t>(ep_->n / 8, 32768)))
        : int64_t(1) << 40;

    const bool eorder = use_2d && epoch_order && ep_->n > nhub_;
    if (eorder) {
        next_count_.reserve(ep_->n, s);
        bulk_.reserve(ep_->n - nhub_, s);
    }
    // One epoch launch on (Yp, schedule state en/enn), claiming rows from 'counter'.
    auto launch = [&](T* Yp, T* en, T* enn, int* counter, unsigned long long* totals, int e_abs, int block,
                      int variant) {
        const T epoch_t = static_cast<T>(e_abs);
        // alpha = lr * (1 - epoch / num_epochs) in the reference's types (optimize_layout.hpp:132-133)
        p.alpha = static_cast<T>(static_cast<double>(lr) * (1.0 - static_cast<double>(epoch_t / static_cast<T>(total))));
        p.epoch = epoch_t;
        p.epoch_u = static_cast<uint32_t>(e_abs);
        RowArgs<T> r;
        r.order = order_.get();
        r.nrows = ep_->n;
        r.ptr = ep_->ptr.get();
        r.targets = ep_->targets.get();
        r.eps = ep_->eps.get();
        r.enext = en;
        r.enneg = enn;
        r.counter = counter;
        r.totals = totals;
        r.nhub = use_2d ? nhub_ : 0;
        r.bulk = nullptr;
        r.next_count = nullptr;
        if (eorder) {
            r.next_count = next_count_.get();
            if (e_abs > first) {   // counts from the previous epoch of this call
                const int32_t nbulk = ep_->n - nhub_;
                epoch_bulk_order_kernel<<<static_cast<unsigned>((nbulk + ORDER_GROUP - 1) / ORDER_GROUP),
                                          EPOCH_ORDER_THREADS, 0, s>>>(order_.get() + nhub_, nbulk,
                                                                      next_count_.get(), bulk_.get());
                UMAPB_LAUNCH_CHECK();
                r.bulk = bulk_.get();
            }
        }
        if (use_2d) {
            if constexpr (std::is_same<T, float>::value) {
                int64_t g = static_cast<int64_t>(sm_count()) * sgd_2d_resident(variant, block);
                g = std::min<int64_t>(g, std::max<int64_t>(1, (window_rows + block - 1) / block));
                if (max_blocks > 0) g = std::min<int64_t>(g, max_blocks);
                SGD_2D_VARIANTS[variant].kernel<<<static_cast<unsigned>(g), block, 0, s>>>(
                    r, reinterpret_cast<float2*>(Yp), p);
            }
        } else {
            int64_t g = static_cast<int64_t>(sm_count()) * generic_resident();
            g = std::min<int64_t>(g, std::max<int64_t>(1, (window_rows + 127) / 128));
            if (max_blocks > 0) g = std::min<int64_t>(g, max_blocks);
            sgd_rows_generic<T><<<static_cast<unsigned>(g), 128, 0, s>>>(r, Yp, num_dim, p);
        }
        UMAPB_LAUNCH_CHECK();
    };

    if (state_epoch_ != first) {
        state_at(first, enext_.get(), enneg_.get(), s);
        state_epoch_ = first;
    }
    if (autotune && use_2d) tune(Y, num_dim, first, launch, s);
    const int W = last - first;
    DevArray<int> counters(2 * static_cast<size_t>(W), s);
    DevArray<unsigned long long> totals(check ? 2 * static_cast<size_t>(W) : 0, s);
    cudaEvent_t start = event_get(), finish = event_get();
    cudaGraphExec_t exec = nullptr;
    try {
        UMAPB_CUDA(cudaEventRecord(start, s));
        auto enqueue = [&] {
            UMAPB_CUDA(cudaMemsetAsync(counters.get(), 0, 2 * W * sizeof(int), s));
            if (check) UMAPB_CUDA(cudaMemsetAsync(totals.get(), 0, 2 * W * sizeof(unsigned long long), s));
            for (int e = first; e < last; ++e)
                launch(Y, enext_.get(), enneg_.get(), counters.get() + 2 * (e - first),
                       check ? totals.get() + 2 * (e - first) : nullptr, e, block_, variant_);
        };
        if (use_graphs) {
            // the epochs of this call as one CUDA graph
            cudaGraph_t graph = nullptr;
            UMAPB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            enqueue();
            UMAPB_CUDA(cudaStreamEndCapture(s, &graph));
            const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ie != cudaSuccess) cuda_fail(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
            UMAPB_CUDA(cudaGraphLaunch(exec, s));
        } else {
            enqueue();
        }
        UMAPB_CUDA(cudaEventRecord(finish, s));
        UMAPB_CUDA(cudaEventSynchronize(finish));
        float ms = 0;
        UMAPB_CUDA(cudaEventElapsedTime(&ms, start, finish));
        if (ms_sgd) *ms_sgd = ms;
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
        if (exec) cudaGraphExecDestroy(exec);
        event_put(start);
        event_put(finish);
        throw;
    }
    if (exec) cudaGraphExecDestroy(exec);
    event_put(start);
    event_put(finish);
    state_epoch_ = last;
    if (check) {
        std::vector<int64_t> want(2 * static_cast<size_t>(W));
        counts(first, last, want.data(), s);
        std::vector<unsigned long long> got(2 * static_cast<size_t>(W));
        UMAPB_CUDA(cudaMemcpyAsync(got.data(), totals.get(), got.size() * sizeof(unsigned long long),
                                   cudaMemcpyDeviceToHost, s));
        UMAPB_SYNC(s);
        for (int w = 0; w < W; ++w)
            require(static_cast<int64_t>(got[2 * w]) == want[2 * w] && static_cast<int64_t>(got[2 * w + 1]) == want[2 * w + 1],
                    "schedule self-check failed at epoch " + std::to_string(first + w), UMAPB_ERR_CUDA);
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

// UMAPB_SGD_VARIANT selects the 2-d kernel variant (index into
// SGD_2D_VARIANTS) when the launch shape is not tuned.
template <typename T>
int SgdEngine<T>::default_variant() {
    const char* e = std::getenv("UMAPB_SGD_VARIANT");
    const int x = e ? std::atoi(e) : -1;
    return (x >= 0 && x < NUM_SGD_2D_VARIANTS) ? x : 0;
}

// UMAPB_SGD_WINDOW_DIV: rows in flight at most max(n / this, min(n / 8, 32768))
// (default 12; 0: no cap).
template <typename T>
int SgdEngine<T>::default_window_div() {
    const char* e = std::getenv("UMAPB_SGD_WINDOW_DIV");
    const int x = e ? std::atoi(e) : -1;
    return (x >= 0 && x <= 1 << 20) ? x : 12;
}

// UMAPB_SGD_EPOCH_ORDER=0 keeps the run's claim order in every epoch.
template <typename T>
bool SgdEngine<T>::default_epoch_order() {
    const char* e = std::getenv("UMAPB_SGD_EPOCH_ORDER");
    return !(e && std::atoi(e) == 0);
}

// UMAPB_SGD_PUBLISH_EVERY: firing edges between publications of a row's head
// (default 1: after every firing edge).
template <typename T>
int SgdEngine<T>::default_publish_every() {
    const char* e = std::getenv("UMAPB_SGD_PUBLISH_EVERY");
    const int x = e ? std::atoi(e) : 0;
    return (x >= 1 && x <= 1 << 20) ? x : 1;
}

template class SgdEngine<float>;
template class SgdEngine<double>;

template <typename T>
void transform_init(int32_t nq, int num_dim, const int64_t* ptr, const int32_t* idx, const T* w, const T* Yref,
                    T* Ynew, cudaStream_t s) {
    if (nq <= 0) return;
    transform_init_kernel<T><<<grid_for(nq, 128), 128, 0, s>>>(nq, num_dim, ptr, idx, w, Yref, Ynew);
    UMAPB_LAUNCH_CHECK();
}

template <typename T>
void transform_layout(const DeviceEpochs<T>& ep, int num_dim, const T* Yref, int32_t nref, T* Ynew, int32_t head0,
                      double a, double b, double gamma, double learning_rate, uint64_t seed, cudaStream_t s) {
    require(num_dim >= 1 && num_dim <= MAX_GENERIC_DIM, "num_dim must be between 1 and 64");
    require(nref >= 1, "the transform needs at least one reference point");
    const int32_t nq = ep.n;
    if (nq <= 0) return;
    SgdParams<T> p{};
    p.a = static_cast<T>(a);
    p.b = static_cast<T>(b);
    p.neg2ab = T(-2) * p.a * p.b;
    p.gamma2b = T(2) * static_cast<T>(gamma) * p.b;
    p.rate = ep.negative_sample_rate;
    p.k0 = static_cast<uint32_t>(seed) ^ RNG_NEGATIVE;
    p.k1 = static_cast<uint32_t>(seed >> 32);
    p.n = nref;
    p.publish_every = 1;
    p.inst_start = nullptr;
    p.num_inst = 1;
    DevArray<T> en(std::max<int64_t>(ep.nnz, 1), s), enn(std::max<int64_t>(ep.nnz, 1), s);
    if (ep.nnz) {
        UMAPB_CUDA(cudaMemcpyAsync(en.get(), ep.enext0.get(), ep.nnz * sizeof(T), cudaMemcpyDeviceToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(enn.get(), ep.enneg0.get(), ep.nnz * sizeof(T), cudaMemcpyDeviceToDevice, s));
    }
    transform_sgd_kernel<T><<<static_cast<unsigned>((nq + 127) / 128), 128, 0, s>>>(
        nq, num_dim, ep.ptr.get(), ep.targets.get(), ep.eps.get(), en.get(), enn.get(), Yref, nref, Ynew, head0,
        ep.total_epochs, static_cast<T>(learning_rate), p);
    UMAPB_LAUNCH_CHECK();
}

template void transform_init<float>(int32_t, int, const int64_t*, const int32_t*, const float*, const float*, float*,
                                    cudaStream_t);
template void transform_init<double>(int32_t, int, const int64_t*, const int32_t*, const double*, const double*,
                                     double*, cudaStream_t);
template void transform_layout<float>(const DeviceEpochs<float>&, int, const float*, int32_t, float*, int32_t, double,
                                      double, double, double, uint64_t, cudaStream_t);
template void transform_layout<double>(const DeviceEpochs<double>&, int, const double*, int32_t, double*, int32_t,
                                       double, double, double, double, uint64_t, cudaStream_t);

}  // namespace umapb
