// Device workspace cache, event pool and stream pool.
//
// Runtime calls that reach the GPU's resource manager (allocation, memory
// queries, stream and event creation) can hold the host for tens to hundreds
// of milliseconds on a busy system, even when the stream-ordered pool already
// has the memory.  A UMAP run makes a few dozen such allocations, so the
// library keeps what it frees: released blocks go to a size-bucketed cache and
// are handed out again without a runtime call.  A block released on stream A
// and reused on stream B is ordered by an event recorded on A at release
// (B waits on it), so reuse never races with work still in flight.
//
// Buckets: below 1 MiB, powers of two (at least 512 B); from 1 MiB, multiples
// of 2 MiB.  A request takes a cached block of its own bucket or one up to a
// quarter larger.  When the device reports out-of-memory the cache hands its
// blocks back to the device pool and the allocation is retried once.
//
// umapb_set_workspace_limit caps the bytes in use: a request beyond it fails
// with UMAPB_ERR_OOM, as a real out-of-memory does; new device memory that
// would take in-use plus cached bytes past the cap first flushes the cache.
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace umapb {

namespace {

struct Block {
    void* ptr;
    size_t bytes;
    int device;
    cudaStream_t released_on;
    cudaEvent_t ready;   // recorded on released_on at release
};

struct Cache {
    std::mutex mu;
    std::multimap<size_t, Block> free_blocks;           // by bucket size
    std::unordered_map<void*, Block> in_use;            // by pointer
    std::vector<cudaEvent_t> spare_events;               // timing disabled
    size_t cached_bytes = 0;
    size_t in_use_bytes = 0;
    size_t limit = 0;                                    // 0: no limit
};

Cache& cache() {
    static Cache* c = new Cache();   // never destroyed: blocks may be released during process exit
    return *c;
}

size_t bucket(size_t bytes) {
    constexpr size_t MiB = size_t(1) << 20;
    if (bytes < MiB) {
        size_t b = 512;
        while (b < bytes) b <<= 1;
        return b;
    }
    return (bytes + 2 * MiB - 1) / (2 * MiB) * (2 * MiB);
}

int current_device() {
    int d = 0;
    cudaGetDevice(&d);
    return d;
}

// Hands every cached block back to the device pool (cache lock held).
void flush_locked(Cache& c) {
    for (auto& kv : c.free_blocks) {
        Block& b = kv.second;
        cudaFreeAsync(b.ptr, b.released_on);   // ordered after the work that released it
        c.spare_events.push_back(b.ready);
    }
    c.free_blocks.clear();
    c.cached_bytes = 0;
}

}  // namespace

void* ws_alloc(size_t bytes, cudaStream_t s) {
    if (bytes == 0) return nullptr;
    const size_t want = bucket(bytes);
    const int dev = current_device();
    Cache& c = cache();
    {
        std::lock_guard<std::mutex> lock(c.mu);
        if (c.limit && c.in_use_bytes + want > c.limit)
            fail(UMAPB_ERR_OOM, "device workspace limit reached (" + std::to_string(c.limit) + " bytes; " +
                                    std::to_string(want) + " more requested)");
        for (auto it = c.free_blocks.lower_bound(want); it != c.free_blocks.end() && it->first <= want + want / 4;
             ++it) {
            if (it->second.device != dev) continue;
            Block b = it->second;
            c.free_blocks.erase(it);
            c.cached_bytes -= b.bytes;
            if (b.released_on != s) {
                const cudaError_t e = cudaStreamWaitEvent(s, b.ready, 0);
                if (e != cudaSuccess) {
                    c.free_blocks.emplace(b.bytes, b);
                    c.cached_bytes += b.bytes;
                    cuda_fail(e, "cudaStreamWaitEvent", __FILE__, __LINE__);
                }
            }
            c.spare_events.push_back(b.ready);
            b.ready = nullptr;
            c.in_use.emplace(b.ptr, b);
            c.in_use_bytes += b.bytes;
            return b.ptr;
        }
        if (c.limit && c.in_use_bytes + c.cached_bytes + want > c.limit) flush_locked(c);
    }
    const double t0 = trace_enabled() ? host_ms() : 0.0;
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, want, s);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        {
            std::lock_guard<std::mutex> lock(c.mu);
            flush_locked(c);
        }
        e = cudaMallocAsync(&p, want, s);
    }
    if (e != cudaSuccess) cuda_fail(e, "cudaMallocAsync", __FILE__, __LINE__);
    if (trace_enabled()) trace_wait("device allocation", t0, want, __FILE__, __LINE__);
    std::lock_guard<std::mutex> lock(c.mu);
    c.in_use.emplace(p, Block{p, want, dev, s, nullptr});
    c.in_use_bytes += want;
    return p;
}

void ws_free(void* p, cudaStream_t s) {
    if (!p) return;
    Cache& c = cache();
    std::lock_guard<std::mutex> lock(c.mu);
    auto it = c.in_use.find(p);
    if (it == c.in_use.end()) {
        cudaFreeAsync(p, s);   // not ours: should not happen, but do not leak
        return;
    }
    Block b = it->second;
    c.in_use.erase(it);
    c.in_use_bytes -= b.bytes;
    cudaEvent_t ev = nullptr;
    if (!c.spare_events.empty()) {
        ev = c.spare_events.back();
        c.spare_events.pop_back();
    } else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeAsync(p, s);   // cannot order a later reuse: give the block back to the pool
        return;
    }
    if (cudaEventRecord(ev, s) != cudaSuccess) {
        cudaGetLastError();
        c.spare_events.push_back(ev);
        cudaFreeAsync(p, s);
        return;
    }
    b.released_on = s;
    b.ready = ev;
    c.free_blocks.emplace(b.bytes, b);
    c.cached_bytes += b.bytes;
}

size_t ws_cached_bytes() {
    Cache& c = cache();
    std::lock_guard<std::mutex> lock(c.mu);
    return c.cached_bytes;
}

void ws_release_cached() {
    Cache& c = cache();
    std::lock_guard<std::mutex> lock(c.mu);
    flush_locked(c);
}

size_t ws_set_limit(size_t bytes) {
    Cache& c = cache();
    std::lock_guard<std::mutex> lock(c.mu);
    const size_t prev = c.limit;
    c.limit = bytes;
    return prev;
}

// ------------------------------------------------------------ event pool --

namespace {
std::mutex g_event_mu;
std::vector<cudaEvent_t>& timing_events() {
    static auto* v = new std::vector<cudaEvent_t>();
    return *v;
}
std::mutex g_stream_mu;
std::vector<std::pair<int, cudaStream_t>>& spare_streams() {   // (device * 2 + high priority, stream)
    static auto* v = new std::vector<std::pair<int, cudaStream_t>>();
    return *v;
}
}  // namespace

cudaEvent_t event_get() {
    {
        std::lock_guard<std::mutex> lock(g_event_mu);
        auto& v = timing_events();
        if (!v.empty()) {
            cudaEvent_t e = v.back();
            v.pop_back();
            return e;
        }
    }
    cudaEvent_t e = nullptr;
    UMAPB_CUDA(cudaEventCreate(&e));
    return e;
}

void event_put(cudaEvent_t e) {
    if (!e) return;
    std::lock_guard<std::mutex> lock(g_event_mu);
    timing_events().push_back(e);
}

cudaStream_t stream_get(bool high_priority) {
    const int dev = current_device();
    const int key = dev * 2 + (high_priority ? 1 : 0);
    {
        std::lock_guard<std::mutex> lock(g_stream_mu);
        auto& v = spare_streams();
        for (size_t i = 0; i < v.size(); ++i) {
            if (v[i].first == key) {
                cudaStream_t s = v[i].second;
                v.erase(v.begin() + static_cast<std::ptrdiff_t>(i));
                return s;
            }
        }
    }
    int least = 0, greatest = 0;
    if (high_priority) UMAPB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    cudaStream_t s = nullptr;
    UMAPB_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, high_priority ? greatest : least));
    return s;
}

// The stream must be idle (synchronised by the caller).
void stream_put(cudaStream_t s) {
    if (!s) return;
    int priority = 0, least = 0, greatest = 0;   // no throw: called from destructors
    const bool high = cudaStreamGetPriority(s, &priority) == cudaSuccess &&
                      cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess && greatest < least &&
                      priority == greatest;
    cudaGetLastError();
    std::lock_guard<std::mutex> lock(g_stream_mu);
    spare_streams().emplace_back(current_device() * 2 + (high ? 1 : 0), s);
}

}  // namespace umapb
