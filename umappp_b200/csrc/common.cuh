// Shared host/device plumbing of libumappp_b200: error reporting, stream-ordered
// device buffers, host/device pointer staging, and the counter-based random
// number generator used by every kernel that samples.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>

#include "umapb.h"

namespace umapb {

extern std::atomic<long long> g_launches;   // defined in capi.cu
// Poll limit of the tensor-core kernels' bounded mbarrier waits
// (umapb_set_device_wait_limit; defined in capi.cu).
extern std::atomic<long long> g_wait_limit;
inline long long device_wait_limit() { return g_wait_limit.load(std::memory_order_relaxed); }

// ---------------------------------------------------------------- errors ---

struct Error : public std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error(code, msg); }

[[noreturn]] inline void cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
    const int code = (e == cudaErrorMemoryAllocation) ? UMAPB_ERR_OOM
                   : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? UMAPB_ERR_NO_DEVICE
                   : UMAPB_ERR_CUDA;
    throw Error(code, std::string(cudaGetErrorString(e)) + " in " + what + " (" + file + ":" + std::to_string(line) + ")");
}

// ---------------------------------------------------------------- tracing ---
// UMAPB_TRACE=1 reports to stderr every runtime call of this library that
// holds the host for longer than a millisecond (synchronisations, allocations,
// copies), with its source line, so that stalls between kernels can be
// attributed.

inline bool trace_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("UMAPB_TRACE");
        return e && *e && *e != '0';
    }();
    return on;
}

inline double host_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

inline void trace_wait(const char* what, double t0, size_t bytes, const char* file, int line) {
    const double dt = host_ms() - t0;
    if (dt <= 1.0) return;
    if (bytes) std::fprintf(stderr, "[umapb] %s of %.0f MB took %.1f ms (%s:%d)\n", what, bytes / 1e6, dt, file, line);
    else std::fprintf(stderr, "[umapb] %s took %.1f ms (%s:%d)\n", what, dt, file, line);
}

#define UMAPB_CUDA(call)                                                           \
    do {                                                                           \
        const double umapb_t0_ = ::umapb::trace_enabled() ? ::umapb::host_ms() : 0.0; \
        cudaError_t umapb_e_ = (call);                                             \
        if (umapb_e_ != cudaSuccess) ::umapb::cuda_fail(umapb_e_, #call, __FILE__, __LINE__); \
        if (::umapb::trace_enabled()) ::umapb::trace_wait(#call, umapb_t0_, 0, __FILE__, __LINE__); \
    } while (0)

// Every kernel launch of this library is followed by this check, which also
// counts the launch (umapb_launch_count()).
#define UMAPB_LAUNCH_CHECK()                                                     \
    do {                                                                         \
        ::umapb::g_launches.fetch_add(1, std::memory_order_relaxed);             \
        UMAPB_CUDA(cudaGetLastError());                                          \
    } while (0)

inline void require(bool cond, const std::string& msg, int code = UMAPB_ERR_INVALID) {
    if (!cond) fail(code, msg);
}

inline void stream_sync(cudaStream_t s, const char* file, int line) {
    const double t0 = trace_enabled() ? host_ms() : 0.0;
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) cuda_fail(e, "cudaStreamSynchronize", file, line);
    if (trace_enabled()) trace_wait("stream synchronise", t0, 0, file, line);
}
#define UMAPB_SYNC(stream) ::umapb::stream_sync((stream), __FILE__, __LINE__)

// Device-side error word values (written by kernels with bounded waits).
enum DeviceStatus : int { DEV_OK = 0, DEV_TIMEOUT = 1, DEV_BAD_INPUT = 2 };

// ------------------------------------------------------- device buffers ---

// Workspace cache (memory.cu): stream-ordered device blocks that are kept
// and reused instead of being returned to the runtime; event and stream pools.
void* ws_alloc(size_t bytes, cudaStream_t s);
void ws_free(void* p, cudaStream_t s);
size_t ws_cached_bytes();
void ws_release_cached();
size_t ws_set_limit(size_t bytes);   // cap on bytes held (in use + cached), 0: none; returns the previous cap
cudaEvent_t event_get();          // timing event from the pool
void event_put(cudaEvent_t e);
cudaStream_t stream_get(bool high_priority = false);   // non-blocking stream of the current device
void stream_put(cudaStream_t s);  // s must be idle

// Stream-ordered device allocation from the workspace cache; released on the
// stream it was allocated on when the owner goes away.
template <typename T>
class DevArray {
public:
    DevArray() = default;
    DevArray(size_t n, cudaStream_t s) { allocate(n, s); }
    ~DevArray() { release(); }
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    DevArray(DevArray&& o) noexcept : ptr_(o.ptr_), n_(o.n_), stream_(o.stream_) { o.ptr_ = nullptr; o.n_ = 0; }
    DevArray& operator=(DevArray&& o) noexcept {
        if (this != &o) {
            release();
            ptr_ = o.ptr_; n_ = o.n_; stream_ = o.stream_;
            o.ptr_ = nullptr; o.n_ = 0;
        }
        return *this;
    }
    void allocate(size_t n, cudaStream_t s) {
        release();
        stream_ = s;
        n_ = n;
        if (n > 0) {
            if (n > SIZE_MAX / sizeof(T)) fail(UMAPB_ERR_OVERFLOW, "device allocation size overflows");
            ptr_ = static_cast<T*>(ws_alloc(n * sizeof(T), s));
        }
    }
    // Grows to at least n elements (contents are not kept); never shrinks.
    void reserve(size_t n, cudaStream_t s) {
        if (n > n_) allocate(n, s);
    }
    void release() {
        if (ptr_) ws_free(ptr_, stream_);
        ptr_ = nullptr;
        n_ = 0;
    }
    T* get() const { return ptr_; }
    size_t size() const { return n_; }
    size_t bytes() const { return n_ * sizeof(T); }
    void zero(cudaStream_t s) const {
        if (n_) UMAPB_CUDA(cudaMemsetAsync(ptr_, 0, n_ * sizeof(T), s));
    }

private:
    T* ptr_ = nullptr;
    size_t n_ = 0;
    cudaStream_t stream_ = nullptr;
};

// True when p is device (or managed) memory usable by kernels on this device.
// Device memory of another GPU is rejected (UMAPB_ERR_INVALID): without peer
// access a kernel reading it would fault, and every buffer of a call must
// belong to the current device.
inline bool is_device_pointer(const void* p) {
    if (!p) return false;
    cudaPointerAttributes attr;
    cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (attr.type == cudaMemoryTypeDevice) {
        int dev = -1;
        if (cudaGetDevice(&dev) != cudaSuccess) {
            cudaGetLastError();
            dev = -1;
        }
        if (attr.device != dev)
            fail(UMAPB_ERR_INVALID, "a device pointer belongs to device " + std::to_string(attr.device) +
                                        ", not to the current device " + std::to_string(dev));
        return true;
    }
    return attr.type == cudaMemoryTypeManaged;
}

// Read-only view of a caller array on the device: the caller's pointer when it
// is already device memory, else a staged copy.
template <typename T>
class DeviceIn {
public:
    DeviceIn(const T* p, size_t n, cudaStream_t s) {
        if (n == 0) return;
        require(p != nullptr, "null input pointer");
        if (is_device_pointer(p)) {
            ptr_ = p;
        } else {
            copy_.allocate(n, s);
            UMAPB_CUDA(cudaMemcpyAsync(copy_.get(), p, n * sizeof(T), cudaMemcpyHostToDevice, s));
            ptr_ = copy_.get();
        }
    }
    const T* get() const { return ptr_; }

private:
    const T* ptr_ = nullptr;
    DevArray<T> copy_;
};

// Writable view: device pointer used in place, or a staged copy that is
// (optionally) filled from the host on entry and written back by finish().
template <typename T>
class DeviceInOut {
public:
    DeviceInOut(T* p, size_t n, cudaStream_t s, bool load) : host_(nullptr), n_(n), stream_(s) {
        if (n == 0) return;
        require(p != nullptr, "null output pointer");
        if (is_device_pointer(p)) {
            ptr_ = p;
        } else {
            host_ = p;
            copy_.allocate(n, s);
            if (load) UMAPB_CUDA(cudaMemcpyAsync(copy_.get(), p, n * sizeof(T), cudaMemcpyHostToDevice, s));
            ptr_ = copy_.get();
        }
    }
    T* get() const { return ptr_; }
    bool staged() const { return host_ != nullptr; }
    void finish() {
        if (host_ && n_) UMAPB_CUDA(cudaMemcpyAsync(host_, ptr_, n_ * sizeof(T), cudaMemcpyDeviceToHost, stream_));
    }

private:
    T* ptr_ = nullptr;
    T* host_;
    size_t n_;
    cudaStream_t stream_;
    DevArray<T> copy_;
};

// Copies a device value array of type Src into the caller's array of type Dst.
inline void copy_out(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes == 0 || dst == nullptr) return;
    UMAPB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s));
}

// ------------------------------------------------------- device context ---

// Per-thread execution context for the stage entry points: the current
// device, a non-blocking stream and a device status word.
struct Context {
    int device = -1;
    cudaStream_t stream = nullptr;
    int* d_status = nullptr;
};

Context& thread_context();                 // defined in capi.cu
void set_last_error(const std::string& m);  // message for umapb_last_error() on this thread
void check_device_status(Context& ctx);     // reads and clears the status word; throws on error

inline unsigned grid_for(size_t work, unsigned block, unsigned max_blocks = 148u * 64u) {
    size_t g = (work + block - 1) / block;
    if (g < 1) g = 1;
    if (g > max_blocks) g = max_blocks;
    return static_cast<unsigned>(g);
}

// ----------------------------------------------------------------- RNG ----

// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC 2011): a counter-based generator, so a draw depends only
// on (key, counter) and parallel kernels need no generator state.
struct Philox4 {
    uint32_t v[4];
};

template <int ROUNDS>
__host__ __device__ __forceinline__ Philox4 philox4x32(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                                       uint32_t k1) {
    constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    constexpr uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < ROUNDS; ++r) {
        const uint64_t p0 = static_cast<uint64_t>(M0) * c0;
        const uint64_t p1 = static_cast<uint64_t>(M1) * c2;
        const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
        const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += W0; k1 += W1;
    }
    return Philox4{{c0, c1, c2, c3}};
}

// The recommended 10 rounds (random initial layouts, jitter).
__host__ __device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                          uint32_t k0, uint32_t k1) {
    return philox4x32<10>(c0, c1, c2, c3, k0, k1);
}

// Uniform float in [0, 1) and double in [0, 1) from 24 / 53 random bits.
__host__ __device__ __forceinline__ float u32_to_unit_float(uint32_t x) { return (x >> 8) * (1.0f / 16777216.0f); }
__host__ __device__ __forceinline__ double u64_to_unit_double(uint32_t hi, uint32_t lo) {
    const uint64_t x = (static_cast<uint64_t>(hi) << 32) | lo;
    return static_cast<double>(x >> 11) * (1.0 / 9007199254740992.0);
}

// Philox stream tags, so different uses of one seed never share counters.
enum RngStream : uint32_t { RNG_NEGATIVE = 0x4E454731u, RNG_RANDOM_INIT = 0x52494E31u, RNG_JITTER = 0x4A495431u,
                            RNG_LANCZOS = 0x4C414E31u };

}  // namespace umapb
