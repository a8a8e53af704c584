// Measured ceilings for the roofline of the SGD epoch kernel.
//
// The embedding of a million observations is 8 MB (float2 per observation)
// and lives in L2, so the epochs are bound by random 8-byte accesses that hit
// L2 (tail and negative-sample gathers, tail and head atomic adds), not by
// HBM.  These kernels measure, on the device at hand, the rate of such
// accesses with nothing else to do: uniformly random float2 loads from an
// n-point array (ld.global.cg, L2 only), and uniformly random float2 atomic
// adds (red.global.add.v2.f32).  Each thread keeps GATHER_BATCH independent
// accesses in flight; indices come from a counter hash (no index array is
// read).
#include <algorithm>
#include <cstdint>

#include "stages.cuh"

namespace umapb {

namespace {

constexpr int PROBE_BLOCK = 256;
constexpr int GATHER_BATCH = 8;

// A 32-bit mixing function (two multiply-xorshift rounds; "lowbias32",
// C. Wellons, hash-prospector): enough to spread counters over the array.
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

__global__ void __launch_bounds__(PROBE_BLOCK) gather_probe_kernel(const float2* __restrict__ Y, uint32_t n,
                                                                  int rounds, uint32_t seed, float* __restrict__ sink) {
    const uint32_t tid = blockIdx.x * PROBE_BLOCK + threadIdx.x;
    float acc = 0.0f;
    uint32_t c = mix32(tid ^ seed);
    for (int r = 0; r < rounds; ++r) {
        float2 v[GATHER_BATCH];
#pragma unroll
        for (int i = 0; i < GATHER_BATCH; ++i) {
            c = mix32(c + i);
            v[i] = __ldcg(&Y[(static_cast<uint64_t>(c) * n) >> 32]);
        }
#pragma unroll
        for (int i = 0; i < GATHER_BATCH; ++i) acc += v[i].x + v[i].y;
    }
    if (acc == 12345.678f) sink[tid] = acc;   // keeps the loads; never true for the zero-filled array
}

__global__ void __launch_bounds__(PROBE_BLOCK) red_probe_kernel(float2* __restrict__ Y, uint32_t n, int rounds,
                                                               uint32_t seed) {
    const uint32_t tid = blockIdx.x * PROBE_BLOCK + threadIdx.x;
    uint32_t c = mix32(tid ^ seed);
    for (int r = 0; r < rounds; ++r) {
#pragma unroll
        for (int i = 0; i < GATHER_BATCH; ++i) {
            c = mix32(c + i);
            atomicAdd(&Y[(static_cast<uint64_t>(c) * n) >> 32], make_float2(0.0f, 0.0f));
        }
    }
}

}  // namespace

// Accesses per second of each probe (mode 0: gathers, 1: atomic adds) over
// an n-point float2 array, from CUDA events around 'reps' launches after one
// warm-up launch; about 'accesses' accesses per launch.
double measure_random_access(int64_t n, int64_t accesses, int mode, int reps, cudaStream_t s) {
    require(n >= 1 && n <= INT32_MAX, "probe array size out of range");
    require(accesses >= 1 && reps >= 1, "probe sizes must be positive");
    require(mode == 0 || mode == 1, "probe mode must be 0 (gather) or 1 (atomic add)");
    int dev = 0, sms = 0, per_sm = 0;
    UMAPB_CUDA(cudaGetDevice(&dev));
    UMAPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (mode == 0) {
        UMAPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gather_probe_kernel, PROBE_BLOCK, 0));
    } else {
        UMAPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, red_probe_kernel, PROBE_BLOCK, 0));
    }
    const int64_t blocks = static_cast<int64_t>(sms) * std::max(per_sm, 1);
    const int64_t threads = blocks * PROBE_BLOCK;
    const int rounds = static_cast<int>(std::max<int64_t>(1, accesses / (threads * GATHER_BATCH)));
    DevArray<float2> Y(static_cast<size_t>(n), s);
    DevArray<float> sink(static_cast<size_t>(threads), s);
    UMAPB_CUDA(cudaMemsetAsync(Y.get(), 0, static_cast<size_t>(n) * sizeof(float2), s));
    cudaEvent_t a = event_get(), b = event_get();
    float ms = 0;
    try {
        for (int rep = -1; rep < reps; ++rep) {
            if (rep == 0) UMAPB_CUDA(cudaEventRecord(a, s));
            if (mode == 0) {
                gather_probe_kernel<<<static_cast<unsigned>(blocks), PROBE_BLOCK, 0, s>>>(
                    Y.get(), static_cast<uint32_t>(n), rounds, 0x9E3779B9u * (rep + 2), sink.get());
            } else {
                red_probe_kernel<<<static_cast<unsigned>(blocks), PROBE_BLOCK, 0, s>>>(
                    Y.get(), static_cast<uint32_t>(n), rounds, 0x9E3779B9u * (rep + 2));
            }
            UMAPB_LAUNCH_CHECK();
        }
        UMAPB_CUDA(cudaEventRecord(b, s));
        UMAPB_CUDA(cudaEventSynchronize(b));
        UMAPB_CUDA(cudaEventElapsedTime(&ms, a, b));
    } catch (...) {
        event_put(a);
        event_put(b);
        throw;
    }
    event_put(a);
    event_put(b);
    const double total = static_cast<double>(threads) * rounds * GATHER_BATCH * reps;
    return total / (static_cast<double>(ms) * 1e-3);
}

}  // namespace umapb
