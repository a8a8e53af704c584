// Exact brute-force Euclidean kNN on the host cores: the stand-in for the
// knncolle search the reference calls (include/umappp/initialize.hpp:140),
// used by ref_shim/knncolle/knncolle.hpp.  Built separately with -O3 and
// AVX2/FMA so the CPU baseline is a fair, vectorised brute force: points are
// processed in tiles of 256 stored dimension-major, each query's squared
// distances to a tile are accumulated from coordinate differences (the
// inner loop over the tile's points vectorises), and a per-query max-heap
// keeps the k best (distance, index) pairs.
//
// Test infrastructure only (CPU baseline and oracle/_ref).
#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <thread>
#include <utility>
#include <vector>

namespace {

template <typename T>
void search(const T* data, std::size_t dim, int nobs, int qstart, int qcount, int k, int nthreads, int* out_idx,
            T* out_d2) {
    constexpr int TILE = 256;
    const int kk = std::min(k, nobs > 0 ? nobs - 1 : 0);
    auto work = [&](int qs, int qe) {
        std::vector<T> tile(dim * TILE);
        std::vector<T> acc(TILE);
        std::vector<std::vector<std::pair<T, int>>> heaps(qe - qs);
        for (auto& h : heaps) h.reserve(kk + 1);
        for (int base = 0; base < nobs; base += TILE) {
            const int w = std::min(TILE, nobs - base);
            for (int j = 0; j < w; ++j)
                for (std::size_t d = 0; d < dim; ++d) tile[d * TILE + j] = data[(std::size_t)(base + j) * dim + d];
            for (int q = qs; q < qe; ++q) {
                const T* xq = data + (std::size_t)q * dim;
                for (int j = 0; j < TILE; ++j) acc[j] = 0;
                for (std::size_t d = 0; d < dim; ++d) {
                    const T qd = xq[d];
                    const T* row = tile.data() + d * TILE;
                    T* a = acc.data();
#pragma GCC ivdep
                    for (int j = 0; j < TILE; ++j) {
                        const T diff = qd - row[j];
                        a[j] += diff * diff;
                    }
                }
                auto& heap = heaps[q - qs];
                for (int j = 0; j < w; ++j) {
                    const int id = base + j;
                    if (id == q) continue;
                    const std::pair<T, int> c(acc[j], id);
                    if ((int)heap.size() < kk) {
                        heap.push_back(c);
                        std::push_heap(heap.begin(), heap.end());
                    } else if (kk > 0 && c < heap.front()) {
                        std::pop_heap(heap.begin(), heap.end());
                        heap.back() = c;
                        std::push_heap(heap.begin(), heap.end());
                    }
                }
            }
        }
        for (int q = qs; q < qe; ++q) {
            auto& heap = heaps[q - qs];
            std::sort_heap(heap.begin(), heap.end());
            for (int t = 0; t < (int)heap.size(); ++t) {
                out_idx[(std::size_t)(q - qstart) * k + t] = heap[t].second;
                out_d2[(std::size_t)(q - qstart) * k + t] = heap[t].first;
            }
            for (int t = (int)heap.size(); t < k; ++t) {
                out_idx[(std::size_t)(q - qstart) * k + t] = -1;
                out_d2[(std::size_t)(q - qstart) * k + t] = T(-1);
            }
        }
    };
    const int nt = std::max(1, nthreads);
    // queries in chunks of 64 per thread task so the tile stays hot in cache across them
    std::vector<std::thread> threads;
    const int chunk = 64;
    std::vector<std::pair<int, int>> tasks;
    for (int s = qstart; s < qstart + qcount; s += chunk) tasks.emplace_back(s, std::min(qstart + qcount, s + chunk));
    for (int t = 0; t < nt; ++t) {
        threads.emplace_back([&, t]() {
            for (std::size_t i = t; i < tasks.size(); i += nt) work(tasks[i].first, tasks[i].second);
        });
    }
    for (auto& th : threads) th.join();
}

}  // namespace

void oracle_bruteforce_knn(const float* data, std::size_t dim, int nobs, int qstart, int qcount, int k, int nthreads,
                           int* out_idx, float* out_d2) {
    search<float>(data, dim, nobs, qstart, qcount, k, nthreads, out_idx, out_d2);
}

void oracle_bruteforce_knn(const double* data, std::size_t dim, int nobs, int qstart, int qcount, int k, int nthreads,
                           int* out_idx, double* out_d2) {
    search<double>(data, dim, nobs, qstart, qcount, k, nthreads, out_idx, out_d2);
}
