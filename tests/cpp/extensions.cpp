// The extension entry points through the C++ drop-in headers: many small runs
// in one batch_run call, then the loss and gradient of each instance's layout.
// Built by the CPU tests (compile and link); it needs a GPU to run.
#include <cstdio>
#include <random>
#include <vector>

#include "umappp/umappp.hpp"

int main() {
    const std::size_t ndim = 8;
    const std::vector<int32_t> sizes{300, 500, 200};
    int32_t total = 0;
    for (auto s : sizes) total += s;
    std::mt19937_64 rng(7);
    std::normal_distribution<float> norm;
    std::vector<float> data(static_cast<std::size_t>(total) * ndim);
    for (auto& x : data) x = norm(rng);

    umappp::Options opt;
    opt.num_epochs = 100;
    std::vector<float> embedding(static_cast<std::size_t>(total) * 2);
    const auto ms = umappp::batch_run(sizes, ndim, data.data(), 2, embedding.data(), opt);
    std::printf("batch: %.2f ms of SGD\n", ms[6]);

    // a ring graph over the first instance's points, weight 0.5 each way
    const int32_t n = sizes[0];
    std::vector<int64_t> ptr(n + 1);
    std::vector<int32_t> idx;
    std::vector<float> w;
    for (int32_t i = 0; i < n; ++i) {
        ptr[i] = static_cast<int64_t>(idx.size());
        idx.push_back((i + n - 1) % n);
        idx.push_back((i + 1) % n);
        w.push_back(0.5f);
        w.push_back(0.5f);
    }
    ptr[n] = static_cast<int64_t>(idx.size());
    const auto lg = umappp::loss_grad<float>(2, embedding.data(), n, ptr.data(), idx.data(), w.data(), 1.58, 0.9, 0.001);
    std::printf("loss %.6g, dL/da %.6g, dL/db %.6g\n", lg.loss, lg.grad_a, lg.grad_b);
    return 0;
}
