// Project-written stand-in for subpar::parallelize_range (absent here):
// splits [0, num_tasks) into at most 'num_workers' contiguous ranges and runs
// fn(worker, start, length) on each in its own std::thread.
//
// Test infrastructure only.
#ifndef ORACLE_SHIM_SUBPAR_HPP
#define ORACLE_SHIM_SUBPAR_HPP

#include <algorithm>
#include <exception>
#include <thread>
#include <vector>

namespace subpar {

template<typename Task_, class Run_>
int parallelize_range(int num_workers, Task_ num_tasks, Run_ run_task_range) {
    if (num_tasks <= 0) {
        return 0;
    }
    if (num_workers < 1) {
        num_workers = 1;
    }
    const Task_ per = num_tasks / num_workers + (num_tasks % num_workers != 0);
    const int used = static_cast<int>((num_tasks + per - 1) / per);
    if (used <= 1) {
        run_task_range(0, static_cast<Task_>(0), num_tasks);
        return 1;
    }

    std::vector<std::thread> workers;
    std::vector<std::exception_ptr> errors(used);
    workers.reserve(used);
    for (int w = 0; w < used; ++w) {
        const Task_ start = per * w;
        const Task_ length = std::min<Task_>(per, num_tasks - start);
        workers.emplace_back([&, w, start, length]() {
            try {
                run_task_range(w, start, length);
            } catch (...) {
                errors[w] = std::current_exception();
            }
        });
    }
    for (auto& t : workers) {
        t.join();
    }
    for (auto& e : errors) {
        if (e) {
            std::rethrow_exception(e);
        }
    }
    return used;
}

}

#endif
