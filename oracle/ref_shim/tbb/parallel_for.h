// Minimal stand-in for oneTBB's parallel_for over a blocked_range: a
// persistent pool of worker threads runs contiguous, equal chunks of the range.
// The reference's CPU LBM steps write each node from exactly one task and
// read only the previous state (src/aero/lbm3d/lbm3d_cpu.cpp:1-4), so their
// results do not depend on how the range is split.  Thread count: the
// ORR_REF_THREADS environment variable, else the hardware concurrency;
// tbb_shim_set_threads() changes it at run time.  Test infrastructure: used
// only to build the reference oracle under oracle/_ref.
#pragma once

#include <algorithm>
#include <condition_variable>
#include <cstddef>
#include <cstdlib>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "tbb/blocked_range.h"

namespace tbb_shim {

class Pool {
public:
    static Pool& instance() {
        static Pool pool;
        return pool;
    }

    [[nodiscard]] int threads() const { return threads_; }

    void set_threads(int n) {
        stop_workers();
        threads_ = std::max(1, n);
        start_workers();
    }

    // Runs task(k) for k in [0, parts) on the pool; the caller runs part 0.
    void run(int parts, const std::function<void(int)>& task) {
        if (parts <= 1 || workers_.empty()) {
            for (int k = 0; k < parts; ++k) {
                task(k);
            }
            return;
        }
        {
            std::unique_lock<std::mutex> lock(mutex_);
            task_ = &task;
            parts_ = parts;
            next_ = 1;
            pending_ = parts - 1;
            ++generation_;
        }
        wake_.notify_all();
        task(0);
        // Help with the remaining parts, then wait for the workers.
        for (;;) {
            int k = -1;
            {
                std::unique_lock<std::mutex> lock(mutex_);
                if (next_ < parts_) {
                    k = next_++;
                }
            }
            if (k < 0) {
                break;
            }
            task(k);
            std::unique_lock<std::mutex> lock(mutex_);
            if (--pending_ == 0) {
                done_.notify_all();
            }
        }
        std::unique_lock<std::mutex> lock(mutex_);
        done_.wait(lock, [this] { return pending_ == 0; });
        task_ = nullptr;
    }

    ~Pool() { stop_workers(); }

private:
    Pool() {
        int n = static_cast<int>(std::thread::hardware_concurrency());
        if (const char* env = std::getenv("ORR_REF_THREADS")) {
            n = std::atoi(env);
        }
        threads_ = std::max(1, n);
        start_workers();
    }

    void start_workers() {
        stopping_ = false;
        for (int t = 1; t < threads_; ++t) {
            workers_.emplace_back([this] { work(); });
        }
    }

    void stop_workers() {
        {
            std::unique_lock<std::mutex> lock(mutex_);
            stopping_ = true;
            ++generation_;
        }
        wake_.notify_all();
        for (std::thread& w : workers_) {
            w.join();
        }
        workers_.clear();
    }

    void work() {
        unsigned long seen = 0;
        for (;;) {
            const std::function<void(int)>* task = nullptr;
            int k = -1;
            {
                std::unique_lock<std::mutex> lock(mutex_);
                wake_.wait(lock, [&] { return stopping_ || generation_ != seen; });
                if (stopping_) {
                    return;
                }
                seen = generation_;
                task = task_;
                if (task != nullptr && next_ < parts_) {
                    k = next_++;
                }
            }
            while (k >= 0) {
                (*task)(k);
                std::unique_lock<std::mutex> lock(mutex_);
                if (--pending_ == 0) {
                    done_.notify_all();
                }
                k = next_ < parts_ ? next_++ : -1;
            }
        }
    }

    int threads_ = 1;
    std::vector<std::thread> workers_;
    std::mutex mutex_;
    std::condition_variable wake_;
    std::condition_variable done_;
    const std::function<void(int)>* task_ = nullptr;
    int parts_ = 0;
    int next_ = 0;
    int pending_ = 0;
    unsigned long generation_ = 0;
    bool stopping_ = false;
};

} // namespace tbb_shim

namespace tbb {

template <typename Value, typename Body>
void parallel_for(const blocked_range<Value>& range, const Body& body) {
    const Value begin = range.begin();
    const Value end = range.end();
    if (!(begin < end)) {
        return;
    }
    const auto total = static_cast<std::size_t>(end - begin);
    tbb_shim::Pool& pool = tbb_shim::Pool::instance();
    const int parts = static_cast<int>(std::min<std::size_t>(total, static_cast<std::size_t>(pool.threads())));
    const std::function<void(int)> task = [&](int k) {
        const std::size_t lo = total * static_cast<std::size_t>(k) / static_cast<std::size_t>(parts);
        const std::size_t hi = total * static_cast<std::size_t>(k + 1) / static_cast<std::size_t>(parts);
        if (lo < hi) {
            body(blocked_range<Value>(begin + static_cast<Value>(lo), begin + static_cast<Value>(hi)));
        }
    };
    pool.run(parts, task);
}

} // namespace tbb
