// Host-only stand-in for the few CUDA runtime calls of the staged host
// transfers (orrery_b200/csrc/host_copy.cpp), for testing their pipeline on
// a machine without a GPU.  A stream is a worker thread that runs its queued
// operations in order, each copy after a short random delay, so an event
// completes only when the work queued before it has run, as on a device.
// Failures can be injected into the n-th event wait or copy call.
#pragma once

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <mutex>
#include <random>
#include <thread>

typedef int cudaError_t;
enum : int {
    cudaSuccess = 0,
    cudaErrorInvalidValue = 1,
    cudaErrorMemoryAllocation = 2,
    cudaErrorInsufficientDriver = 35,
    cudaErrorNoDevice = 100,
    cudaErrorLaunchFailure = 719,
    cudaErrorUnknown = 999,
};
enum cudaMemcpyKind { cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2 };
inline constexpr unsigned cudaEventDisableTiming = 2;
inline constexpr unsigned cudaHostAllocPortable = 1;

namespace fake {

// Calls left before an injected failure (negative: none).
inline std::atomic<long> fail_event_wait{-1};
inline std::atomic<long> fail_copy{-1};

inline bool trips(std::atomic<long>& counter) {
    long v = counter.load();
    while (v >= 0) {
        if (counter.compare_exchange_weak(v, v - 1)) {
            return v == 0;
        }
    }
    return false;
}

inline void jitter(unsigned scale_us) {
    thread_local std::mt19937 g(std::random_device{}());
    if (g() % 3 == 0) {
        std::this_thread::sleep_for(std::chrono::microseconds(g() % scale_us));
    }
}

struct Stream {
    std::mutex m;
    std::condition_variable cv;
    std::deque<std::function<void()>> ops;
    std::size_t queued = 0, finished = 0;
    bool stop = false;
    std::thread runner;

    Stream() : runner([this] { run(); }) {}
    ~Stream() {
        {
            std::lock_guard<std::mutex> g(m);
            stop = true;
        }
        cv.notify_all();
        runner.join();
    }
    void push(std::function<void()> op) {
        {
            std::lock_guard<std::mutex> g(m);
            ops.push_back(std::move(op));
            ++queued;
        }
        cv.notify_all();
    }
    void drain() {
        std::unique_lock<std::mutex> g(m);
        cv.wait(g, [&] { return finished == queued; });
    }
    void run() {
        for (;;) {
            std::function<void()> op;
            {
                std::unique_lock<std::mutex> g(m);
                cv.wait(g, [&] { return stop || !ops.empty(); });
                if (ops.empty()) {
                    return;
                }
                op = std::move(ops.front());
                ops.pop_front();
            }
            op();
            {
                std::lock_guard<std::mutex> g(m);
                ++finished;
            }
            cv.notify_all();
        }
    }
};

struct Event {
    std::mutex m;
    std::condition_variable cv;
    std::size_t recorded = 0, reached = 0;
};

} // namespace fake

typedef fake::Stream* cudaStream_t;
typedef fake::Event* cudaEvent_t;

inline cudaError_t cudaSetDevice(int) { return cudaSuccess; }

inline cudaError_t cudaHostAlloc(void** p, std::size_t n, unsigned) {
    *p = std::malloc(n);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}

inline cudaError_t cudaEventCreateWithFlags(cudaEvent_t* e, unsigned) {
    *e = new fake::Event;
    return cudaSuccess;
}

inline cudaError_t cudaEventDestroy(cudaEvent_t e) {
    delete e;
    return cudaSuccess;
}

inline cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t s) {
    std::size_t mark;
    {
        std::lock_guard<std::mutex> g(e->m);
        mark = ++e->recorded;
    }
    s->push([e, mark] {
        // Notified under the lock: a waiter returns (and may destroy the
        // event) only after this operation is done with it.
        std::lock_guard<std::mutex> g(e->m);
        e->reached = mark;
        e->cv.notify_all();
    });
    return cudaSuccess;
}

inline cudaError_t cudaEventSynchronize(cudaEvent_t e) {
    if (fake::trips(fake::fail_event_wait)) {
        return cudaErrorLaunchFailure;
    }
    fake::jitter(100);
    std::unique_lock<std::mutex> g(e->m);
    const std::size_t mark = e->recorded;
    e->cv.wait(g, [&] { return e->reached >= mark; });
    return cudaSuccess;
}

inline cudaError_t cudaMemcpyAsync(void* dst, const void* src, std::size_t n, cudaMemcpyKind, cudaStream_t s) {
    if (fake::trips(fake::fail_copy)) {
        return cudaErrorInvalidValue;
    }
    s->push([dst, src, n] {
        fake::jitter(300);
        std::memcpy(dst, src, n);
    });
    return cudaSuccess;
}

inline cudaError_t cudaStreamSynchronize(cudaStream_t s) {
    s->drain();
    return cudaSuccess;
}
