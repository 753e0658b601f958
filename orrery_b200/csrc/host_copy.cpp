// Staged copies between pageable host memory and device memory (host_copy.h).
//
// The ring holds kSlots chunks of kChunk bytes of pinned memory.  Chunk j of
// a copy uses slot j % kSlots.  A read-back (device to host): the calling
// thread queues the DMA of chunk j into its slot once every worker has
// emptied the slot's previous chunk, records the slot's event and posts j;
// each worker waits for the post and the event, then copies its stripe of
// the chunk to the destination.  An upload (host to device) runs the other
// way round: the workers fill a slot once the DMA of its previous chunk has
// completed (its event), and the calling thread queues the chunk's DMA when
// every worker has filled its stripe.  A failed CUDA call on any thread
// stops all of them; the error is raised on the calling thread after the
// workers have joined.
#include "host_copy.h"

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "common.h"

namespace orr {
namespace {

constexpr std::size_t kChunk = std::size_t(4) << 20;
constexpr int kSlots = 8;
constexpr int kMaxWorkers = 16;

// One staged copy at a time in the process: the ring is shared.  It is
// allocated on first use (portable, so every device's DMA can use it) and
// kept for the life of the process.
std::mutex g_ring_lock;
unsigned char* g_ring = nullptr;

unsigned char* ring() {
    if (g_ring == nullptr) {
        void* p = nullptr;
        check(cudaHostAlloc(&p, kChunk * kSlots, cudaHostAllocPortable), "pinned staging buffer");
        g_ring = static_cast<unsigned char*>(p);
    }
    return g_ring;
}

// A read-back writes the caller's arrays, usually fresh ones whose pages
// fault in on first touch: it takes a thread per core.  An upload reads
// pages that exist already; half the cores keep up with the bus.
int worker_count(bool upload) {
    const unsigned n = std::thread::hardware_concurrency();
    return static_cast<int>(std::clamp<unsigned>(upload ? n / 2 : n, 1, kMaxWorkers));
}

struct Events {
    cudaEvent_t e[kSlots] = {};
    Events() {
        for (auto& x : e) {
            check(cudaEventCreateWithFlags(&x, cudaEventDisableTiming), "staging event");
        }
    }
    ~Events() {
        for (auto x : e) {
            if (x) cudaEventDestroy(x);
        }
    }
};

// Progress shared by the calling thread and the workers.
struct Progress {
    std::mutex m;
    std::condition_variable cv;
    std::size_t posted = 0;      // chunks whose DMA is queued and event recorded
    std::vector<int> filled;     // per chunk: workers done with their stripe
    bool stop = false;
    cudaError_t error = cudaSuccess;
    const char* what = nullptr;

    void fail(cudaError_t e, const char* text) {
        std::lock_guard<std::mutex> g(m);
        if (error == cudaSuccess) {
            error = e;
            what = text;
        }
        stop = true;
        cv.notify_all();
    }
    // Waits until `ready()` holds or the copy stopped; true when ready.
    template <class F> bool wait(F&& ready) {
        std::unique_lock<std::mutex> g(m);
        cv.wait(g, [&] { return stop || ready(); });
        return !stop;
    }
    void mark_filled(std::size_t j) {
        std::lock_guard<std::mutex> g(m);
        ++filled[j];
        cv.notify_all();
    }
    void post(std::size_t j) {
        std::lock_guard<std::mutex> g(m);
        posted = j + 1;
        cv.notify_all();
    }
};

// Stripe [a, b) of a chunk of `len` bytes for worker t of n (64-byte aligned
// boundaries, so workers never share a cache line).
void stripe(std::size_t len, int t, int n, std::size_t& a, std::size_t& b) {
    const std::size_t part = ((len + n - 1) / n + 63) & ~std::size_t(63);
    a = std::min(len, part * t);
    b = std::min(len, a + part);
}

// Chunk j of a copy: `len` bytes at `device` and at `host` (2 * len there
// for a widening chunk).
struct Chunk {
    unsigned char* host;
    unsigned char* device;
    std::size_t len;
    bool widen = false;
    double add = 0.0;
};

// Binary32 values [a, b) (byte offsets) of a staged chunk to the host as
// binary64 plus `add`.
void widen_stripe(const Chunk& c, const unsigned char* from, std::size_t a, std::size_t b) {
    const auto* src = reinterpret_cast<const float*>(from + a);
    auto* dst = reinterpret_cast<double*>(c.host + 2 * a);
    const std::size_t n = (b - a) / sizeof(float);
    for (std::size_t k = 0; k < n; ++k) {
        dst[k] = static_cast<double>(src[k]) + c.add;
    }
}

void staged(bool upload, const std::vector<Chunk>& chunks, cudaStream_t stream, int device) {
    std::lock_guard<std::mutex> hold(g_ring_lock);
    unsigned char* slots = ring();
    Events ev;
    const std::size_t n = chunks.size();
    const int nworkers = worker_count(upload);
    Progress pr;
    pr.filled.assign(n, 0);
    const auto slot = [&](std::size_t j) { return slots + (j % kSlots) * kChunk; };

    auto worker = [&](int t) {
        const cudaError_t e = cudaSetDevice(device);
        if (e != cudaSuccess) {
            pr.fail(e, "cudaSetDevice");
            return;
        }
        for (std::size_t j = 0; j < n; ++j) {
            std::size_t a = 0, b = 0;
            stripe(chunks[j].len, t, nworkers, a, b);
            if (upload) {
                // The slot is free once the DMA of chunk j - kSlots is done.
                if (j >= static_cast<std::size_t>(kSlots)) {
                    if (!pr.wait([&] { return pr.posted > j - kSlots; })) {
                        return;
                    }
                    const cudaError_t s = cudaEventSynchronize(ev.e[j % kSlots]);
                    if (s != cudaSuccess) {
                        pr.fail(s, "staged upload");
                        return;
                    }
                }
                std::memcpy(slot(j) + a, chunks[j].host + a, b - a);
            } else {
                if (!pr.wait([&] { return pr.posted > j; })) {
                    return;
                }
                const cudaError_t s = cudaEventSynchronize(ev.e[j % kSlots]);
                if (s != cudaSuccess) {
                    pr.fail(s, "staged read-back");
                    return;
                }
                if (chunks[j].widen) {
                    widen_stripe(chunks[j], slot(j), a, b);
                } else {
                    std::memcpy(chunks[j].host + a, slot(j) + a, b - a);
                }
            }
            pr.mark_filled(j);
        }
    };

    std::vector<std::thread> threads;
    threads.reserve(nworkers);
    try {
        for (int t = 0; t < nworkers; ++t) {
            threads.emplace_back(worker, t);
        }
    } catch (...) {
        pr.fail(cudaErrorUnknown, "staging threads");
        for (auto& th : threads) th.join();
        throw;
    }
    for (std::size_t j = 0; j < n; ++j) {
        if (upload) {
            if (!pr.wait([&] { return pr.filled[j] == nworkers; })) {
                break;
            }
        } else if (j >= static_cast<std::size_t>(kSlots)) {
            if (!pr.wait([&] { return pr.filled[j - kSlots] == nworkers; })) {
                break;
            }
        }
        const Chunk& c = chunks[j];
        cudaError_t e = upload ? cudaMemcpyAsync(c.device, slot(j), c.len, cudaMemcpyHostToDevice, stream)
                               : cudaMemcpyAsync(slot(j), c.device, c.len, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) {
            e = cudaEventRecord(ev.e[j % kSlots], stream);
        }
        if (e != cudaSuccess) {
            pr.fail(e, upload ? "staged upload" : "staged read-back");
            break;
        }
        pr.post(j);
    }
    for (auto& th : threads) th.join();
    if (pr.error == cudaSuccess && upload && n > 0) {
        // The DMAs run in stream order: the last one's event covers them all.
        const cudaError_t e = cudaEventSynchronize(ev.e[(n - 1) % kSlots]);
        if (e != cudaSuccess) {
            pr.fail(e, "staged upload");
        }
    }
    if (pr.error != cudaSuccess) {
        // Nothing may still read or write the ring when it is released.
        cudaStreamSynchronize(stream);
        throw CudaError{pr.error, pr.what};
    }
}

void copy(bool upload, const HostSpan* spans, int count, cudaStream_t stream, int device) {
    std::size_t total = 0;
    bool widen = false;
    for (int k = 0; k < count; ++k) {
        total += spans[k].bytes;
        if (spans[k].widen) {
            if (upload || spans[k].bytes % sizeof(float) != 0) {
                throw CudaError{cudaErrorInvalidValue, "widening copy (read-backs of binary32 values only)"};
            }
            widen = true;
        }
    }
    // Widening spans always take the ring: the host threads do the widening.
    if (total < kStagedCopyBytes && !widen) {
        const char* what = upload ? "upload" : "read-back";
        for (int k = 0; k < count; ++k) {
            const HostSpan& s = spans[k];
            if (s.bytes > 0) {
                check(upload ? cudaMemcpyAsync(s.device, s.host, s.bytes, cudaMemcpyHostToDevice, stream)
                             : cudaMemcpyAsync(s.host, s.device, s.bytes, cudaMemcpyDeviceToHost, stream),
                      what);
            }
        }
        check(cudaStreamSynchronize(stream), what);
        return;
    }
    std::vector<Chunk> chunks;
    chunks.reserve(total / kChunk + count);
    for (int k = 0; k < count; ++k) {
        auto* h = static_cast<unsigned char*>(spans[k].host);
        auto* d = static_cast<unsigned char*>(spans[k].device);
        const std::size_t scale = spans[k].widen ? 2 : 1;
        for (std::size_t off = 0; off < spans[k].bytes; off += kChunk) {
            chunks.push_back(Chunk{h + scale * off, d + off, std::min(kChunk, spans[k].bytes - off), spans[k].widen,
                                   spans[k].add});
        }
    }
    staged(upload, chunks, stream, device);
}

} // namespace

void copy_to_device(const HostSpan* spans, int count, cudaStream_t stream, int device) {
    copy(true, spans, count, stream, device);
}

void copy_to_host(const HostSpan* spans, int count, cudaStream_t stream, int device) {
    copy(false, spans, count, stream, device);
}

} // namespace orr
