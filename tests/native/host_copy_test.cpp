// Pipeline test of the staged host transfers (orrery_b200/csrc/host_copy.cpp)
// against the host-only CUDA stand-in under fake_cuda/: random span lists
// (empty spans, ragged chunk tails, totals on both sides of the staging
// threshold) go up and come back byte for byte through an asynchronous
// "device"; injected failures of event waits and copies end the copy with
// the error on the calling thread, and the next copy still works.
// Prints "ok" and exits 0 on success.
#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

#include "common.h"
#include "host_copy.h"

namespace {

int round_trips(std::mt19937_64& g, fake::Stream& s, int trials) {
    for (int trial = 0; trial < trials; ++trial) {
        const int n = 1 + static_cast<int>(g() % 4);
        std::vector<std::vector<uint8_t>> host(n), dev(n), back(n);
        std::vector<orr::HostSpan> up(n), down(n);
        for (int k = 0; k < n; ++k) {
            std::size_t bytes = 0;
            switch (g() % 4) {
            case 0: bytes = 0; break;
            case 1: bytes = g() % 5000; break;
            case 2: bytes = (std::size_t(4) << 20) * (1 + g() % 3) + g() % 3; break;
            default: bytes = g() % (std::size_t(24) << 20); break;
            }
            host[k].resize(bytes);
            for (auto& b : host[k]) b = static_cast<uint8_t>(g());
            dev[k].assign(bytes, 0);
            back[k].assign(bytes, 0);
            up[k] = {host[k].data(), dev[k].data(), bytes};
            down[k] = {back[k].data(), dev[k].data(), bytes};
        }
        orr::copy_to_device(up.data(), n, &s, 0);
        for (int k = 0; k < n; ++k) {
            if (dev[k] != host[k]) {
                std::printf("upload differs: trial %d span %d\n", trial, k);
                return 1;
            }
        }
        orr::copy_to_host(down.data(), n, &s, 0);
        for (int k = 0; k < n; ++k) {
            if (back[k] != host[k]) {
                std::printf("read-back differs: trial %d span %d\n", trial, k);
                return 1;
            }
        }
    }
    return 0;
}

int failures(fake::Stream& s) {
    const std::size_t bytes = std::size_t(37) << 20;    // ten chunks, a ragged tail
    std::vector<uint8_t> a(bytes, 7), b(bytes, 0);
    int raised = 0;
    for (int k = 0; k < 24; ++k) {
        if (k % 2 == 0) {
            fake::fail_event_wait = k % 11;
        } else {
            fake::fail_copy = k % 7;
        }
        orr::HostSpan span{a.data(), b.data(), bytes};
        try {
            if (k % 4 < 2) {
                orr::copy_to_device(&span, 1, &s, 0);
            } else {
                orr::copy_to_host(&span, 1, &s, 0);
            }
        } catch (const orr::CudaError& e) {
            ++raised;
        }
        fake::fail_event_wait = -1;
        fake::fail_copy = -1;
    }
    if (raised == 0) {
        std::printf("no injected failure was raised\n");
        return 1;
    }
    // The ring is free again and a copy completes.
    std::fill(b.begin(), b.end(), 0);
    orr::HostSpan span{a.data(), b.data(), bytes};
    orr::copy_to_device(&span, 1, &s, 0);
    if (b != a) {
        std::printf("copy after failures differs\n");
        return 1;
    }
    return 0;
}

// Widening read-backs: binary32 values on the "device" come back as binary64
// plus the span's offset, exactly, for spans on both sides of the staging
// threshold and ragged chunk tails; a widening upload is refused.
int widening(std::mt19937_64& g, fake::Stream& s) {
    std::uniform_real_distribution<float> value(-2.0f, 2.0f);
    for (int trial = 0; trial < 12; ++trial) {
        const int n = 1 + static_cast<int>(g() % 4);
        std::vector<std::vector<float>> dev(n);
        std::vector<std::vector<double>> back(n);
        std::vector<orr::HostSpan> down(n);
        for (int k = 0; k < n; ++k) {
            std::size_t count = 0;
            switch (g() % 3) {
            case 0: count = g() % 3000; break;
            case 1: count = (std::size_t(1) << 20) * (1 + g() % 3) + g() % 5; break;
            default: count = g() % (std::size_t(6) << 20); break;
            }
            dev[k].resize(count);
            for (auto& v : dev[k]) v = value(g);
            back[k].assign(count, -7.0);
            const double add = k % 2 == 0 ? 1.0 : 0.0;
            down[k] = {back[k].data(), dev[k].data(), count * sizeof(float), true, add};
        }
        orr::copy_to_host(down.data(), n, &s, 0);
        for (int k = 0; k < n; ++k) {
            for (std::size_t i = 0; i < dev[k].size(); ++i) {
                if (back[k][i] != static_cast<double>(dev[k][i]) + down[k].add) {
                    std::printf("widening differs: trial %d span %d value %zu\n", trial, k, i);
                    return 1;
                }
            }
        }
    }
    std::vector<float> d(16, 1.0f);
    std::vector<double> h(16, 0.0);
    orr::HostSpan up{h.data(), d.data(), d.size() * sizeof(float), true, 0.0};
    try {
        orr::copy_to_device(&up, 1, &s, 0);
        std::printf("a widening upload was accepted\n");
        return 1;
    } catch (const orr::CudaError&) {
    }
    return 0;
}

} // namespace

int main() {
    std::mt19937_64 g(12345);
    fake::Stream s;
    if (round_trips(g, s, 24) != 0 || failures(s) != 0 || widening(g, s) != 0) {
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
