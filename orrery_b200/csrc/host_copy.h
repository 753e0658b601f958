// Large copies between pageable host memory and device memory.
//
// A plain cudaMemcpy from or to pageable memory runs at the speed of one
// host thread: the driver stages the data through its own pinned buffer,
// and a destination freshly allocated by the caller (the usual case for the
// read-back arrays) also takes its page faults on that one thread.  Copies
// of at least kStagedCopyBytes in all go through a process-wide ring of
// pinned chunks instead: host threads copy their stripes of one chunk while the
// DMA engine moves the next, so the host side runs on several cores and
// overlaps the bus transfer.  Smaller copies take the plain call.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace orr {

inline constexpr std::size_t kStagedCopyBytes = std::size_t(8) << 20;

// One contiguous range of a copy: `bytes` at `host` and at `device`.  A
// widening span (read-backs only) holds binary32 values on the device
// (`bytes` of them) and receives them on the host as binary64 values plus
// `add` (2 * bytes at `host`): the host threads widen while they copy, so
// the bus moves half the bytes.
struct HostSpan {
    void* host;
    void* device;
    std::size_t bytes;
    bool widen = false;
    double add = 0.0;
};

// Copies every span (host to device, or device to host) as one pipeline and
// returns when all are complete (the host buffers may be reused or read),
// with work queued earlier on `stream` ordered before the copies.  Errors
// throw CudaError.  `device` is the device of `stream`.
void copy_to_device(const HostSpan* spans, int count, cudaStream_t stream, int device);
void copy_to_host(const HostSpan* spans, int count, cudaStream_t stream, int device);

} // namespace orr
