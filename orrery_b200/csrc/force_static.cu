// orr_lbm3d_force_static: the momentum-exchange force and moment of a D3Q19
// lattice computed without allocating device memory.
//
// Some callers cannot allocate device memory: an application whose device
// memory is owned by its own allocator or pool, a real-time loop that must
// not enter the allocator, a process that reserved all device memory up
// front.  For them the reduction's scratch lives in a file-scope device
// array of fixed size, compiled into the library, instead of a buffer from
// cudaMalloc.  The caller passes the populations and the link tables it holds
// on the device and receives the six doubles on the host.
//
// Two passes, both in a fixed order, so the result is the same every call:
//   pass 1  block b sums the links [b * kChunk, (b + 1) * kChunk) in binary64
//           and writes its six partial sums to slot b of the scratch array;
//   pass 2  one block adds the partial sums of all slots in slot order and
//           writes the six totals to the last slot.
// Every slot pass 2 reads is written by pass 1 of the same call; the one
// value that must start at zero, the flag a link outside the lattice raises
// (such links are skipped: the tables come from the caller), is cleared by a
// memset of the array at the start of each call.  A call's contents stay in
// the array until the next call overwrites them.  Calls that overlap on the
// GPU race on the array; callers serialise them (one stream, or one call at
// a time).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "common.h"
#include "kernels3d.cuh"
#include "lattice.h"
#include "plan.h"

namespace {

using namespace orr;

constexpr unsigned kThreads = 256;
constexpr uint64_t kChunk = 2048;                      // links per block of pass 1
constexpr uint64_t kSlots = ORR_FORCE_STATIC_MAX_LINKS / kChunk;  // 4096 partial-sum slots
static_assert(kSlots * kChunk == ORR_FORCE_STATIC_MAX_LINKS, "whole chunks");

// 4096 slots of 6 partial sums, the slot of the totals and the flag slot
// (its first value is set when a link of the caller's tables is out of
// range): 196,704 bytes.
__device__ __align__(256) double g_force_scratch[(kSlots + 2) * 6];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch_address[kMaxDevices] = {};

// Device address of the scratch array on `device` (current), looked up once.
double* scratch_on(int device) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_address[device] == nullptr) {
        void* ptr = nullptr;
        check(cudaGetSymbolAddress(&ptr, g_force_scratch), "cudaGetSymbolAddress of the force scratch");
        g_scratch_address[device] = static_cast<double*>(ptr);
    }
    return g_scratch_address[device];
}

// Sum of six doubles over the block in a fixed order (shuffle tree, then
// warp partials in warp order); the result is valid in thread 0.
__device__ void block_sum6(double (&v)[6]) {
    __shared__ double part[6][kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) part[k][warp] = v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            double s = 0.0;
            for (int w = 0; w < static_cast<int>(kThreads / 32); ++w) s += part[k][w];
            v[k] = s;
        }
    }
}

// Pass 1: the links of chunk blockIdx.x (add_link3, the solver's per-link
// routine, with the caller's tables checked: a link whose cell, direction or
// interpolation source lies outside the lattice is skipped and raises the
// flag slot).
template <class S>
__global__ void __launch_bounds__(kThreads) force_static_partials(
    uint64_t nx, uint64_t ny, uint64_t cells, const S* __restrict__ f,
    const uint32_t* __restrict__ lcell, const uint32_t* __restrict__ ldir,
    const double* __restrict__ lq, uint64_t links, double* __restrict__ scratch) {
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const uint64_t begin = static_cast<uint64_t>(blockIdx.x) * kChunk;
    const uint64_t end = begin + kChunk < links ? begin + kChunk : links;
    const uint64_t plane = nx * ny;
    bool bad = false;
    for (uint64_t k = begin + threadIdx.x; k < end; k += kThreads) {
        if (!add_link3<S, true>(nx, plane, cells, f, lcell[k], static_cast<int>(ldir[k]), lq[k], acc)) {
            bad = true;
        }
    }
    if (bad) {
        scratch[(kSlots + 1) * 6] = 1.0;
    }
    block_sum6(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int v = 0; v < 6; ++v) scratch[static_cast<uint64_t>(blockIdx.x) * 6 + v] = acc[v];
    }
}

// Pass 2: the totals of `used` slots into slot kSlots.
__global__ void __launch_bounds__(kThreads) force_static_total(uint64_t used, double* __restrict__ scratch) {
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (uint64_t s = threadIdx.x; s < used; s += kThreads) {
#pragma unroll
        for (int v = 0; v < 6; ++v) acc[v] += scratch[s * 6 + v];
    }
    block_sum6(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int v = 0; v < 6; ++v) scratch[kSlots * 6 + v] = acc[v];
    }
}

template <class S>
void launch_partials(const orr_force_links& a, cudaStream_t s, unsigned blocks, double* scratch) {
    force_static_partials<S><<<blocks, kThreads, 0, s>>>(
        a.nx, a.ny, a.nx * a.ny * a.nz, static_cast<const S*>(a.populations), a.link_cell, a.link_dir,
        a.link_q, a.links, scratch);
}

} // namespace

extern "C" orr_status orr_lbm3d_force_static(const orr_force_links* args, double force_moment[6]) {
    return orr::guarded(nullptr, [&]() -> orr_status {
        if (args == nullptr || force_moment == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d force_static: null argument"};
        }
        const orr_force_links& a = *args;
        if (a.links > ORR_FORCE_STATIC_MAX_LINKS) {
            throw Refusal{ORR_ERR_INVALID,
                          "lbm3d force_static: " + std::to_string(a.links) + " links exceed the " +
                              std::to_string(ORR_FORCE_STATIC_MAX_LINKS) +
                              " the fixed scratch array holds; use orr_lbm3d_force"};
        }
        uint64_t plane = 0, cells = 0;
        if (a.nx < 1 || a.ny < 1 || a.nz < 1 || a.nx > kMaxGridCells || a.ny > kMaxGridCells ||
            a.nz > kMaxGridCells || __builtin_mul_overflow(a.nx, a.ny, &plane) ||
            __builtin_mul_overflow(plane, a.nz, &cells) || cells > kMaxGridCells) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d force_static: lattice dimensions out of range"};
        }
        if (a.storage < ORR_STORAGE_F32 || a.storage > ORR_STORAGE_F64) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d force_static: unknown population storage"};
        }
        if (a.device < 0 || a.device >= kMaxDevices) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d force_static: device ordinal out of range"};
        }
        if (a.links > 0 && (a.populations == nullptr || a.link_cell == nullptr ||
                            a.link_dir == nullptr || a.link_q == nullptr)) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d force_static: null device pointer"};
        }
        check(cudaSetDevice(a.device), "cudaSetDevice");
        double* scratch = scratch_on(a.device);
        if (a.links == 0) {
            std::memset(force_moment, 0, 6 * sizeof(double));
            return ORR_OK;
        }
        cudaStream_t s = static_cast<cudaStream_t>(a.stream);
        const unsigned blocks = static_cast<unsigned>((a.links + kChunk - 1) / kChunk);
        // The flag slot starts clear; the totals and the flag come back in
        // one copy.
        check(cudaMemsetAsync(scratch + (kSlots + 1) * 6, 0, sizeof(double), s), "force_static flag");
        switch (a.storage) {
            case ORR_STORAGE_F16:
                launch_partials<__half>(a, s, blocks, scratch);
                break;
            case ORR_STORAGE_BF16:
                launch_partials<__nv_bfloat16>(a, s, blocks, scratch);
                break;
            case ORR_STORAGE_F64:
                launch_partials<double>(a, s, blocks, scratch);
                break;
            default:
                launch_partials<float>(a, s, blocks, scratch);
                break;
        }
        check(cudaGetLastError(), "force_static partial sums");
        force_static_total<<<1, kThreads, 0, s>>>(blocks, scratch);
        check(cudaGetLastError(), "force_static total");
        double result[7];
        check(cudaMemcpyAsync(result, scratch + kSlots * 6, 7 * sizeof(double), cudaMemcpyDeviceToHost, s),
              "force_static read-back");
        check(cudaStreamSynchronize(s), "force_static read-back");
        if (result[6] != 0.0) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d force_static: a link's cell, direction or interpolation "
                                           "source lies outside the lattice"};
        }
        std::memcpy(force_moment, result, 6 * sizeof(double));
        return ORR_OK;
    });
}
