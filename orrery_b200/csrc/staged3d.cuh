// Persistent D3Q19 step over one or many lattices, with the source rows of
// every interior row tile staged in shared memory by bulk asynchronous
// copies (cp.async.bulk, completion on an mbarrier).
//
// The kernel serves lattices with g.flat set (periodic or free-slip sides,
// halfway walls), whose every pull is one stored value.
//
// Work items.
//   staged items   spans of N = NPT * B consecutive nodes (flattened order) of
//                  the interior rows (1 <= y <= ny-2) of an interior z-plane
//                  (1 <= z <= nz-2), for lattices whose rows are 16-node
//                  aligned.  The pull sources of a span are contiguous in
//                  every population plane: plane i needs
//                  f*_i([c0 - o_i - H, c0 - o_i + N + H)), o_i = cx_i + nx cy_i +
//                  nx ny cz_i, so one bulk copy per plane (the halo H covers
//                  cx = +-1) and one for the span's class bytes fill a
//                  pipeline stage.  A span may cover several short rows or
//                  part of a long one; x-edge nodes take their fix-ups.
//   direct items   every other row, in tiles of B nodes (the y and z face
//                  rows, and all rows of a lattice that cannot be staged):
//                  the per-node gather of step_node3 from global memory.
// Items of all lattices are numbered globally (prefix offsets in the lattice
// table) and CTA b takes items b, b + G, b + 2G, ... so that the CTAs in
// flight work on neighbouring spans, as a one-shot grid would.
//
// Pipeline.  A CTA has B consumer threads and one producer warp.  The
// producer keeps up to `stages` items in flight: for each it waits until
// every consumer warp has released the stage (the stage's empty mbarrier),
// records the item, arms the stage's full mbarrier with the byte count, and
// its lanes 0-18 copy one population plane's segment each, lane 19 the
// class bytes.  Each consumer thread owns NPT nodes of the span (k = tid +
// p B): it waits for the full barrier, and for each node reads the 19 values
// and the class into registers and finishes the node; after its last
// node's reads its warp releases the stage (one arrive per warp on the empty
// barrier).  Consumer warps never wait for each other.  The finish is the one of step_node3
// (x-edge fix-ups, bounce-back overrides from global memory for the rare
// boundary nodes, inlet, collision, 19 stores), so a node's arithmetic does
// not depend on which item or lattice mix carried it.
//
// Every wait is bounded: a barrier that does not complete within the limit
// sets kStatusWaitTimeout in the status word and the CTA's abort word, every
// warp leaves its loop, and the CTA waits (bounded again) for the copies it
// still has in flight before it returns.
//
// The word after the status word is the stall request that tests of this
// path set (0 when none): a CTA whose index + 1 it holds, and that has a
// staged span, clears it and withholds the copies of its first span, so that
// its consumers' bounded wait runs out exactly as when a copy never lands.
#pragma once

#include <cstdint>

#include "kernels3d.cuh"
#include "plan.h"

namespace orr {

constexpr uint32_t kStatusWaitTimeout = 1u;
constexpr uint32_t kMaxStages = 8;
// Shared header: full barriers (64 B), empty barriers (64 B), item records
// (128 B), the abort word and the issued-item count.
constexpr uint32_t kStagedHeader = 384;

// One lattice of a persistent step (entries are built on the host,
// lattice_table.cuh).
template <class A> struct Lattice3D {
    Geom3D g;              // g.tiles_x is ceil(nx / B) of the launch's B
    Phys3D<A> p;
    StepBuffers3D b;
    void* f[2];            // population buffers
    uint32_t parity;       // f[parity ^ flip] is the source of a step launched with `flip`
    uint32_t staged;       // interior rows go through shared memory
    uint64_t staged_begin; // first global staged item of this lattice
    uint64_t direct_begin; // first global direct item of this lattice
    uint32_t spans;        // staged spans per interior z-plane
    uint32_t magic;        // ceil(2^32 / nx) when nx <= kMagicMaxNx (exact quotients n / nx, n < 2^16), else 0
};

// Shared memory of one pipeline stage: 19 segments of N + 2H values, then N
// class bytes (every piece starts on a 16-byte boundary), N = NPT * B.
template <class S> constexpr int kHalo = 16 / static_cast<int>(sizeof(S));
template <class S, int N> constexpr uint32_t kSegment = N + 2 * kHalo<S>;
template <class S, int N> constexpr uint32_t kPopBytes = d3::Q * kSegment<S, N> * sizeof(S);
template <class S, int N> constexpr uint32_t kStageBytes = kPopBytes<S, N> + N;

template <class S, int N> constexpr uint32_t staged_smem_bytes(uint32_t stages) {
    return kStagedHeader + stages * kStageBytes<S, N>;
}

// Threads of a staged CTA: B consumers and one producer warp.
template <int B> constexpr int kStagedThreads = B + 32;

// The largest nx with exact multiply-high quotients of span offsets: for
// n < 2^16 and nx < 2^16, floor(n / nx) = umulhi(n, ceil(2^32 / nx)); span
// offsets reach nx + N with N <= 1024.
constexpr uint32_t kMagicMaxNx = 65536u - 1024u;

// ----------------------------------------------------------- PTX helpers --

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrive once and add `bytes` to the transactions the phase waits for.
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

// One poll of the phase of `parity`; if it has not completed, the thread may
// sleep until it completes or about kSuspendNs nanoseconds pass (the hint of
// mbarrier.try_wait), instead of spinning on the barrier.
constexpr uint32_t kSuspendNs = 20000;
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity), "n"(kSuspendNs)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Waits for the phase of `parity` to complete, giving up after a bounded
// number of polls (each sleeps at most kSuspendNs: about 1.3 s in all) or
// when another warp has raised the CTA's abort word.
constexpr uint32_t kWaitPolls = 1u << 16;
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity,
                                                  const volatile uint32_t* abort_word) {
    if (mbar_try_wait(bar, parity)) {
        return true;
    }
    for (uint32_t k = 0; k < kWaitPolls; ++k) {
        if (*abort_word != 0u) {
            return false;
        }
        if (mbar_try_wait(bar, parity)) {
            return true;
        }
    }
    return false;
}

// Global -> shared bulk copy completing on `bar` (addresses and size are
// multiples of 16 bytes).
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}

// --------------------------------------------------------------- items --

// The lattice holding global item k: the last one whose first item is <= k
// (lattices without items of the kind share their successor's offset).
template <class A, bool kStaged>
__device__ __forceinline__ uint32_t find_lattice(const Lattice3D<A>* __restrict__ lats, uint32_t n,
                                                 uint64_t k) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint64_t begin = kStaged ? lats[mid].staged_begin : lats[mid].direct_begin;
        if (begin <= k) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// Row of direct item r of a lattice: the face rows (z = 0, z = nz - 1, then
// y = 0 and y = ny - 1 of the inner z) when its interior is staged, else
// every row.
__device__ __forceinline__ void direct_row(const Geom3D& g, bool staged, uint64_t r, uint32_t& y,
                                           uint32_t& z) {
    if (!staged) {
        y = static_cast<uint32_t>(r % g.ny);
        z = static_cast<uint32_t>(r / g.ny);
        return;
    }
    const uint32_t ny = g.ny, nz = g.nz;
    const uint32_t q = static_cast<uint32_t>(r);
    if (q < ny) {
        y = q;
        z = 0;
    } else if (q < 2 * ny) {
        y = q - ny;
        z = nz - 1;
    } else if (q < 2 * ny + (nz - 2)) {
        y = 0;
        z = 1 + (q - 2 * ny);
    } else {
        y = ny - 1;
        z = 1 + (q - 2 * ny - (nz - 2));
    }
}

// --------------------------------------------------------- node finish --

// Finish of a staged node: f holds the 19 plain pulls of the node, and for a
// bulk node at the outlet (x = nx - 1, inflow / outflow) already the
// zero-gradient copies of its c_x < 0 directions (the consumer loop takes
// them from the stage).
template <class S, bool kSmag>
__device__ __forceinline__ void staged_node3(const Geom3D& g, const Phys3D<typename Storage<S>::A>& p,
                                             const StepBuffers3D& b, const S* __restrict__ src,
                                             S* __restrict__ dst, typename Storage<S>::A (&f)[d3::Q],
                                             uint8_t cls, uint32_t x, uint32_t y, uint32_t z) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    const uint64_t here = x + static_cast<uint64_t>(g.nx) * (y + static_cast<uint64_t>(g.ny) * z);
    if (cls == kSolid) {
#pragma unroll
        for (int i = 0; i < d3::Q; ++i) {
            T::store(dst + static_cast<uint64_t>(i) * g.cells + here, T::kShifted ? A(0) : A(d3::w(i)));
        }
        return;
    }
    if (cls == kBoundary) {
        const uint32_t mask = b.nmask[here];
        if (x == 0u || x + 1u == g.nx) {
            gather_flat3<S>(g, src, mask, static_cast<int>(x), static_cast<int>(y), static_cast<int>(z), here, f);
            if (x + 1u == g.nx && g.x_mode == ORR_X_INFLOW_OUTFLOW) {
                convective_blend3<S>(g, p, b, y, z, f);
            }
        } else {
            // Halfway bounce-back: the staged pull of every solid-source
            // direction is replaced by f*_opp at the node (independent loads).
#pragma unroll
            for (int i = 0; i < d3::Q; ++i) {
                if ((mask >> i) & 1u) {
                    f[i] = T::load(src + static_cast<uint64_t>(d3::opposite(i)) * g.cells + here);
                }
            }
        }
    } else if (x + 1u == g.nx && g.x_mode == ORR_X_INFLOW_OUTFLOW) {
        convective_blend3<S>(g, p, b, y, z, f);
    } else {
        bulk_edges3<S>(g, p, src, b, x, y, z, here, f);
    }
    if (g.x_mode == ORR_X_INFLOW_OUTFLOW && x == 0u) {
        inlet_west3<A, T::kShifted>(f, static_cast<const A*>(b.inlet));
    }
    finish3<S, kSmag>(g, p, b, f, x, y, z, here, dst);
}

// ---------------------------------------------------------------- kernel --

template <class S, int B> constexpr int kStagedMinBlocks =
    sizeof(typename Storage<S>::A) == 8 ? (B == 256 ? 2 : 3) : (B == 256 ? 3 : 6);

// The staged step.  kSingle: the one lattice is the by-value parameter `one`
// (its fields are constant-bank operands); otherwise lattices come from the
// device table `lats` of n entries.  B consumer threads, NPT nodes each per
// span; warp B/32 produces (waits until every consumer warp has released
// stage j % stages, records span j, arms the full barrier with the stage's
// bytes and issues its 20 bulk copies).  No block-wide barrier in the loop.
template <class S, bool kSmag, int B, int NPT, bool kSingle>
__global__ void __launch_bounds__(kStagedThreads<B>, kStagedMinBlocks<S, B>)
    step3d_staged_kernel(const __grid_constant__ Lattice3D<typename Storage<S>::A> one,
                         const Lattice3D<typename Storage<S>::A>* __restrict__ lats, uint32_t n,
                         uint32_t staged_total, uint32_t direct_total, uint32_t flip, uint32_t stages,
                         uint32_t* __restrict__ status) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    constexpr int H = kHalo<S>;
    constexpr uint32_t N = static_cast<uint32_t>(B * NPT);
    constexpr uint32_t SEG = kSegment<S, N>;
    constexpr uint32_t POP = kPopBytes<S, N>;
    constexpr uint32_t STAGE = kStageBytes<S, N>;
    constexpr uint32_t kConsumerWarps = B / 32;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = reinterpret_cast<uint64_t*>(smem + 64);
    uint4* info = reinterpret_cast<uint4*>(smem + 128);
    volatile uint32_t* abort_word = reinterpret_cast<volatile uint32_t*>(smem + 256);
    volatile uint32_t* issued_word = reinterpret_cast<volatile uint32_t*>(smem + 260);
    unsigned char* ring = smem + kStagedHeader;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    const uint32_t warp = tid >> 5;
    // Entries: the by-value parameter (its address is in the constant
    // bank) or the device table.
    const Lattice3D<A>* const table = kSingle ? &one : lats;

    if (tid == 0) {
        for (uint32_t s = 0; s < stages; ++s) {
            mbar_init(smem_u32(full + s), 1);
            mbar_init(smem_u32(empty + s), kConsumerWarps);
        }
        *abort_word = 0u;
        *issued_word = 0u;
        mbar_fence_init();
    }
    __syncthreads();

    const uint32_t G = gridDim.x;
    const uint32_t count = staged_total > blockIdx.x ? (staged_total - blockIdx.x + G - 1) / G : 0u;

    if (warp == kConsumerWarps) {
        // ---- producer warp
        // A stall request naming this CTA is claimed by one launch only.
        uint32_t claim = 0u;
        if (status != nullptr && lane == 0 && count > 0u &&
            *reinterpret_cast<volatile uint32_t*>(status + 1) == blockIdx.x + 1u) {
            claim = atomicCAS(status + 1, blockIdx.x + 1u, 0u) == blockIdx.x + 1u ? 1u : 0u;
        }
        const bool withhold = __shfl_sync(0xffffffffu, claim, 0) != 0u;
        uint32_t s = 0, phase = 0;
        for (uint32_t j = 0; j < count; ++j) {
            if (j >= stages) {
                // Stage s last held span j - stages (phase ^ 1 of the ring).
                if (!mbar_wait_bounded(smem_u32(empty + s), phase ^ 1u, abort_word)) {
                    if (lane == 0) {
                        *abort_word = 1u;
                        if (status != nullptr) atomicOr(status, kStatusWaitTimeout);
                    }
                    break;
                }
            }
            const uint32_t k = blockIdx.x + j * G;
            const uint32_t l = kSingle ? 0u : find_lattice<A, true>(lats, n, k);
            const Lattice3D<A>& L = table[kSingle ? 0u : l];
            const uint32_t local = k - static_cast<uint32_t>(L.staged_begin);
            const uint32_t zi = local / L.spans;
            const uint32_t off = (local - zi * L.spans) * N;   // node offset in the plane's interior rows
            const uint32_t nx = L.g.nx;
            const uint32_t dy = off / nx;
            const uint32_t x0 = off - dy * nx, y0 = 1u + dy, z = 1u + zi;
            const uint64_t c0 = static_cast<uint64_t>(z) * L.g.plane + static_cast<uint64_t>(nx) * y0 + x0;
            const uint32_t bar = smem_u32(full + s);
            unsigned char* stage = ring + s * STAGE;
            if (withhold && j == 0u) {
                // The stall request: this stage is never armed or filled.
            } else if (lane == 0) {
                info[s] = make_uint4(l, x0, y0, z);
                mbar_expect_tx(bar, STAGE);
            }
            __syncwarp();
            if (withhold && j == 0u) {
                // no copies
            } else if (lane < static_cast<uint32_t>(d3::Q)) {
                int cx, cy, cz;
                c_rt(static_cast<int>(lane), cx, cy, cz);
                const S* src = static_cast<const S*>(L.f[L.parity ^ flip]);
                const int64_t shift = static_cast<int64_t>(nx) * cy + static_cast<int64_t>(L.g.plane) * cz + H;
                const S* from = src + static_cast<uint64_t>(lane) * L.g.cells +
                                static_cast<uint64_t>(static_cast<int64_t>(c0) - shift);
                bulk_load(smem_u32(stage + lane * SEG * sizeof(S)), from, SEG * sizeof(S), bar);
            } else if (lane == static_cast<uint32_t>(d3::Q)) {
                bulk_load(smem_u32(stage + POP), L.b.cls + c0, N, bar);
            }
            if (lane == 0) {
                *issued_word = j + 1u;
            }
            if (++s == stages) {
                s = 0;
                phase ^= 1u;
            }
        }
    } else {
        // ---- consumer warps: the direct items (face rows, unstaged
        // lattices) first, while the first stages load.
        const auto run_direct = [&]() {
            for (uint32_t d = blockIdx.x; d < direct_total; d += G) {
                const uint32_t l = kSingle ? 0u : find_lattice<A, false>(lats, n, d);
                const Lattice3D<A>& L = table[kSingle ? 0u : l];
                const uint32_t tiles = L.g.tiles_x;
                const uint32_t local = d - static_cast<uint32_t>(L.direct_begin);
                const uint32_t x = (local % tiles) * B + tid;
                uint32_t y, z;
                direct_row(L.g, L.staged != 0, local / tiles, y, z);
                if (x < L.g.nx) {
                    const uint32_t from = L.parity ^ flip;
                    step_node3<S, kSmag, true>(L.g, L.p, static_cast<const S*>(L.f[from]),
                                               static_cast<S*>(L.f[from ^ 1u]), L.b, x, y, z);
                }
            }
        };
        run_direct();
        uint32_t s = 0, phase = 0;
        for (uint32_t j = 0; j < count; ++j) {
            if (!mbar_wait_bounded(smem_u32(full + s), phase, abort_word)) {
                if (lane == 0) {
                    *abort_word = 1u;
                    if (status != nullptr) atomicOr(status, kStatusWaitTimeout);
                }
                break;
            }
            const unsigned char* stage = ring + s * STAGE;
            const uint4 it = info[s];
            const S* seg = reinterpret_cast<const S*>(stage);
            const Lattice3D<A>& L = table[kSingle ? 0u : it.x];
            const uint32_t from = L.parity ^ flip;
#pragma unroll
            for (int p = 0; p < NPT; ++p) {
                const uint32_t k = tid + static_cast<uint32_t>(p) * B;
                A f[d3::Q];
#pragma unroll
                for (int i = 0; i < d3::Q; ++i) {
                    f[i] = T::value(seg[i * SEG + (H - d3::cx(i)) + k]);
                }
                const uint8_t cls = stage[POP + k];
                // Node coordinates: x0 + k = dy nx + x, in row y0 + dy.
                const uint32_t m = it.y + k;
                const uint32_t dy = L.magic != 0u ? __umulhi(m, L.magic) : m / L.g.nx;
                const uint32_t x = m - dy * L.g.nx, y = it.z + dy;
                if (cls == kBulk && x + 1u == L.g.nx && L.g.x_mode == ORR_X_INFLOW_OUTFLOW) {
                    // Outlet: the zero-gradient copy f*_i(nx - 1) of the
                    // c_x < 0 directions is the node's own staged value.
#pragma unroll
                    for (int i = 0; i < d3::Q; ++i) {
                        if (d3::cx(i) < 0) {
                            f[i] = T::value(seg[i * SEG + H + k]);
                        }
                    }
                }
                if (p == NPT - 1) {
                    __syncwarp();
                    if (lane == 0) {
                        mbar_arrive(smem_u32(empty + s));
                    }
                }
                if (y + 1u < L.g.ny) {
                    staged_node3<S, kSmag>(L.g, L.p, L.b, static_cast<const S*>(L.f[from]),
                                           static_cast<S*>(L.f[from ^ 1u]), f, cls, x, y, it.w);
                }
            }
            if (++s == stages) {
                s = 0;
                phase ^= 1u;
            }
        }
    }
    __syncthreads();
    if (*abort_word != 0u && tid == 0) {
        // Let the copies still in flight land before the CTA's shared memory
        // goes away: the last `stages` issued spans (bounded waits).
        const uint32_t issued = *issued_word;
        const uint32_t first = issued > stages ? issued - stages : 0u;
        for (uint32_t j = first; j < issued; ++j) {
            const uint32_t bar = smem_u32(full + j % stages);
            const uint32_t parity = (j / stages) & 1u;
            for (uint32_t k = 0; k < kWaitPolls && !mbar_try_wait(bar, parity); ++k) {
            }
        }
    }
}

} // namespace orr
