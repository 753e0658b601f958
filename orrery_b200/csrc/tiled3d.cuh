// Persistent D3Q19 step of one flat lattice whose interior rows are moved
// into shared memory as two-dimensional tiles by tensor copies
// (cp.async.bulk.tensor, completion on an mbarrier).
//
// Tiles.  The interior of the lattice (1 <= y <= ny-2, 1 <= z <= nz-2, every
// x) is cut into tiles of kTileW nodes along x by R rows along y in one
// z-plane.  The population buffer is seen as the three-dimensional tensor
// (x: nx, y: ny, d: 19 nz) with d = i nz + z, so the pull sources of
// direction i for a whole tile are one box of (kTileW + 2H) x R x 1 at
// (x0 - H, y0 - cy_i, i nz + z - cz_i): rows y0 - cy_i ... of plane z - cz_i,
// with a halo of H values (16 bytes) on both sides for c_x = +-1.  The class
// bytes are the box kTileW x R of the tensor (x: nx, row: ny nz).  One stage
// thus takes 20 tensor copies for kTileW R nodes (the span kernel of
// staged3d.cuh takes 20 per B nodes), and boxes outside the lattice are
// filled with zeros by the copy engine (x < 0, x >= nx, y >= ny: values no
// node of the tile uses).
//
// Work.  Tiles are numbered x fastest, then y, then z; CTA b takes tiles
// b, b + G, ... so the CTAs in flight work on neighbouring tiles and the
// shifted rows they share stay in L2.  The face rows (y = 0, y = ny - 1,
// z = 0, z = nz - 1) are direct items, as in the span kernel: the per-node
// gather of step_node3 from global memory.
//
// Pipeline.  A CTA has B consumer threads and one producer warp.  The
// producer keeps up to `stages` tiles in flight (full / empty mbarriers per
// stage); consumer thread t owns the nodes (x0 + t % kTileW, y0 + t / kTileW
// + p B / kTileW) of a tile, reads their 19 values and class from the stage
// (a warp reads 32 consecutive x of one row: no bank conflicts), releases
// the stage after its last node's reads and finishes each node exactly as
// the span kernel does (staged_node3: x-edge fix-ups, bounce-back overrides
// from global memory for the rare boundary nodes, inlet, collision and the
// 19 stores), so a node's bits do not depend on the kernel that carried it.
//
// Every wait is bounded as in staged3d.cuh, and the stall request of a test
// (the word after the status word) withholds the first tile of the CTA it
// names.  Tensor maps cover this GPU's own buffers only; no copy uses
// cluster multicast.
#pragma once

#include <cstdint>

#include "staged3d.cuh"
#include "tiles.h"

namespace orr {

template <class S> constexpr int kTileHalo = 16 / static_cast<int>(sizeof(S));
// Values per staged row, bytes of one direction's box, of a stage.
template <class S> constexpr uint32_t kTileRow = kTileW + 2 * kTileHalo<S>;
template <class S, int R> constexpr uint32_t kTileBox = R * kTileRow<S> * sizeof(S);
// Shared bytes between the boxes of consecutive directions: the box rounded
// up to 128 bytes (every tensor copy lands on a 128-byte boundary).
template <class S, int R> constexpr uint32_t kTileBoxStride = (kTileBox<S, R> + 127u) & ~127u;
template <class S, int R> constexpr uint32_t kTilePop = d3::Q * kTileBoxStride<S, R>;
template <class S, int R> constexpr uint32_t kTileStage = kTilePop<S, R> + R * kTileW;
// Shared header: full barriers (64 B), empty barriers (64 B), tile records
// (128 B), the abort word and the issued-tile count; the stages start on the
// next 128-byte boundary of the dynamic window (128 bytes of slack).
constexpr uint32_t kTileHeader = 384;

template <class S, int R> constexpr uint32_t tiled_smem_bytes(uint32_t stages) {
    return kTileHeader + 128 + stages * kTileStage<S, R>;
}

// Threads of a tiled CTA: B consumers and one producer warp.
template <int B> constexpr int kTiledThreads = B + 32;
// Resident CTAs per SM the kernel is compiled for (registers): one CTA of
// 512 consumers, or three of 256.
template <int B> constexpr int kTiledMinBlocks = B >= 512 ? 1 : 3;

// Tensor copy of a three-dimensional box into shared memory completing on
// `bar` (the box's x coordinate times the value size is a multiple of 16).
__device__ __forceinline__ void tensor_load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                                               uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
        "%4}], [%5];" ::"r"(dst),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tensor_load_2d(uint32_t dst, const CUtensorMap* map, int c0, int c1,
                                               uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(dst),
        "l"(map), "r"(c0), "r"(c1), "r"(bar)
        : "memory");
}

// The tiled step of lattice L (by value: its fields are constant-bank
// operands), source buffer f[L.parity ^ flip].  R rows per tile, B consumer
// threads, NPT = kTileW R / B nodes per consumer thread and tile.
template <class S, bool kSmag, int R, int B>
__global__ void __launch_bounds__(kTiledThreads<B>, kTiledMinBlocks<B>)
    step3d_tiled_kernel(const __grid_constant__ Lattice3D<typename Storage<S>::A> L,
                        const __grid_constant__ TileMaps maps, TileGrid tg, uint32_t flip, uint32_t stages,
                        uint32_t* __restrict__ status) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    constexpr int H = kTileHalo<S>;
    constexpr uint32_t ROW = kTileRow<S>;
    constexpr uint32_t BOX = kTileBoxStride<S, R>;
    constexpr uint32_t DIR = BOX / sizeof(S);   // values between consecutive directions' boxes
    constexpr uint32_t POP = kTilePop<S, R>;
    constexpr uint32_t STAGE = kTileStage<S, R>;
    // Bytes the copies of a stage bring (the boxes without their padding).
    constexpr uint32_t TX = d3::Q * kTileBox<S, R> + R * kTileW;
    constexpr uint32_t kConsumerWarps = B / 32;
    constexpr uint32_t kRowsPerPass = B / kTileW;
    constexpr int NPT = static_cast<int>(kTileW) * R / B;
    static_assert(B % kTileW == 0 && (kTileW * R) % B == 0, "tile shape");
    static_assert(BOX % 128 == 0 && POP % 128 == 0 && STAGE % 128 == 0, "tensor boxes start on 128-byte boundaries");
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = reinterpret_cast<uint64_t*>(smem + 64);
    uint4* info = reinterpret_cast<uint4*>(smem + 128);
    volatile uint32_t* abort_word = reinterpret_cast<volatile uint32_t*>(smem + 256);
    volatile uint32_t* issued_word = reinterpret_cast<volatile uint32_t*>(smem + 260);
    // Stages on a 128-byte boundary of the shared window.
    const uint32_t ring_addr = (smem_u32(smem + kTileHeader) + 127u) & ~127u;
    unsigned char* ring = smem + (ring_addr - smem_u32(smem));
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    const uint32_t warp = tid >> 5;
    const uint32_t nx = L.g.nx, ny = L.g.ny, nz = L.g.nz;
    const uint32_t from = L.parity ^ flip;
    const S* src = static_cast<const S*>(L.f[from]);
    S* dst = static_cast<S*>(L.f[from ^ 1u]);

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
    const uint32_t count = tg.tiles > blockIdx.x ? (tg.tiles - blockIdx.x + G - 1) / G : 0u;

    if (warp == kConsumerWarps) {
        // ---- producer warp
        uint32_t claim = 0u;
        if (status != nullptr && lane == 0 && count > 0u &&
            *reinterpret_cast<volatile uint32_t*>(status + 1) == blockIdx.x + 1u) {
            claim = atomicCAS(status + 1, blockIdx.x + 1u, 0u) == blockIdx.x + 1u ? 1u : 0u;
        }
        const bool withhold = __shfl_sync(0xffffffffu, claim, 0) != 0u;
        const CUtensorMap* pop = &maps.pop[from];
        uint32_t s = 0, phase = 0;
        for (uint32_t j = 0; j < count; ++j) {
            if (j >= stages) {
                // Stage s last held tile j - stages (phase ^ 1 of the ring).
                if (!mbar_wait_bounded(smem_u32(empty + s), phase ^ 1u, abort_word)) {
                    if (lane == 0) {
                        *abort_word = 1u;
                        if (status != nullptr) atomicOr(status, kStatusWaitTimeout);
                    }
                    break;
                }
            }
            const uint32_t k = blockIdx.x + j * G;
            const uint32_t zi = k / tg.tiles_plane;
            const uint32_t rest = k - zi * tg.tiles_plane;
            const uint32_t ty = rest / tg.tiles_x;
            const uint32_t x0 = (rest - ty * tg.tiles_x) * kTileW, y0 = 1u + ty * R, z = 1u + zi;
            const uint32_t bar = smem_u32(full + s);
            const uint32_t stage = ring_addr + s * STAGE;
            const bool skip = withhold && j == 0u;   // the stall request: never armed or filled
            if (!skip && lane == 0) {
                info[s] = make_uint4(x0, y0, z, 0u);
                mbar_expect_tx(bar, TX);
            }
            __syncwarp();
            if (!skip && lane < static_cast<uint32_t>(d3::Q)) {
                int cx, cy, cz;
                c_rt(static_cast<int>(lane), cx, cy, cz);
                (void)cx;
                tensor_load_3d(stage + lane * BOX, pop, static_cast<int>(x0) - H, static_cast<int>(y0) - cy,
                               static_cast<int>(lane * nz + z) - cz, bar);
            } else if (!skip && lane == static_cast<uint32_t>(d3::Q)) {
                tensor_load_2d(stage + POP, &maps.cls, static_cast<int>(x0), static_cast<int>(z * ny + y0), bar);
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
        // ---- consumer warps: the face rows first, while the first stages load.
        for (uint32_t d = blockIdx.x; d < tg.direct; d += G) {
            const uint32_t per_row = (nx + B - 1) / B;
            const uint32_t x = (d % per_row) * B + tid;
            uint32_t y, z;
            direct_row(L.g, true, d / per_row, y, z);
            if (x < nx) {
                step_node3<S, kSmag, true>(L.g, L.p, src, dst, L.b, x, y, z);
            }
        }
        const uint32_t xx = tid % kTileW;
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
            const uint32_t x = it.x + xx;
            // Every node's stored values first (kept in the storage type),
            // then the stage is released, then the nodes are finished: the
            // producer refills the stage while the collisions run.
            S raw[NPT][d3::Q];
            uint8_t cls[NPT];
#pragma unroll
            for (int p = 0; p < NPT; ++p) {
                const uint32_t r = tid / kTileW + static_cast<uint32_t>(p) * kRowsPerPass;
                const S* row = seg + r * ROW + xx;
                cls[p] = stage[POP + r * kTileW + xx];
                const bool outlet = cls[p] == kBulk && x + 1u == nx && L.g.x_mode == ORR_X_INFLOW_OUTFLOW;
#pragma unroll
                for (int i = 0; i < d3::Q; ++i) {
                    // Outlet: the zero-gradient copy f*_i(nx - 1) of the
                    // c_x < 0 directions is the node's own staged value.
                    const int at = outlet && d3::cx(i) < 0 ? H : H - d3::cx(i);
                    raw[p][i] = row[i * DIR + at];
                }
            }
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(smem_u32(empty + s));
            }
#pragma unroll
            for (int p = 0; p < NPT; ++p) {
                const uint32_t r = tid / kTileW + static_cast<uint32_t>(p) * kRowsPerPass;
                const uint32_t y = it.y + r;
                if (x < nx && y + 1u < ny) {
                    A f[d3::Q];
#pragma unroll
                    for (int i = 0; i < d3::Q; ++i) {
                        f[i] = T::value(raw[p][i]);
                    }
                    staged_node3<S, kSmag>(L.g, L.p, L.b, src, dst, f, cls[p], x, y, it.z);
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
        // goes away: the last `stages` issued tiles (bounded waits).
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
