// Host side of the persistent step: lattice-table entries, item numbering
// and the launch shape.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "ops3d.h"
#include "staged3d.cuh"

namespace orr {

// A lattice's interior rows can be staged: rows of a multiple of 16 nodes
// (every row segment and class row starts on a 16-byte boundary for all
// storage forms) and at least one interior row.
inline bool stageable(const Geom3D& g) {
    return g.nx % 16 == 0 && g.ny >= 3 && g.nz >= 3;
}

struct ItemCounts {
    uint64_t staged = 0;
    uint64_t direct = 0;
};

// Numbers the items of lattices[0, n) for direct tiles of `block` nodes and
// staged spans of block * npt nodes: sets each tiles_x, spans, magic and the
// prefix offsets, returns the totals.
template <class A>
ItemCounts number_items(Lattice3D<A>* lats, std::size_t n, uint32_t block, uint32_t npt) {
    ItemCounts c;
    const uint64_t span = static_cast<uint64_t>(block) * npt;
    for (std::size_t k = 0; k < n; ++k) {
        Lattice3D<A>& L = lats[k];
        L.g.tiles_x = (L.g.nx + block - 1) / block;
        const uint64_t tiles = L.g.tiles_x;
        L.staged_begin = c.staged;
        L.direct_begin = c.direct;
        L.spans = 0;
        L.magic = L.g.nx <= kMagicMaxNx ? static_cast<uint32_t>(((uint64_t{1} << 32) + L.g.nx - 1) / L.g.nx) : 0u;
        if (L.staged) {
            const uint64_t interior = static_cast<uint64_t>(L.g.nx) * (L.g.ny - 2ull);
            L.spans = static_cast<uint32_t>((interior + span - 1) / span);
            c.staged += static_cast<uint64_t>(L.spans) * (L.g.nz - 2ull);
            c.direct += tiles * (2ull * L.g.ny + 2ull * (L.g.nz - 2ull));
        } else {
            c.direct += tiles * L.g.ny * static_cast<uint64_t>(L.g.nz);
        }
    }
    return c;
}

// Launch shape of the persistent step.
struct StagedShape {
    uint32_t block = 256;
    uint32_t npt = 1;      // nodes per consumer thread of a span
    uint32_t stages = 0;
    uint32_t grid = 0;     // CTAs (resident CTAs per SM x SMs)
    int per_sm = 0;
};

// Picks the stages (the most, up to 4, that keep the register-limited
// residency, unless `stages` is given) and the grid for (block, npt).  A
// shape with per_sm == 0 cannot launch.
inline StagedShape staged_shape(const Ops3D& ops, bool smag, uint32_t block, uint32_t npt, uint32_t stages,
                                int device) {
    StagedShape s;
    s.block = block;
    s.npt = npt;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        return s;
    }
    if (stages != 0) {
        s.stages = stages;
        s.per_sm = ops.staged_occupancy(smag, block, npt, stages);
    } else {
        const int best = ops.staged_occupancy(smag, block, npt, 1);
        s.stages = 2;
        s.per_sm = ops.staged_occupancy(smag, block, npt, 2);
        for (uint32_t k = 4; k > 2; --k) {
            const int o = ops.staged_occupancy(smag, block, npt, k);
            if (o == best && o > 0) {
                s.stages = k;
                s.per_sm = o;
                break;
            }
        }
    }
    s.grid = static_cast<uint32_t>(std::max(s.per_sm, 0)) * static_cast<uint32_t>(sms);
    return s;
}

// Launch shape of the tiled step for tiles of `rows` rows and `block`
// consumer threads: the most stages (up to 4) that keep the residency of one
// stage, unless `stages` is given; npt holds the nodes per consumer thread
// and tile.
inline StagedShape tiled_shape(const Ops3D& ops, bool smag, uint32_t rows, uint32_t block, uint32_t stages,
                               int device) {
    StagedShape s;
    s.block = block;
    s.npt = kTileW * rows / block;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        return s;
    }
    if (stages != 0) {
        s.stages = stages;
        s.per_sm = ops.tiled_occupancy(smag, rows, block, stages);
    } else {
        const int best = ops.tiled_occupancy(smag, rows, block, 1);
        s.stages = 2;
        s.per_sm = ops.tiled_occupancy(smag, rows, block, 2);
        for (uint32_t k = 4; k > 2; --k) {
            const int o = ops.tiled_occupancy(smag, rows, block, k);
            if (o == best && o > 0) {
                s.stages = k;
                s.per_sm = o;
                break;
            }
        }
    }
    s.grid = static_cast<uint32_t>(std::max(s.per_sm, 0)) * static_cast<uint32_t>(sms);
    return s;
}

} // namespace orr
