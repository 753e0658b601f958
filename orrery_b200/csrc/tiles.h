// Host and device types of the tiled D3Q19 step (tiled3d.cuh): the tensor
// maps of a lattice and its tile numbering, and the host routine that encodes
// the maps.
#pragma once

#include <cuda.h>

#include <cstddef>
#include <cstdint>
#include <string>

namespace orr {

struct Geom3D;

// Nodes along x of a tile.
constexpr uint32_t kTileW = 128;

// The tensor maps of one lattice: its two population buffers (load boxes of
// kTileW + 2H x R x 1 values of the tensor (x: nx, y: ny, d: 19 nz)) and its
// class bytes (boxes of kTileW x R of the tensor (x: nx, row: ny nz)).
struct TileMaps {
    CUtensorMap pop[2];
    CUtensorMap cls;
};

// Tile numbering of a lattice (host-computed, by value).
struct TileGrid {
    uint32_t tiles_x;      // tiles along x: ceil(nx / kTileW)
    uint32_t tiles_plane;  // tiles per z-plane: tiles_x ceil((ny - 2) / R)
    uint32_t tiles;        // tiles_plane (nz - 2)
    uint32_t direct;       // direct items: face rows x ceil(nx / B)
};

// The lattice's interior can be tiled: rows of a multiple of 16 nodes (every
// box row and class row starts on a 16-byte boundary), at least one
// interior row, and tensor dimensions within the copy engine's 2^32.
bool tileable(const Geom3D& g);

// Tile numbering for tiles of R rows and B consumer threads.
TileGrid tile_grid(const Geom3D& g, uint32_t rows, uint32_t block);

// Encodes the maps of a lattice whose population buffers f0, f1 hold values
// of `value_bytes` bytes (2, 4 or 8) and whose class bytes are at `cls`, for
// tiles of `rows` rows.  Returns an empty string, or why it failed.
std::string encode_tile_maps(TileMaps& maps, const Geom3D& g, const void* f0, const void* f1, const uint8_t* cls,
                             std::size_t value_bytes, uint32_t rows);

} // namespace orr
