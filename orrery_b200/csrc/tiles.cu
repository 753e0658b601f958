// Tensor maps and tile numbering of the tiled D3Q19 step (tiles.h).
//
// cuTensorMapEncodeTiled is a driver entry point; it is reached through the
// runtime's cudaGetDriverEntryPoint, so the library does not link the driver
// library itself.
#include "tiles.h"

#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "kernels3d.cuh"

namespace orr {

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encoder(std::string& why) {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::string failure;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || p == nullptr) {
            cudaGetLastError();
            failure = "the driver has no cuTensorMapEncodeTiled";
            return;
        }
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    why = failure;
    return fn;
}

CUtensorMapDataType value_type(std::size_t bytes) {
    switch (bytes) {
        case 1:
            return CU_TENSOR_MAP_DATA_TYPE_UINT8;
        case 2:
            return CU_TENSOR_MAP_DATA_TYPE_UINT16;
        case 4:
            return CU_TENSOR_MAP_DATA_TYPE_UINT32;
        default:
            return CU_TENSOR_MAP_DATA_TYPE_UINT64;
    }
}

} // namespace

bool tileable(const Geom3D& g) {
    return g.flat != 0 && g.nx % 16 == 0 && g.ny >= 3 && g.nz >= 3 &&
           static_cast<uint64_t>(d3::Q) * g.nz < (uint64_t{1} << 31) &&
           static_cast<uint64_t>(g.ny) * g.nz < (uint64_t{1} << 31);
}

TileGrid tile_grid(const Geom3D& g, uint32_t rows, uint32_t block) {
    TileGrid t{};
    t.tiles_x = (g.nx + kTileW - 1) / kTileW;
    t.tiles_plane = t.tiles_x * ((g.ny - 2 + rows - 1) / rows);
    t.tiles = t.tiles_plane * (g.nz - 2);
    t.direct = ((g.nx + block - 1) / block) * (2 * g.ny + 2 * (g.nz - 2));
    return t;
}

std::string encode_tile_maps(TileMaps& maps, const Geom3D& g, const void* f0, const void* f1, const uint8_t* cls,
                             std::size_t value_bytes, uint32_t rows) {
    std::string why;
    const auto encode = encoder(why);
    if (encode == nullptr) {
        return why;
    }
    const cuuint32_t halo = static_cast<cuuint32_t>(16 / value_bytes);
    const void* bufs[2] = {f0, f1};
    for (int k = 0; k < 2; ++k) {
        const cuuint64_t dims[3] = {g.nx, g.ny, static_cast<cuuint64_t>(d3::Q) * g.nz};
        const cuuint64_t strides[2] = {static_cast<cuuint64_t>(g.nx) * value_bytes,
                                       static_cast<cuuint64_t>(g.plane) * value_bytes};
        const cuuint32_t box[3] = {kTileW + 2 * halo, rows, 1};
        const cuuint32_t elem[3] = {1, 1, 1};
        const CUresult r = encode(&maps.pop[k], value_type(value_bytes), 3, const_cast<void*>(bufs[k]), dims,
                                  strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            return "cuTensorMapEncodeTiled refused the population map (" + std::to_string(static_cast<int>(r)) + ")";
        }
    }
    const cuuint64_t dims[2] = {g.nx, static_cast<cuuint64_t>(g.ny) * g.nz};
    const cuuint64_t strides[1] = {g.nx};
    const cuuint32_t box[2] = {kTileW, rows};
    const cuuint32_t elem[2] = {1, 1};
    const CUresult r = encode(&maps.cls, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(cls), dims, strides,
                              box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        return "cuTensorMapEncodeTiled refused the class map (" + std::to_string(static_cast<int>(r)) + ")";
    }
    return {};
}

} // namespace orr
