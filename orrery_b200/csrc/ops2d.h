// Per-storage launch table of the D2Q9 kernels (instantiated next to the
// D3Q19 ones in kernels_f32/f16/bf16/f64.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace orr {

struct Geom2D;
struct StepBuffers2D;

struct Ops2D {
    // One fused step src -> dst (one launch over all rows).
    cudaError_t (*step)(const Geom2D& g, const void* phys, const void* src, void* dst,
                        const StepBuffers2D& b, bool smag, uint32_t block, cudaStream_t s);
    cudaError_t (*init)(const Geom2D& g, const uint8_t* cls, const double* rho, const double* ux,
                        const double* uy, double u0x, double u0y, void* f0, cudaStream_t s);
    cudaError_t (*history)(const Geom2D& g, const void* f, void* hist, cudaStream_t s);
    cudaError_t (*moments)(const Geom2D& g, const void* phys, const uint8_t* cls, const void* f,
                           void* m, cudaStream_t s);
    cudaError_t (*force)(const Geom2D& g, const void* f, const uint32_t* lcell,
                         const uint32_t* ldir, uint64_t links, double* out, cudaStream_t s);
    cudaError_t (*mass)(const Geom2D& g, const uint8_t* cls, const void* f, double* out,
                        cudaStream_t s);
};

const Ops2D& ops2d_f32();
const Ops2D& ops2d_f16();
const Ops2D& ops2d_bf16();
const Ops2D& ops2d_f64();

} // namespace orr
