// Per-storage launch table of the D3Q19 kernels.  The kernels are
// instantiated in kernels_binary32.cu (float, FP16S, bfloat16) and
// kernels_binary64.cu (double, built without FMA contraction); the solver
// reaches them only through this table.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace orr {

struct Geom3D;
struct StepBuffers3D;

struct Ops3D {
    // One fused step src -> dst (one launch).  `phys` points at a Phys3D of
    // the storage's arithmetic type; `block` is the block width (threads
    // along x of a row, and list entries per block).
    cudaError_t (*step)(const Geom3D& g, const void* phys, const void* src, void* dst,
                        const StepBuffers3D& b, bool smag, uint32_t block, cudaStream_t s);
    // Equilibrium initialisation of a population buffer; rho..uz may be
    // device arrays (all non-null) or null for the uniform state (r0, u0).
    cudaError_t (*init)(const Geom3D& g, const uint8_t* cls, const double* rho, const double* ux,
                        const double* uy, const double* uz, double r0, double u0x, double u0y,
                        double u0z, void* f0, cudaStream_t s);
    cudaError_t (*history)(const Geom3D& g, const void* f, void* hist, cudaStream_t s);
    cudaError_t (*moments)(const Geom3D& g, const void* phys, const uint8_t* cls, const void* f,
                           void* m, cudaStream_t s);
    cudaError_t (*force)(const Geom3D& g, const void* f, const uint32_t* lcell,
                         const uint32_t* ldir, const double* lq, uint64_t links, double* out,
                         cudaStream_t s);
    cudaError_t (*mass)(const Geom3D& g, const uint8_t* cls, const void* f, double* out,
                        cudaStream_t s);
    // Registers per thread of the step kernel (for the tuner and the docs).
    int (*step_registers)(bool smag);
};

const Ops3D& ops3d_f32();
const Ops3D& ops3d_f16();
const Ops3D& ops3d_bf16();
const Ops3D& ops3d_f64();

} // namespace orr
