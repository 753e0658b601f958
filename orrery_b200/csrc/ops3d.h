// Per-storage launch table of the D3Q19 kernels.  The kernels are
// instantiated in kernels_f32.cu, kernels_f16.cu, kernels_bf16.cu and
// kernels_f64.cu (double, built without FMA contraction); the solver
// reaches them only through this table.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tiles.h"

namespace orr {

struct Geom3D;
struct StepBuffers3D;

struct Ops3D {
    // One fused step src -> dst (one launch).  `phys` points at a Phys3D of
    // the storage's arithmetic type; `block` is the block width (threads
    // along x of a row); npt 2 takes the pair step (two neighbouring nodes
    // per thread) where pairs_ok allows it, the one-node step otherwise.
    cudaError_t (*step)(const Geom3D& g, const void* phys, const void* src, void* dst,
                        const StepBuffers3D& b, bool smag, uint32_t block, uint32_t npt, cudaStream_t s);
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
    int (*step_registers)(bool smag, uint32_t npt);
    // Whether the pair step serves lattice g with blocks of `block` threads
    // (2-byte storage, periodic or free-slip sides and halfway walls, even nx,
    // whole warps up to 128 threads).
    bool (*pairs_ok)(const Geom3D& g, uint32_t block);
    // Persistent step over a device table of n Lattice3D entries of the
    // storage's arithmetic type (staged3d.cuh): `grid` CTAs of `block`
    // consumer threads (128 or 256) plus a producer warp, spans of
    // block * npt nodes (npt 1 or 2), `stages` pipeline stages, source buffer
    // f[parity ^ flip] of every lattice.  With n == 1 and `host_one` (a host
    // copy of the entry) the entry is passed by value.
    cudaError_t (*staged)(const void* host_one, const void* table, uint32_t n, uint64_t staged_items,
                          uint64_t direct_items, uint32_t flip, uint32_t stages, bool smag,
                          uint32_t block, uint32_t npt, uint32_t grid, uint32_t* status, cudaStream_t s);
    // Resident CTAs per SM of the persistent step for (smag, block, npt,
    // stages), after raising the kernel's dynamic shared-memory limit; 0 if
    // it cannot launch.
    int (*staged_occupancy)(bool smag, uint32_t block, uint32_t npt, uint32_t stages);
    // Dynamic shared memory of the persistent step, bytes.
    uint32_t (*staged_smem)(uint32_t block, uint32_t npt, uint32_t stages);
    // Registers per thread of the persistent step.
    int (*staged_registers)(bool smag, uint32_t block, uint32_t npt);
    // Persistent tiled step of one flat lattice (tiled3d.cuh): `host_one` a
    // host copy of its Lattice3D entry (passed by value), `maps` its tensor
    // maps, `tg` its tile numbering for tiles of `rows` rows and `block`
    // consumer threads (rows 8 with 512 threads, or rows 4 with 256), `grid`
    // CTAs, `stages` pipeline stages, source buffer f[parity ^ flip].
    cudaError_t (*tiled)(const void* host_one, const TileMaps& maps, const TileGrid& tg, uint32_t flip,
                         uint32_t stages, bool smag, uint32_t rows, uint32_t block, uint32_t grid, uint32_t* status,
                         cudaStream_t s);
    // Resident CTAs per SM of the tiled step (0: cannot launch) and its
    // registers per thread.
    int (*tiled_occupancy)(bool smag, uint32_t rows, uint32_t block, uint32_t stages);
    int (*tiled_registers)(bool smag, uint32_t rows, uint32_t block);
    // Momentum exchange of n lattices (device table of ForceJob, kernels3d.cuh)
    // summed in a fixed order: pass 1 over `chunks` link chunks into
    // `partial` (6 doubles per chunk), pass 2 into out[6 l ..] (added to it
    // when `accumulate`).
    cudaError_t (*force_batch)(const void* jobs, uint32_t n, uint64_t chunks, double* partial,
                               double* out, bool accumulate, cudaStream_t s);
};

const Ops3D& ops3d_f32();
const Ops3D& ops3d_f16();
const Ops3D& ops3d_bf16();
const Ops3D& ops3d_f64();

} // namespace orr
