// Launchers of the D3Q19 kernels for one storage type (included by the
// instantiation units).
#pragma once

#include <algorithm>

#include "kernels3d.cuh"
#include "ops3d.h"
#include "staged3d.cuh"
#include "tiled3d.cuh"

namespace orr {

template <class S> struct Launch3D {
    using A = typename Storage<S>::A;

    static cudaError_t step(const Geom3D& g, const void* phys, const void* src, void* dst,
                            const StepBuffers3D& b, bool smag, uint32_t block, uint32_t npt, cudaStream_t s) {
        Geom3D gg = g;
        gg.tiles_x = (g.nx + block - 1) / block;
        const auto& p = *static_cast<const Phys3D<A>*>(phys);
        const auto* in = static_cast<const S*>(src);
        auto* out = static_cast<S*>(dst);
        if constexpr (sizeof(S) == 2) {
            if (npt == 2 && pairs_ok(g, block)) {
                gg.tiles_x = (g.nx + 2 * block - 1) / (2 * block);
                const dim3 grid2(gg.tiles_x, g.ny, g.nz);
                if (smag) {
                    step3d_pair_kernel<S, true><<<grid2, block, 0, s>>>(gg, p, in, out, b);
                } else {
                    step3d_pair_kernel<S, false><<<grid2, block, 0, s>>>(gg, p, in, out, b);
                }
                return cudaGetLastError();
            }
        }
        const dim3 grid(gg.tiles_x, g.ny, g.nz);
        if (smag) {
            if (g.flat) {
                step3d_kernel<S, true, true><<<grid, block, 0, s>>>(gg, p, in, out, b);
            } else {
                step3d_kernel<S, true, false><<<grid, block, 0, s>>>(gg, p, in, out, b);
            }
        } else {
            if (g.flat) {
                step3d_kernel<S, false, true><<<grid, block, 0, s>>>(gg, p, in, out, b);
            } else {
                step3d_kernel<S, false, false><<<grid, block, 0, s>>>(gg, p, in, out, b);
            }
        }
        return cudaGetLastError();
    }

    static cudaError_t init(const Geom3D& g, const uint8_t* cls, const double* rho,
                            const double* ux, const double* uy, const double* uz, double r0,
                            double u0x, double u0y, double u0z, void* f0, cudaStream_t s) {
        const unsigned blocks = static_cast<unsigned>((g.cells + 255) / 256);
        init3d_kernel<S><<<blocks, 256, 0, s>>>(g, cls, rho, ux, uy, uz, r0, u0x, u0y, u0z,
                                                static_cast<S*>(f0));
        return cudaGetLastError();
    }

    static cudaError_t history(const Geom3D& g, const void* f, void* hist, cudaStream_t s) {
        const unsigned face = g.ny * g.nz;
        history3d_kernel<S><<<(face + 255) / 256, 256, 0, s>>>(g, static_cast<const S*>(f),
                                                               static_cast<A*>(hist));
        return cudaGetLastError();
    }

    static cudaError_t moments(const Geom3D& g, const void* phys, const uint8_t* cls,
                               const void* f, void* m, cudaStream_t s) {
        const unsigned blocks = static_cast<unsigned>((g.cells + 255) / 256);
        moments3d_kernel<S><<<blocks, 256, 0, s>>>(g, *static_cast<const Phys3D<A>*>(phys), cls,
                                                   static_cast<const S*>(f), static_cast<A*>(m));
        return cudaGetLastError();
    }

    static cudaError_t force(const Geom3D& g, const void* f, const uint32_t* lcell,
                             const uint32_t* ldir, const double* lq, uint64_t links, double* out,
                             cudaStream_t s) {
        cudaError_t e = cudaMemsetAsync(out, 0, 6 * sizeof(double), s);
        if (e != cudaSuccess || links == 0) {
            return e;
        }
        const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((links + 255) / 256, 1184));
        force3d_kernel<S><<<blocks, 256, 0, s>>>(g, static_cast<const S*>(f), lcell, ldir, lq,
                                                 links, out);
        return cudaGetLastError();
    }

    static cudaError_t mass(const Geom3D& g, const uint8_t* cls, const void* f, double* out,
                            cudaStream_t s) {
        cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), s);
        if (e != cudaSuccess) {
            return e;
        }
        const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((g.cells + 255) / 256, 1184));
        mass3d_kernel<S><<<blocks, 256, 0, s>>>(g, cls, static_cast<const S*>(f), out);
        return cudaGetLastError();
    }

    // The pair step serves 2-byte storage on flat lattices with even nx, in
    // blocks of whole warps up to 128 threads.
    static bool pairs_ok(const Geom3D& g, uint32_t block) {
        return sizeof(S) == 2 && g.flat && g.nx % 2 == 0 && block % 32 == 0 && block <= 128;
    }

    static int step_registers(bool smag, uint32_t npt) {
        cudaFuncAttributes a{};
        cudaError_t e = cudaErrorInvalidValue;
        if constexpr (sizeof(S) == 2) {
            if (npt == 2) {
                e = smag ? cudaFuncGetAttributes(&a, step3d_pair_kernel<S, true>)
                         : cudaFuncGetAttributes(&a, step3d_pair_kernel<S, false>);
                return e == cudaSuccess ? a.numRegs : -1;
            }
        }
        e = smag ? cudaFuncGetAttributes(&a, step3d_kernel<S, true, true>)
                 : cudaFuncGetAttributes(&a, step3d_kernel<S, false, true>);
        return e == cudaSuccess ? a.numRegs : -1;
    }

    template <bool kSmag, int B, int NPT, bool kSingle> static constexpr auto staged_kernel() {
        return &step3d_staged_kernel<S, kSmag, B, NPT, kSingle>;
    }

    // Calls f.template operator()<kSmag, B, NPT>() for a supported runtime
    // shape (B 128 or 256, NPT 1 or 2); false otherwise.
    template <class F> static bool with_shape(bool smag, uint32_t block, uint32_t npt, F&& f) {
        const auto go = [&]<bool K>() {
            if (block == 256 && npt == 1) { f.template operator()<K, 256, 1>(); return true; }
            if (block == 256 && npt == 2) { f.template operator()<K, 256, 2>(); return true; }
            if (block == 128 && npt == 1) { f.template operator()<K, 128, 1>(); return true; }
            if (block == 128 && npt == 2) { f.template operator()<K, 128, 2>(); return true; }
            return false;
        };
        return smag ? go.template operator()<true>() : go.template operator()<false>();
    }

    // One lattice (host_one non-null, n == 1) travels by value, so its fields
    // are constant-bank operands; otherwise the kernel reads the device table.
    static cudaError_t staged(const void* host_one, const void* table, uint32_t n, uint64_t staged_items,
                              uint64_t direct_items, uint32_t flip, uint32_t stages, bool smag,
                              uint32_t block, uint32_t npt, uint32_t grid, uint32_t* status, cudaStream_t s) {
        if (stages == 0 || stages > kMaxStages || grid == 0 || staged_items >= (1ull << 31) ||
            direct_items >= (1ull << 31)) {
            return cudaErrorInvalidValue;
        }
        const auto* one = static_cast<const Lattice3D<A>*>(host_one);
        const auto* lats = static_cast<const Lattice3D<A>*>(table);
        const auto si = static_cast<uint32_t>(staged_items), di = static_cast<uint32_t>(direct_items);
        const bool ok = with_shape(smag, block, npt, [&]<bool K, int B, int NPT>() {
            const uint32_t smem = staged_smem_bytes<S, B * NPT>(stages);
            if (one != nullptr && n == 1) {
                staged_kernel<K, B, NPT, true>()<<<grid, kStagedThreads<B>, smem, s>>>(
                    *one, lats, n, si, di, flip, stages, status);
            } else {
                staged_kernel<K, B, NPT, false>()<<<grid, kStagedThreads<B>, smem, s>>>(
                    Lattice3D<A>{}, lats, n, si, di, flip, stages, status);
            }
        });
        return ok ? cudaGetLastError() : cudaErrorInvalidValue;
    }

    static uint32_t staged_smem(uint32_t block, uint32_t npt, uint32_t stages) {
        uint32_t bytes = 0;
        with_shape(false, block, npt, [&]<bool K, int B, int NPT>() { bytes = staged_smem_bytes<S, B * NPT>(stages); });
        return bytes;
    }

    // The kernel's dynamic shared-memory limit is raised to the device's
    // opt-in maximum (not to `smem`: solvers with different stage counts
    // share the kernel).
    template <class K> static int occupancy_of(K kernel, uint32_t threads, uint32_t smem) {
        int device = 0, optin = 0;
        if (cudaGetDevice(&device) != cudaSuccess ||
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        if (static_cast<int>(smem) > optin) {
            return 0;
        }
        if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        int blocks = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, static_cast<int>(threads), smem) !=
            cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        return blocks;
    }

    // Both variants (single and table) get the attribute; the occupancy is
    // the smaller of the two.
    static int staged_occupancy(bool smag, uint32_t block, uint32_t npt, uint32_t stages) {
        if (stages == 0 || stages > kMaxStages) {
            return 0;
        }
        int result = 0;
        with_shape(smag, block, npt, [&]<bool K, int B, int NPT>() {
            const uint32_t smem = staged_smem_bytes<S, B * NPT>(stages);
            const int a = occupancy_of(staged_kernel<K, B, NPT, true>(), kStagedThreads<B>, smem);
            const int b = occupancy_of(staged_kernel<K, B, NPT, false>(), kStagedThreads<B>, smem);
            result = a < b ? a : b;
        });
        return result;
    }

    static int staged_registers(bool smag, uint32_t block, uint32_t npt) {
        int regs = -1;
        with_shape(smag, block, npt, [&]<bool K, int B, int NPT>() {
            cudaFuncAttributes a{};
            if (cudaFuncGetAttributes(&a, staged_kernel<K, B, NPT, true>()) == cudaSuccess) {
                regs = a.numRegs;
            }
        });
        return regs;
    }

    // Calls f.template operator()<kSmag, R, B>() for a supported tile shape
    // (rows 8 with 512 consumers, rows 4 with 256); false otherwise.
    template <class F> static bool with_tile(bool smag, uint32_t rows, uint32_t block, F&& f) {
        const auto go = [&]<bool K>() {
            if (rows == 8 && block == 512) { f.template operator()<K, 8, 512>(); return true; }
            if (rows == 4 && block == 256) { f.template operator()<K, 4, 256>(); return true; }
            if (rows == 2 && block == 256) { f.template operator()<K, 2, 256>(); return true; }
            return false;
        };
        return smag ? go.template operator()<true>() : go.template operator()<false>();
    }

    static cudaError_t tiled(const void* host_one, const TileMaps& maps, const TileGrid& tg, uint32_t flip,
                             uint32_t stages, bool smag, uint32_t rows, uint32_t block, uint32_t grid,
                             uint32_t* status, cudaStream_t s) {
        if (stages == 0 || stages > kMaxStages || grid == 0 || host_one == nullptr) {
            return cudaErrorInvalidValue;
        }
        const auto& one = *static_cast<const Lattice3D<A>*>(host_one);
        const bool ok = with_tile(smag, rows, block, [&]<bool K, int R, int B>() {
            step3d_tiled_kernel<S, K, R, B><<<grid, kTiledThreads<B>, tiled_smem_bytes<S, R>(stages), s>>>(
                one, maps, tg, flip, stages, status);
        });
        return ok ? cudaGetLastError() : cudaErrorInvalidValue;
    }

    static int tiled_occupancy(bool smag, uint32_t rows, uint32_t block, uint32_t stages) {
        if (stages == 0 || stages > kMaxStages) {
            return 0;
        }
        int result = 0;
        with_tile(smag, rows, block, [&]<bool K, int R, int B>() {
            result = occupancy_of(&step3d_tiled_kernel<S, K, R, B>, kTiledThreads<B>,
                                  tiled_smem_bytes<S, R>(stages));
        });
        return result;
    }

    static int tiled_registers(bool smag, uint32_t rows, uint32_t block) {
        int regs = -1;
        with_tile(smag, rows, block, [&]<bool K, int R, int B>() {
            cudaFuncAttributes a{};
            if (cudaFuncGetAttributes(&a, &step3d_tiled_kernel<S, K, R, B>) == cudaSuccess) {
                regs = a.numRegs;
            }
        });
        return regs;
    }

    static cudaError_t force_batch(const void* jobs, uint32_t n, uint64_t chunks, double* partial,
                                   double* out, bool accumulate, cudaStream_t s) {
        if (n == 0) {
            return cudaSuccess;
        }
        const auto* j = static_cast<const ForceJob*>(jobs);
        if (chunks > 0) {
            force_batch_partials<S><<<static_cast<unsigned>(chunks), kForceThreads, 0, s>>>(j, n, partial);
        }
        force_batch_totals<S><<<n, kForceThreads, 0, s>>>(j, partial, out, accumulate ? 1 : 0);
        return cudaGetLastError();
    }

    static const Ops3D& table() {
        static const Ops3D ops{&step,   &init,   &history,        &moments,          &force,
                               &mass,   &step_registers, &pairs_ok, &staged, &staged_occupancy,
                               &staged_smem, &staged_registers, &tiled, &tiled_occupancy,
                               &tiled_registers, &force_batch};
        return ops;
    }
};

} // namespace orr
