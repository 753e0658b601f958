// Launchers of the D3Q19 kernels for one storage type (included by the
// instantiation units).
#pragma once

#include <algorithm>

#include "kernels3d.cuh"
#include "ops3d.h"

namespace orr {

template <class S> struct Launch3D {
    using A = typename Storage<S>::A;

    static cudaError_t step(const Geom3D& g, const void* phys, const void* src, void* dst,
                            const StepBuffers3D& b, bool smag, uint32_t block, cudaStream_t s) {
        Geom3D gg = g;
        gg.tiles_x = (g.nx + block - 1) / block;
        const dim3 grid(gg.tiles_x, g.ny, g.nz);
        const auto& p = *static_cast<const Phys3D<A>*>(phys);
        if (smag) {
            step3d_kernel<S, true><<<grid, block, 0, s>>>(gg, p, static_cast<const S*>(src),
                                                          static_cast<S*>(dst), b);
        } else {
            step3d_kernel<S, false><<<grid, block, 0, s>>>(gg, p, static_cast<const S*>(src),
                                                           static_cast<S*>(dst), b);
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

    static int step_registers(bool smag) {
        cudaFuncAttributes a{};
        const cudaError_t e = smag ? cudaFuncGetAttributes(&a, step3d_kernel<S, true>)
                                   : cudaFuncGetAttributes(&a, step3d_kernel<S, false>);
        return e == cudaSuccess ? a.numRegs : -1;
    }

    static const Ops3D& table() {
        static const Ops3D ops{&step, &init, &history, &moments, &force, &mass, &step_registers};
        return ops;
    }
};

} // namespace orr
