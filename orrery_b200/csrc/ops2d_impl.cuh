// Launchers of the D2Q9 kernels for one storage type.
#pragma once

#include <algorithm>

#include "kernels2d.cuh"
#include "ops2d.h"

namespace orr {

template <class S> struct Launch2D {
    using A = typename Storage<S>::A;
    static cudaError_t step(const Geom2D& g, const void* phys, const void* src, void* dst,
                            const StepBuffers2D& b, bool smag, uint32_t block, cudaStream_t s) {
        Geom2D gg = g;
        gg.tiles_x = (g.nx + block - 1) / block;
        const unsigned blocks = g.ny * gg.tiles_x;
        const auto& p = *static_cast<const Phys2D<A>*>(phys);
        if (smag) {
            step2d_kernel<S, true><<<blocks, block, 0, s>>>(gg, p, static_cast<const S*>(src),
                                                            static_cast<S*>(dst), b);
        } else {
            step2d_kernel<S, false><<<blocks, block, 0, s>>>(gg, p, static_cast<const S*>(src),
                                                             static_cast<S*>(dst), b);
        }
        return cudaGetLastError();
    }

    static cudaError_t init(const Geom2D& g, const uint8_t* cls, const double* rho,
                            const double* ux, const double* uy, double u0x, double u0y, void* f0,
                            cudaStream_t s) {
        const unsigned blocks = static_cast<unsigned>((g.cells + 255) / 256);
        init2d_kernel<S><<<blocks, 256, 0, s>>>(g, cls, rho, ux, uy, u0x, u0y, static_cast<S*>(f0));
        return cudaGetLastError();
    }

    static cudaError_t history(const Geom2D& g, const void* f, void* hist, cudaStream_t s) {
        history2d_kernel<S><<<(g.ny + 255) / 256, 256, 0, s>>>(g, static_cast<const S*>(f),
                                                               static_cast<A*>(hist));
        return cudaGetLastError();
    }

    static cudaError_t moments(const Geom2D& g, const void* phys, const uint8_t* cls,
                               const void* f, void* m, cudaStream_t s) {
        const unsigned blocks = static_cast<unsigned>((g.cells + 255) / 256);
        moments2d_kernel<S><<<blocks, 256, 0, s>>>(g, *static_cast<const Phys2D<A>*>(phys), cls,
                                                   static_cast<const S*>(f), static_cast<A*>(m));
        return cudaGetLastError();
    }

    static cudaError_t force(const Geom2D& g, const void* f, const uint32_t* lcell,
                             const uint32_t* ldir, uint64_t links, double* out, cudaStream_t s) {
        cudaError_t e = cudaMemsetAsync(out, 0, 3 * sizeof(double), s);
        if (e != cudaSuccess || links == 0) {
            return e;
        }
        const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((links + 255) / 256, 1184));
        force2d_kernel<S><<<blocks, 256, 0, s>>>(g, static_cast<const S*>(f), lcell, ldir, links, out);
        return cudaGetLastError();
    }

    static cudaError_t mass(const Geom2D& g, const uint8_t* cls, const void* f, double* out,
                            cudaStream_t s) {
        cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), s);
        if (e != cudaSuccess) {
            return e;
        }
        const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((g.cells + 255) / 256, 1184));
        mass2d_kernel<S><<<blocks, 256, 0, s>>>(g, cls, static_cast<const S*>(f), out);
        return cudaGetLastError();
    }

    static const Ops2D& table() {
        static const Ops2D ops{&step, &init, &history, &moments, &force, &mass};
        return ops;
    }
};

} // namespace orr
