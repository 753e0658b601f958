// D2Q9 device kernels: the fused pull-stream + collide step, initialisation,
// moments, binary64 momentum-exchange force and mass reductions.
//
// The step follows the reference's D2Q9 pull step
//   CPU   CpuLbm2D::update_row + collide  (src/aero/lbm/lbm2d_cpu.cpp:26-75, 352-404)
//   GPU   lbm_d2q9_step                   (src/render/shaders/lbm/lbm_d2q9_step.comp.glsl,
//                                          lbm_d2q9_common.glsl)
// with resolve_source (src/aero/lbm/lbm2d_internal.h:36-75), organised like
// the D3Q19 step: one thread per node over all rows, every lane storing its
// node in the same step (whole sectors), lanes branching by node class.
#pragma once

#include <cstdint>

#include "kernels3d.cuh"
#include "lattice.h"
#include "orrery_lbm.h"
#include "storage.cuh"

namespace orr {

struct Geom2D {
    uint32_t nx, ny;
    uint64_t cells;
    uint32_t tiles_x;
    int32_t x_mode, outlet_mode;
    int32_t bottom, top; // ORR_WALL_*
    int32_t forced;
};

template <class A> struct Phys2D {
    A tau;
    A smag_c;
    A smag_c2;
    A fx, fy;
    A wall_ux[2]; // bottom, top
    A outlet_speed;
    A inlet_ux, inlet_uy;
};

__device__ __forceinline__ void c2_rt(int j, int& x, int& y) {
    constexpr uint32_t kX = [] {
        uint32_t v = 0;
        for (int i = 0; i < d2::Q; ++i) v |= static_cast<uint32_t>(d2::cx(i) + 1) << (2 * i);
        return v;
    }();
    constexpr uint32_t kY = [] {
        uint32_t v = 0;
        for (int i = 0; i < d2::Q; ++i) v |= static_cast<uint32_t>(d2::cy(i) + 1) << (2 * i);
        return v;
    }();
    x = static_cast<int>((kX >> (2 * j)) & 3u) - 1;
    y = static_cast<int>((kY >> (2 * j)) & 3u) - 1;
}

__device__ __forceinline__ int opposite2_rt(int j) {
    // 1<->3, 2<->4, 5<->7, 6<->8
    return j == 0 ? 0 : (j <= 4 ? ((j + 1) & 3) + 1 : ((j - 5 + 2) & 3) + 5);
}

__device__ __forceinline__ double w2_rt(int j) {
    return j == 0 ? 4.0 / 9.0 : (j <= 4 ? 1.0 / 9.0 : 1.0 / 36.0);
}

// BGK + Guo + Smagorinsky (shifted: lbm_collide, lbm_d2q9_common.glsl;
// unshifted binary64: collide, lbm2d_cpu.cpp:26-75, same operation order).
template <class A, bool kShifted, bool kSmag>
__device__ __forceinline__ void collide2(A (&f)[d2::Q], const Phys2D<A>& p, int forced) {
    if constexpr (kShifted) {
        A drho = 0;
#pragma unroll
        for (int i = 0; i < d2::Q; ++i) drho += f[i];
        const A jx = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
        const A jy = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
        const A rho = A(1) + drho;
        const A inv = A(1) / rho;
        const A ux = (jx + A(0.5) * p.fx) * inv;
        const A uy = (jy + A(0.5) * p.fy) * inv;
        const A uu = ux * ux + uy * uy;
        A tau = p.tau;
        if constexpr (kSmag) {
            // Pi_neq from the second moments (sum c c f_eq = rho (c_s^2 I + u u)).
            const A sxx = f[1] + f[3] + f[5] + f[6] + f[7] + f[8];
            const A syy = f[2] + f[4] + f[5] + f[6] + f[7] + f[8];
            const A sxy = f[5] - f[6] + f[7] - f[8];
            const A iso = drho * A(1.0 / 3.0);
            const A pxx = sxx - iso - rho * ux * ux;
            const A pyy = syy - iso - rho * uy * uy;
            const A pxy = sxy - rho * ux * uy;
            const A strain = sqrt(pxx * pxx + pyy * pyy + A(2) * pxy * pxy);
            tau = A(0.5) * (tau + sqrt(tau * tau + A(kSmagFactor) * p.smag_c2 * strain * inv));
        }
        const A omega = A(1) / tau;
        const A scale = A(1) - A(0.5) * omega;
#pragma unroll
        for (int i = 0; i < d2::Q; ++i) {
            const A ex = A(d2::cx(i)), ey = A(d2::cy(i));
            const A cu = ex * ux + ey * uy;
            const A feq = A(d2::w(i)) * (drho + rho * (A(3) * cu + A(4.5) * cu * cu - A(1.5) * uu));
            A v = f[i] - omega * (f[i] - feq);
            if (forced) {
                v += scale * A(d2::w(i)) *
                     (A(3) * ((ex - ux) * p.fx + (ey - uy) * p.fy) + A(9) * cu * (ex * p.fx + ey * p.fy));
            }
            f[i] = v;
        }
    } else {
        const double rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
        const double jx = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
        const double jy = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
        const double fx = p.fx, fy = p.fy;
        const double ux = (jx + 0.5 * fx) / rho;
        const double uy = (jy + 0.5 * fy) / rho;
        const double base = 1.0 - 1.5 * (ux * ux + uy * uy);
        const double cu[d2::Q] = {0.0, ux, uy, -ux, -uy, ux + uy, uy - ux, -ux - uy, ux - uy};
        double feq[d2::Q];
#pragma unroll
        for (int i = 0; i < d2::Q; ++i) feq[i] = d2::w(i) * rho * (base + cu[i] * (3.0 + 4.5 * cu[i]));
        double tau = p.tau;
        if constexpr (kSmag) {
            double pxx = 0.0, pyy = 0.0, pxy = 0.0;
#pragma unroll
            for (int i = 0; i < d2::Q; ++i) {
                const double neq = f[i] - feq[i];
                const double ex = d2::cx(i), ey = d2::cy(i);
                pxx += ex * ex * neq;
                pyy += ey * ey * neq;
                pxy += ex * ey * neq;
            }
            const double strain = sqrt(pxx * pxx + pyy * pyy + 2.0 * pxy * pxy);
            const double c = p.smag_c;
            tau = 0.5 * (tau + sqrt(tau * tau + kSmagFactor * c * c * strain / rho));
        }
        const double omega = 1.0 / tau;
        const double scale = 1.0 - 0.5 * omega;
#pragma unroll
        for (int i = 0; i < d2::Q; ++i) {
            double v = f[i] - omega * (f[i] - feq[i]);
            if (forced) {
                const double ex = d2::cx(i), ey = d2::cy(i);
                v += scale * d2::w(i) * (3.0 * ((ex - ux) * fx + (ey - uy) * fy) + 9.0 * cu[i] * (ex * fx + ey * fy));
            }
            f[i] = v;
        }
    }
}

// Zou-He west inlet, then regularized (shifted: lbm_zou_he_west; unshifted:
// zou_he_west, lbm2d_internal.h:77-111).
template <class A, bool kShifted>
__device__ __forceinline__ void inlet_west2(A (&f)[d2::Q], A ux, A uy) {
    A rho, drho;
    if constexpr (kShifted) {
        const A s = f[0] + f[2] + f[4] + A(2) * (f[3] + f[6] + f[7]);
        drho = (s + ux) / (A(1) - ux);
        rho = A(1) + drho;
    } else {
        rho = (f[0] + f[2] + f[4] + 2.0 * (f[3] + f[6] + f[7])) / (1.0 - ux);
        drho = 0;
    }
    f[1] = f[3] + (A(2) / A(3)) * rho * ux;
    f[5] = f[7] - A(0.5) * (f[2] - f[4]) + (A(1) / A(6)) * rho * ux + A(0.5) * rho * uy;
    f[8] = f[6] + A(0.5) * (f[2] - f[4]) + (A(1) / A(6)) * rho * ux - A(0.5) * rho * uy;
    const A uu = ux * ux + uy * uy;
    A feq[d2::Q];
    A pxx = 0, pyy = 0, pxy = 0;
#pragma unroll
    for (int i = 0; i < d2::Q; ++i) {
        const A ex = A(d2::cx(i)), ey = A(d2::cy(i));
        const A cu = ex * ux + ey * uy;
        if constexpr (kShifted) {
            feq[i] = A(d2::w(i)) * (drho + rho * (A(3) * cu + A(4.5) * cu * cu - A(1.5) * uu));
        } else {
            feq[i] = A(d2::w(i)) * rho * (A(1) + A(3) * cu + A(4.5) * cu * cu - A(1.5) * uu);
        }
        const A neq = f[i] - feq[i];
        pxx += ex * ex * neq;
        pyy += ey * ey * neq;
        pxy += ex * ey * neq;
    }
    const A cs2 = A(1.0 / 3.0);
#pragma unroll
    for (int i = 0; i < d2::Q; ++i) {
        const A ex = A(d2::cx(i)), ey = A(d2::cy(i));
        f[i] = feq[i] + A(4.5) * A(d2::w(i)) *
                            ((ex * ex - cs2) * pxx + (ey * ey - cs2) * pyy + A(2) * ex * ey * pxy);
    }
}

struct StepBuffers2D {
    const uint8_t* cls;
    const uint32_t* nmask; // per node, bit i: direction i bounces back
    void* hist;
};

template <class S, int I>
__device__ __forceinline__ void gather_one2(const Geom2D& g, const Phys2D<typename Storage<S>::A>& p,
                                            const S* __restrict__ src, const StepBuffers2D& b,
                                            uint32_t mask, int x, int y, uint64_t here,
                                            typename Storage<S>::A& wall_rho,
                                            typename Storage<S>::A& out) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    constexpr int CX = d2::cx(I), CY = d2::cy(I), MY = d2::mirror_y(I);
    const uint64_t cells = g.cells;
    int sx = x - CX, sy = y - CY;
    bool ymir = false;
    if (CY != 0 && (sy < 0 || sy >= static_cast<int>(g.ny))) {
        const int kind = sy < 0 ? g.bottom : g.top;
        if (kind == ORR_WALL_PERIODIC) {
            sy = sy < 0 ? static_cast<int>(g.ny) - 1 : 0;
        } else if (kind == ORR_WALL_SLIP) {
            sy = y;
            ymir = true;
        } else {
            if (wall_rho < A(0)) {
                A r = 0;
#pragma unroll
                for (int k = 0; k < d2::Q; ++k) r += T::load(src + static_cast<uint64_t>(k) * cells + here);
                wall_rho = T::kShifted ? A(1) + r : r;
            }
            out = T::load(src + static_cast<uint64_t>(d2::opposite(I)) * cells + here) +
                  A(6) * A(d2::w(I)) * wall_rho * A(CX) * p.wall_ux[sy < 0 ? 0 : 1];
            return;
        }
    }
    const int dir = ymir ? MY : I;
    if (CX != 0 && (sx < 0 || sx >= static_cast<int>(g.nx))) {
        if (g.x_mode == ORR_X_PERIODIC) {
            sx = sx < 0 ? static_cast<int>(g.nx) - 1 : 0;
        } else if (sx < 0) {
            out = A(0);
            return;
        } else {
            const uint64_t column = (g.nx - 1u) + static_cast<uint64_t>(g.nx) * static_cast<uint64_t>(sy);
            const A up = T::load(src + static_cast<uint64_t>(dir) * cells + column);
            if (g.outlet_mode == ORR_OUTLET_EXTRAPOLATION) {
                out = up;
            } else {
                A* hist = static_cast<A*>(b.hist);
                const uint64_t k = static_cast<uint64_t>(d2::outlet_slot(I)) * g.ny + static_cast<uint64_t>(y);
                const A u = p.outlet_speed;
                const A v = (hist[k] + u * up) / (A(1) + u);
                hist[k] = v;
                out = v;
            }
            return;
        }
    }
    const uint64_t source = static_cast<uint64_t>(sx) + static_cast<uint64_t>(g.nx) * static_cast<uint64_t>(sy);
    if (((mask >> I) & 1u) != 0u) {
        out = T::load(src + static_cast<uint64_t>(d2::opposite(I)) * cells + here);
        return;
    }
    out = T::load(src + static_cast<uint64_t>(dir) * cells + source);
}

template <class S, int I>
__device__ __forceinline__ void gather_all2(const Geom2D& g, const Phys2D<typename Storage<S>::A>& p,
                                            const S* __restrict__ src, const StepBuffers2D& b,
                                            uint32_t mask, int x, int y, uint64_t here,
                                            typename Storage<S>::A& wall_rho,
                                            typename Storage<S>::A (&f)[d2::Q]) {
    if constexpr (I < d2::Q) {
        gather_one2<S, I>(g, p, src, b, mask, x, y, here, wall_rho, f[I]);
        gather_all2<S, I + 1>(g, p, src, b, mask, x, y, here, wall_rho, f);
    }
}

// One fused step src -> dst: one thread per node, one block per row tile,
// all rows; solid lanes store their rest populations, bulk lanes (interior
// rows, x-edges shifted) pull plainly, face and boundary lanes take the
// general gather (see step3d_kernel for the reasons).
template <class S, bool kSmag>
__global__ void __launch_bounds__(256) step2d_kernel(Geom2D g, Phys2D<typename Storage<S>::A> p,
                                                     const S* __restrict__ src, S* __restrict__ dst,
                                                     StepBuffers2D b) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    const uint32_t y = blockIdx.x / g.tiles_x;
    const uint32_t x = (blockIdx.x - y * g.tiles_x) * blockDim.x + threadIdx.x;
    if (x >= g.nx) {
        return;
    }
    const uint64_t here = x + static_cast<uint64_t>(g.nx) * y;
    const uint8_t cls = b.cls[here];
    if (cls == kSolid) {
#pragma unroll
        for (int i = 0; i < d2::Q; ++i) {
            T::store(dst + static_cast<uint64_t>(i) * g.cells + here, T::kShifted ? A(0) : A(d2::w(i)));
        }
        return;
    }
    A f[d2::Q];
    if (cls == kBulk) {
        const int64_t nx = g.nx;
        const bool xlo = x == 0u, xhi = x + 1u == g.nx;
        const int64_t shift_lo = g.x_mode == ORR_X_PERIODIC ? nx : 0;
        const int64_t shift_hi = g.x_mode == ORR_X_PERIODIC ? -nx : -1;
#pragma unroll
        for (int i = 0; i < d2::Q; ++i) {
            int64_t source = static_cast<int64_t>(here) - (d2::cx(i) + nx * d2::cy(i));
            if (d2::cx(i) > 0 && xlo) source += shift_lo;
            if (d2::cx(i) < 0 && xhi) source += shift_hi;
            f[i] = T::load(src + static_cast<uint64_t>(i) * g.cells + static_cast<uint64_t>(source));
        }
        if (xhi && g.x_mode == ORR_X_INFLOW_OUTFLOW && g.outlet_mode == ORR_OUTLET_CONVECTIVE) {
            A* hist = static_cast<A*>(b.hist);
            const A u = p.outlet_speed;
#pragma unroll
            for (int i = 0; i < d2::Q; ++i) {
                if (d2::cx(i) < 0) {
                    const uint64_t k = static_cast<uint64_t>(d2::outlet_slot(i)) * g.ny + y;
                    const A v = (hist[k] + u * f[i]) / (A(1) + u);
                    hist[k] = v;
                    f[i] = v;
                }
            }
        }
    } else {
        const uint32_t mask = cls == kBoundary ? b.nmask[here] : 0u;
        A wall_rho = A(-1);
        gather_all2<S, 0>(g, p, src, b, mask, static_cast<int>(x), static_cast<int>(y), here,
                          wall_rho, f);
    }
    if (g.x_mode == ORR_X_INFLOW_OUTFLOW && x == 0u) {
        inlet_west2<A, T::kShifted>(f, p.inlet_ux, p.inlet_uy);
    }
    collide2<A, T::kShifted, kSmag>(f, p, g.forced);
#pragma unroll
    for (int i = 0; i < d2::Q; ++i) T::store(dst + static_cast<uint64_t>(i) * g.cells + here, f[i]);
}

// Equilibrium initialisation (initial_populations, lbm2d_common.cpp:178-193).
template <class S>
__global__ void init2d_kernel(Geom2D g, const uint8_t* __restrict__ cls, const double* rho,
                              const double* ux, const double* uy, double u0x, double u0y,
                              S* __restrict__ f0) {
    using T = Storage<S>;
    const uint64_t c = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= g.cells) {
        return;
    }
    double r = 1.0, vx = 0.0, vy = 0.0;
    if (cls[c] != kSolid) {
        if (rho != nullptr) {
            r = rho[c];
            vx = ux[c];
            vy = uy[c];
        } else {
            vx = u0x;
            vy = u0y;
        }
    }
#pragma unroll
    for (int i = 0; i < d2::Q; ++i) {
        const double cu = static_cast<double>(d2::cx(i)) * vx + static_cast<double>(d2::cy(i)) * vy;
        const double uu = vx * vx + vy * vy;
        double feq = d2::w(i) * r * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * uu);
        if (T::kShifted) {
            feq -= d2::w(i);
        }
        f0[static_cast<uint64_t>(i) * g.cells + c] = T::encode(feq);
    }
}

// Outlet history (reset_outlet, lbm2d_cpu.cpp:287-297).
template <class S>
__global__ void history2d_kernel(Geom2D g, const S* __restrict__ f, typename Storage<S>::A* __restrict__ hist) {
    using T = Storage<S>;
    const uint32_t y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= g.ny) {
        return;
    }
    const uint64_t cell = (g.nx - 1u) + static_cast<uint64_t>(g.nx) * y;
    constexpr int dirs[3] = {3, 6, 7};
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        hist[static_cast<uint64_t>(d2::outlet_slot(dirs[s])) * g.ny + y] =
            T::load(f + static_cast<uint64_t>(dirs[s]) * g.cells + cell);
    }
}

template <class S>
__global__ void moments2d_kernel(Geom2D g, Phys2D<typename Storage<S>::A> p, const uint8_t* __restrict__ cls,
                                 const S* __restrict__ f, typename Storage<S>::A* __restrict__ m) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    const uint64_t c = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= g.cells) {
        return;
    }
    A r = T::kShifted ? A(0) : A(1), ux = 0, uy = 0;
    if (cls[c] != kSolid) {
        A v[d2::Q];
#pragma unroll
        for (int i = 0; i < d2::Q; ++i) v[i] = T::load(f + static_cast<uint64_t>(i) * g.cells + c);
        A s = 0;
#pragma unroll
        for (int i = 0; i < d2::Q; ++i) s += v[i];
        // CpuLbm2D::macroscopic accumulates c_i v_i in direction order.
        A jx = 0, jy = 0;
#pragma unroll
        for (int i = 0; i < d2::Q; ++i) {
            if (d2::cx(i) > 0) jx = jx + v[i];
            if (d2::cx(i) < 0) jx = jx - v[i];
            if (d2::cy(i) > 0) jy = jy + v[i];
            if (d2::cy(i) < 0) jy = jy - v[i];
        }
        const A rho = T::kShifted ? A(1) + s : s;
        r = s;
        ux = (jx - A(0.5) * p.fx) / rho;
        uy = (jy - A(0.5) * p.fy) / rho;
    }
    m[c] = r;
    m[g.cells + c] = ux;
    m[2 * g.cells + c] = uy;
}

// Force2D over the links: 2 c_o f*_o at the halfway wall point, binary64
// (CpuLbm2D::force, lbm2d_cpu.cpp:265-272; add_link_force, lbm2d.h:145-155).
template <class S>
__global__ void force2d_kernel(Geom2D g, const S* __restrict__ f, const uint32_t* __restrict__ lcell,
                               const uint32_t* __restrict__ ldir, uint64_t links, double* __restrict__ out) {
    using T = Storage<S>;
    double acc[3] = {0, 0, 0};
    for (uint64_t k = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < links;
         k += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t h = lcell[k];
        const int j = static_cast<int>(ldir[k]);
        const int o = opposite2_rt(j);
        int jx, jy;
        c2_rt(j, jx, jy);
        double v = static_cast<double>(T::load(f + static_cast<uint64_t>(o) * g.cells + h));
        if (T::kShifted) {
            v += w2_rt(o);
        }
        const double fx = -2.0 * jx * v, fy = -2.0 * jy * v;
        const uint32_t y = static_cast<uint32_t>(h / g.nx), x = static_cast<uint32_t>(h - static_cast<uint64_t>(y) * g.nx);
        const double rx = static_cast<double>(x) - 0.5 * jx, ry = static_cast<double>(y) - 0.5 * jy;
        acc[0] += fx;
        acc[1] += fy;
        acc[2] += rx * fy - ry * fx;
    }
    block_reduce_add<3>(acc, out);
}

template <class S>
__global__ void mass2d_kernel(Geom2D g, const uint8_t* __restrict__ cls, const S* __restrict__ f,
                              double* __restrict__ out) {
    using T = Storage<S>;
    double acc[1] = {0.0};
    for (uint64_t c = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < g.cells;
         c += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (cls[c] != kSolid) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < d2::Q; ++i) s += static_cast<double>(T::load(f + static_cast<uint64_t>(i) * g.cells + c));
            acc[0] += s;
        }
    }
    block_reduce_add<1>(acc, out);
}

} // namespace orr
