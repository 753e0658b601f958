// D3Q19 device kernels: the fused pull-stream + collide step, initialisation,
// moments, binary64 momentum-exchange force and mass reductions.
//
// The step follows the reference's fused pull step
//   CPU   CpuLbm3D::update_row + collide  (src/aero/lbm3d/lbm3d_cpu.cpp:32-100, 261-322)
//   GPU   lbm_d3q19_step                  (src/render/shaders/lbm/lbm_d3q19_step.comp.glsl,
//                                          lbm_d3q19_common.glsl:87-368)
// with the boundary rules of resolve_source (src/aero/lbm3d/lbm3d_internal.h:57-130).
// A step is one launch of step3d_kernel over all rows; lanes branch by node
// class (see there).
//
// Shifted storage forms collide in binary32 on f - w (the GLSL formulation);
// the binary64 form stores f itself and evaluates every expression in the
// reference CPU solver's order (this translation unit is compiled without
// FMA contraction for it), which makes it the FP64 device oracle.
#pragma once

#include <cstdint>
#include <initializer_list>

#include "lattice.h"
#include "orrery_lbm.h"
#include "storage.cuh"

namespace orr {

// Lattice geometry and launch partition (all integers; by value).
struct Geom3D {
    uint32_t nx, ny, nz;
    uint32_t plane;           // nx * ny
    uint64_t cells;           // nx * ny * nz
    uint32_t tiles_x;         // blocks per row (set by the launcher)
    int32_t x_mode;           // ORR_X_PERIODIC / ORR_X_INFLOW_OUTFLOW
    int32_t outlet_mode;      // ORR_OUTLET_*
    int32_t y_lo, y_hi, z_lo, z_hi; // ORR_WALL_*
    int32_t forced;           // a body force is set (Guo forcing)
    int32_t sponge;           // absorbing layers active
    uint32_t sponge_inlet, sponge_outlet, sponge_sides;
    // Every source resolves to one stored value or an inlet unknown (the
    // convective outlet then blends the zero-gradient copy): y and z sides
    // periodic or free-slip, halfway solid walls (gather_flat3 then serves
    // face and boundary nodes).
    int32_t flat;
};

// Real parameters in the arithmetic type (binary32 parameters are the
// binary32 roundings of the configuration, as a Float32Uniform delivers them,
// src/aero/compute/include/orrery/aero/compute/compute_backend.h:19-23).
template <class A> struct Phys3D {
    A tau;
    A smag_c;     // Smagorinsky constant C (binary64 form)
    A smag_c2;    // C^2 (binary32 forms, as u_smagorinsky_c2)
    A fx, fy, fz; // body force density
    A wall_ux[4]; // y_lo, y_hi, z_lo, z_hi tangential wall speeds
    A outlet_speed;
    A sponge_strength;
};

// 18 sqrt(2) (src/aero/lbm3d/lbm3d_cpu.cpp:23-26).
constexpr double kSmagFactor = 18.0 * 1.4142135623730951;

// c components of a direction known only at run time (the force links), from
// bit-packed tables.
__device__ __forceinline__ void c_rt(int j, int& x, int& y, int& z) {
    // bits 2j..2j+1 hold c + 1 for j = 0..18
    constexpr uint64_t kX = [] {
        uint64_t v = 0;
        for (int i = 0; i < d3::Q; ++i) v |= static_cast<uint64_t>(d3::cx(i) + 1) << (2 * i);
        return v;
    }();
    constexpr uint64_t kY = [] {
        uint64_t v = 0;
        for (int i = 0; i < d3::Q; ++i) v |= static_cast<uint64_t>(d3::cy(i) + 1) << (2 * i);
        return v;
    }();
    constexpr uint64_t kZ = [] {
        uint64_t v = 0;
        for (int i = 0; i < d3::Q; ++i) v |= static_cast<uint64_t>(d3::cz(i) + 1) << (2 * i);
        return v;
    }();
    x = static_cast<int>((kX >> (2 * j)) & 3ULL) - 1;
    y = static_cast<int>((kY >> (2 * j)) & 3ULL) - 1;
    z = static_cast<int>((kZ >> (2 * j)) & 3ULL) - 1;
}

__device__ __forceinline__ int opposite_rt(int j) {
    return j == 0 ? 0 : ((j & 1) ? j + 1 : j - 1);
}

__device__ __forceinline__ double w_rt(int j) {
    return j == 0 ? 1.0 / 3.0 : (j <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
}

// Arithmetic with explicit rounding.  The binary32 step is written with
// these: each operation rounds on its own or is an explicit fused
// multiply-add, so the compiler cannot contract differently in the kernels
// that inline the same node code (row, staged, batched), and all of
// them give the same bits.  The binary64 overloads are the plain operators:
// their unit is built without contraction and keeps the reference CPU
// solver's order (r_fma is an unfused a * b + c there).
__device__ __forceinline__ float r_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float r_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float r_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float r_div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float r_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double r_add(double a, double b) { return a + b; }
__device__ __forceinline__ double r_sub(double a, double b) { return a - b; }
__device__ __forceinline__ double r_mul(double a, double b) { return a * b; }
__device__ __forceinline__ double r_div(double a, double b) { return a / b; }
__device__ __forceinline__ double r_fma(double a, double b, double c) { return a * b + c; }

// Reciprocal and square root of the binary32 collision: the hardware
// approximations refined by one Newton-Raphson step, r' = r + r (1 - x r)
// and s' = s + (y / 2)(x - s^2) with s = x y, y ~ 1/sqrt(x), which lands
// within about half an ulp of the exact value for the positive, normal
// arguments the collision forms (rho, tau, strain sums); a zero square-root
// argument gives zero.  Binary64 keeps exact division and sqrt (it follows
// the reference CPU solver's rounding).
__device__ __forceinline__ float fast_rcp(float x) {
    const float r = __fdividef(1.0f, x);
    return __fmaf_rn(r, __fmaf_rn(-x, r, 1.0f), r);
}
__device__ __forceinline__ double fast_rcp(double x) {
    return 1.0 / x;
}
__device__ __forceinline__ float fast_sqrt(float x) {
    const float y = rsqrtf(x);
    const float s = __fmul_rn(x, y);
    return x == 0.0f ? 0.0f : __fmaf_rn(__fmul_rn(0.5f, y), __fmaf_rn(-s, s, x), s);
}
__device__ __forceinline__ double fast_sqrt(double x) {
    return sqrt(x);
}

// ---------------------------------------------------------------- collide --

// BGK relaxation of two opposite pairs of the shifted binary32 form in
// packed lanes (FMUL2 / FFMA2 / FADD2 of sm_100, each lane rounded like the
// scalar instruction): plus members (fa, fb) with c.u = cu, minus members
// (fa1, fb1) with -cu; f += omega (f_eq - f) with f_eq - w = even +- odd,
// even = w (base + 4.5 rho (c.u)^2), odd = 3 w rho c.u.
__device__ __forceinline__ void relax_pairs2(float& fa, float& fb, float& fa1, float& fb1, float2 cu,
                                             float2 w, float2 w3rho, float2 base2, float2 rho45_2,
                                             float2 omega2) {
    const float2 neg = make_float2(-1.0f, -1.0f);
    const float2 even = __fmul2_rn(w, __ffma2_rn(rho45_2, __fmul2_rn(cu, cu), base2));
    const float2 odd = __fmul2_rn(w3rho, cu);
    const float2 eqp = __fadd2_rn(even, odd);
    const float2 eqm = __ffma2_rn(odd, neg, even);
    float2 P = make_float2(fa, fb), M = make_float2(fa1, fb1);
    P = __ffma2_rn(omega2, __ffma2_rn(P, neg, eqp), P);
    M = __ffma2_rn(omega2, __ffma2_rn(M, neg, eqm), M);
    fa = P.x;
    fb = P.y;
    fa1 = M.x;
    fb1 = M.y;
}

// BGK collision with Guo forcing and the optional Smagorinsky closure.
// Shifted form: lbm3_collide (lbm_d3q19_common.glsl:261-326).
// Unshifted binary64 form: collide (lbm3d_cpu.cpp:32-93), same operation order.
template <class A, bool kShifted, bool kSmag>
__device__ __forceinline__ void collide3(A (&f)[d3::Q], const Phys3D<A>& p, int forced,
                                         A& out_ux, A& out_uy, A& out_uz) {
    if constexpr (kShifted) {
        // Pairwise sums: the density deviation (about 1e-3) is a sum of
        // terms about ten times larger, so a balanced tree keeps more digits
        // than a running sum.  Opposite pairs are summed and differenced two
        // at a time in packed lanes: (f1, f3) with (f2, f4), (f5, f7) with
        // (f6, f8), (f9, f11) with (f10, f12), (f13, f15) with (f14, f16).
        const float2 neg = make_float2(-1.0f, -1.0f);
        const float2 a1 = make_float2(f[1], f[3]), b1 = make_float2(f[2], f[4]);
        const float2 a2 = make_float2(f[5], f[7]), b2 = make_float2(f[6], f[8]);
        const float2 a3 = make_float2(f[9], f[11]), b3 = make_float2(f[10], f[12]);
        const float2 a4 = make_float2(f[13], f[15]), b4 = make_float2(f[14], f[16]);
        const float2 s1 = __fadd2_rn(a1, b1), d1 = __ffma2_rn(b1, neg, a1);
        const float2 s2 = __fadd2_rn(a2, b2), d2 = __ffma2_rn(b2, neg, a2);
        const float2 s3 = __fadd2_rn(a3, b3), d3v = __ffma2_rn(b3, neg, a3);
        const float2 s4 = __fadd2_rn(a4, b4), d4 = __ffma2_rn(b4, neg, a4);
        const float p1 = s1.x, p3 = s1.y, p5 = s2.x, p7 = s2.y, p9 = s3.x, p11 = s3.y, p13 = s4.x,
                    p15 = s4.y, p17 = r_add(f[17], f[18]);
        const float m1 = d1.x, m3 = d1.y, m5 = d2.x, m7 = d2.y, m9 = d3v.x, m11 = d3v.y, m13 = d4.x,
                    m15 = d4.y, m17 = r_sub(f[17], f[18]);
        const float drho = r_add(f[0], r_add(r_add(r_add(p1, p3), r_add(p5, p7)),
                                             r_add(r_add(p9, p11), r_add(r_add(p13, p15), p17))));
        const float jx = r_add(r_add(m1, m7), r_add(m9, r_add(m11, m13)));
        const float jy = r_add(r_add(m3, m7), r_sub(r_add(m15, m17), m9));
        const float jz = r_add(r_add(m5, m11), r_sub(r_sub(m15, m13), m17));
        const float rho = r_add(1.0f, drho);
        const float inv = fast_rcp(rho);
        const float ux = r_mul(r_fma(0.5f, p.fx, jx), inv);
        const float uy = r_mul(r_fma(0.5f, p.fy, jy), inv);
        const float uz = r_mul(r_fma(0.5f, p.fz, jz), inv);
        const float uu = r_fma(uz, uz, r_fma(uy, uy, r_mul(ux, ux)));
        float tau = p.tau;
        if constexpr (kSmag) {
            // Pi_neq = sum c c (f - f_eq).  For the second-order D3Q19
            // equilibrium sum c_a c_b f_eq = rho (c_s^2 delta_ab + u_a u_b)
            // exactly, and sum c c w = c_s^2 delta, so on shifted values
            // Pi_neq = sum c c f_s - drho c_s^2 delta - rho u u; f_eq is then
            // formed on the fly in the relaxation below.  The second moments
            // reuse the opposite-pair sums of the density.
            const float sxx = r_add(r_add(p1, p7), r_add(p9, r_add(p11, p13)));
            const float syy = r_add(r_add(p3, p7), r_add(p9, r_add(p15, p17)));
            const float szz = r_add(r_add(p5, p11), r_add(p13, r_add(p15, p17)));
            const float sxy = r_sub(p7, p9);
            const float sxz = r_sub(p11, p13);
            const float syz = r_sub(p15, p17);
            const float iso = r_mul(drho, 1.0f / 3.0f);
            const float rux = r_mul(rho, ux), ruy = r_mul(rho, uy), ruz = r_mul(rho, uz);
            const float pxx = r_fma(-rux, ux, r_sub(sxx, iso));
            const float pyy = r_fma(-ruy, uy, r_sub(syy, iso));
            const float pzz = r_fma(-ruz, uz, r_sub(szz, iso));
            const float pxy = r_fma(-rux, uy, sxy);
            const float pxz = r_fma(-rux, uz, sxz);
            const float pyz = r_fma(-ruy, uz, syz);
            const float diag = r_fma(pzz, pzz, r_fma(pyy, pyy, r_mul(pxx, pxx)));
            const float off = r_fma(pyz, pyz, r_fma(pxz, pxz, r_mul(pxy, pxy)));
            const float strain = fast_sqrt(r_fma(2.0f, off, diag));
            const float k = r_mul(r_mul(r_mul(static_cast<float>(kSmagFactor), p.smag_c2), strain), inv);
            tau = r_mul(0.5f, r_add(tau, fast_sqrt(r_fma(tau, tau, k))));
        }
        const float omega = fast_rcp(tau);
        // Relaxation towards f_eq,i - w_i = w_i (drho + rho (3 c.u + 4.5 (c.u)^2
        // - 1.5 u.u)), by opposite pairs (c_{i+1} = -c_i for odd i): the even
        // part w (drho - 1.5 rho u.u + 4.5 rho (c.u)^2) is shared and the odd
        // part 3 w rho c.u changes sign.  Two opposite pairs at a time in
        // packed lanes; c.u is written out per direction (components 0, +-1).
        const float base = r_fma(r_mul(-1.5f, rho), uu, drho);
        const float rho45 = r_mul(4.5f, rho);
        constexpr float w0 = 1.0f / 3.0f, w1 = 1.0f / 18.0f, w2 = 1.0f / 36.0f;
        f[0] = r_fma(omega, r_fma(w0, base, -f[0]), f[0]);
        const float2 base2 = make_float2(base, base), rho45_2 = make_float2(rho45, rho45);
        const float2 omega2 = make_float2(omega, omega);
        const float r3a = r_mul(3.0f * w1, rho), r3b = r_mul(3.0f * w2, rho);
        relax_pairs2(f[1], f[3], f[2], f[4], make_float2(ux, uy), make_float2(w1, w1),
                     make_float2(r3a, r3a), base2, rho45_2, omega2);
        relax_pairs2(f[5], f[7], f[6], f[8], make_float2(uz, r_add(ux, uy)), make_float2(w1, w2),
                     make_float2(r3a, r3b), base2, rho45_2, omega2);
        relax_pairs2(f[9], f[11], f[10], f[12], make_float2(r_sub(ux, uy), r_add(ux, uz)), make_float2(w2, w2),
                     make_float2(r3b, r3b), base2, rho45_2, omega2);
        relax_pairs2(f[13], f[15], f[14], f[16], make_float2(r_sub(ux, uz), r_add(uy, uz)), make_float2(w2, w2),
                     make_float2(r3b, r3b), base2, rho45_2, omega2);
        {
            const float cu = r_sub(uy, uz); // direction 17 (0, 1, -1)
            const float even = r_mul(w2, r_fma(rho45, r_mul(cu, cu), base));
            const float odd = r_mul(r3b, cu);
            f[17] = r_fma(omega, r_sub(r_add(even, odd), f[17]), f[17]);
            f[18] = r_fma(omega, r_sub(r_sub(even, odd), f[18]), f[18]);
        }
        if (forced) {
            // Guo forcing: w (1 - omega / 2) (3 (c - u).F + 9 (c.u)(c.F)).
            const float scale = r_fma(-0.5f, omega, 1.0f);
#pragma unroll
            for (int i = 0; i < d3::Q; ++i) {
                const float ex = static_cast<float>(d3::cx(i)), ey = static_cast<float>(d3::cy(i)),
                            ez = static_cast<float>(d3::cz(i));
                const float cu = r_fma(ez, uz, r_fma(ey, uy, r_mul(ex, ux)));
                const float cf = r_fma(ez, p.fz, r_fma(ey, p.fy, r_mul(ex, p.fx)));
                const float uf = r_fma(r_sub(ez, uz), p.fz, r_fma(r_sub(ey, uy), p.fy, r_mul(r_sub(ex, ux), p.fx)));
                const float term = r_fma(3.0f, uf, r_mul(r_mul(9.0f, cu), cf));
                f[i] = r_fma(r_mul(scale, static_cast<float>(d3::w(i))), term, f[i]);
            }
        }
        out_ux = ux;
        out_uy = uy;
        out_uz = uz;
    } else {
        double rho = 0.0;
#pragma unroll
        for (int i = 0; i < d3::Q; ++i) rho += f[i];
        const double jx = f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[11] - f[12] + f[13] - f[14];
        const double jy = f[3] - f[4] + f[7] - f[8] - f[9] + f[10] + f[15] - f[16] + f[17] - f[18];
        const double jz = f[5] - f[6] + f[11] - f[12] - f[13] + f[14] + f[15] - f[16] - f[17] + f[18];
        const double fx = p.fx, fy = p.fy, fz = p.fz;
        const double ux = (jx + 0.5 * fx) / rho;
        const double uy = (jy + 0.5 * fy) / rho;
        const double uz = (jz + 0.5 * fz) / rho;
        const double base = 1.0 - 1.5 * (ux * ux + uy * uy + uz * uz);
        const double cu[d3::Q] = {0.0,     ux,       -ux,     uy,      -uy,     uz,       -uz,
                                  ux + uy, -ux - uy, ux - uy, uy - ux, ux + uz, -ux - uz, ux - uz,
                                  uz - ux, uy + uz,  -uy - uz, uy - uz, uz - uy};
        double feq[d3::Q];
#pragma unroll
        for (int i = 0; i < d3::Q; ++i) {
            feq[i] = d3::w(i) * rho * (base + cu[i] * (3.0 + 4.5 * cu[i]));
        }
        double tau = p.tau;
        if constexpr (kSmag) {
            double pi[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int i = 0; i < d3::Q; ++i) {
                const double neq = f[i] - feq[i];
                const double ex = d3::cx(i), ey = d3::cy(i), ez = d3::cz(i);
                pi[0] += ex * ex * neq;
                pi[1] += ey * ey * neq;
                pi[2] += ez * ez * neq;
                pi[3] += ex * ey * neq;
                pi[4] += ex * ez * neq;
                pi[5] += ey * ez * neq;
            }
            const double strain = sqrt(pi[0] * pi[0] + pi[1] * pi[1] + pi[2] * pi[2] +
                                       2.0 * (pi[3] * pi[3] + pi[4] * pi[4] + pi[5] * pi[5]));
            const double c = p.smag_c;
            tau = 0.5 * (tau + sqrt(tau * tau + kSmagFactor * c * c * strain / rho));
        }
        const double omega = 1.0 / tau;
        const double scale = 1.0 - 0.5 * omega;
#pragma unroll
        for (int i = 0; i < d3::Q; ++i) {
            double v = f[i] - omega * (f[i] - feq[i]);
            if (forced) {
                const double ex = d3::cx(i), ey = d3::cy(i), ez = d3::cz(i);
                v += scale * d3::w(i) *
                     (3.0 * ((ex - ux) * fx + (ey - uy) * fy + (ez - uz) * fz) +
                      9.0 * cu[i] * (ex * fx + ey * fy + ez * fz));
            }
            f[i] = v;
        }
        out_ux = ux;
        out_uy = uy;
        out_uz = uz;
    }
}

// Relaxation rate of the absorbing layers at (x, y, z)
// (sponge_sigma, lbm3d_internal.h:255-281; lbm3_sponge, glsl:336-353).
template <class A>
__device__ __forceinline__ A sponge_rate3(const Geom3D& g, const Phys3D<A>& p, uint32_t x,
                                          uint32_t y, uint32_t z) {
    A best = 0;
    const auto layer = [&best](uint32_t d, uint32_t t) {
        if (d < t) {
            const A r = r_div(A(t - d), A(t));
            const A v = r_mul(r, r);
            best = best < v ? v : best;
        }
    };
    layer(x, g.sponge_inlet);
    layer(g.nx - 1u - x, g.sponge_outlet);
    if (g.y_lo != ORR_WALL_PERIODIC) {
        layer(y, g.sponge_sides);
        layer(g.ny - 1u - y, g.sponge_sides);
    }
    if (g.z_lo != ORR_WALL_PERIODIC) {
        layer(z, g.sponge_sides);
        layer(g.nz - 1u - z, g.sponge_sides);
    }
    return r_mul(p.sponge_strength, best);
}

// Absorbing-layer relaxation towards f_eq(1, u_inlet)
// (collide tail, lbm3d_cpu.cpp:94-99; lbm3_absorb, glsl:355-368).
template <class A, bool kShifted>
__device__ __forceinline__ void absorb3(A (&f)[d3::Q], A s, const A* inlet) {
    const A ux = inlet[0], uy = inlet[1], uz = inlet[2];
#pragma unroll
    for (int i = 0; i < d3::Q; ++i) {
        const A cu = r_add(r_add(r_mul(A(d3::cx(i)), ux), r_mul(A(d3::cy(i)), uy)), r_mul(A(d3::cz(i)), uz));
        const A uu = r_add(r_add(r_mul(ux, ux), r_mul(uy, uy)), r_mul(uz, uz));
        const A quad = r_add(r_mul(A(3), cu), r_mul(r_mul(A(4.5), cu), cu));
        A target;
        if constexpr (kShifted) {
            target = r_mul(A(d3::w(i)), r_sub(quad, r_mul(A(1.5), uu)));
        } else {
            target = r_mul(r_mul(A(d3::w(i)), A(1)),
                           r_sub(r_add(r_add(A(1), r_mul(A(3), cu)), r_mul(r_mul(A(4.5), cu), cu)),
                                 r_mul(A(1.5), uu)));
        }
        f[i] = r_sub(f[i], r_mul(s, r_sub(f[i], target)));
    }
}

// Two nodes at once in packed binary32 lanes (node A in .x, node B in .y).
// Each helper rounds every lane like the scalar r_* operation it stands for
// (a - b as the single-rounding fma(b, -1, a); -a as a * -1, exact), so the
// pair collision gives the bits of two single-node collisions.
__device__ __forceinline__ float2 v2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 p_sub(float2 a, float2 b) { return __ffma2_rn(b, v2(-1.0f), a); }
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 p_neg(float2 a) { return __fmul2_rn(a, v2(-1.0f)); }
__device__ __forceinline__ float2 p_rcp(float2 a) { return make_float2(fast_rcp(a.x), fast_rcp(a.y)); }
__device__ __forceinline__ float2 p_sqrt(float2 a) { return make_float2(fast_sqrt(a.x), fast_sqrt(a.y)); }

// One opposite pair (plus member with c.u = cu, minus member with -cu) of two
// nodes: the relaxation of relax_pairs2 lane by lane.
__device__ __forceinline__ void relax_opposite2(float2& fp, float2& fm, float2 cu, float w, float2 r3, float2 base,
                                                float2 rho45, float2 omega) {
    const float2 even = p_mul(v2(w), p_fma(rho45, p_mul(cu, cu), base));
    const float2 odd = p_mul(r3, cu);
    const float2 eqp = p_add(even, odd);
    const float2 eqm = p_sub(even, odd);
    fp = p_fma(omega, p_sub(eqp, fp), fp);
    fm = p_fma(omega, p_sub(eqm, fm), fm);
}

// The shifted binary32 collision of collide3 for two nodes, operation for
// operation (each scalar operation there is one packed operation here, each
// packed pair there two here).
template <bool kSmag>
__device__ __forceinline__ void collide3_pair(float2 (&f)[d3::Q], const Phys3D<float>& p, int forced) {
    const float2 p1 = p_add(f[1], f[2]), p3 = p_add(f[3], f[4]), p5 = p_add(f[5], f[6]);
    const float2 p7 = p_add(f[7], f[8]), p9 = p_add(f[9], f[10]), p11 = p_add(f[11], f[12]);
    const float2 p13 = p_add(f[13], f[14]), p15 = p_add(f[15], f[16]), p17 = p_add(f[17], f[18]);
    const float2 m1 = p_sub(f[1], f[2]), m3 = p_sub(f[3], f[4]), m5 = p_sub(f[5], f[6]);
    const float2 m7 = p_sub(f[7], f[8]), m9 = p_sub(f[9], f[10]), m11 = p_sub(f[11], f[12]);
    const float2 m13 = p_sub(f[13], f[14]), m15 = p_sub(f[15], f[16]), m17 = p_sub(f[17], f[18]);
    const float2 drho = p_add(f[0], p_add(p_add(p_add(p1, p3), p_add(p5, p7)),
                                          p_add(p_add(p9, p11), p_add(p_add(p13, p15), p17))));
    const float2 jx = p_add(p_add(m1, m7), p_add(m9, p_add(m11, m13)));
    const float2 jy = p_add(p_add(m3, m7), p_sub(p_add(m15, m17), m9));
    const float2 jz = p_add(p_add(m5, m11), p_sub(p_sub(m15, m13), m17));
    const float2 rho = p_add(v2(1.0f), drho);
    const float2 inv = p_rcp(rho);
    const float2 ux = p_mul(p_fma(v2(0.5f), v2(p.fx), jx), inv);
    const float2 uy = p_mul(p_fma(v2(0.5f), v2(p.fy), jy), inv);
    const float2 uz = p_mul(p_fma(v2(0.5f), v2(p.fz), jz), inv);
    const float2 uu = p_fma(uz, uz, p_fma(uy, uy, p_mul(ux, ux)));
    float2 omega;
    if constexpr (kSmag) {
        const float2 sxx = p_add(p_add(p1, p7), p_add(p9, p_add(p11, p13)));
        const float2 syy = p_add(p_add(p3, p7), p_add(p9, p_add(p15, p17)));
        const float2 szz = p_add(p_add(p5, p11), p_add(p13, p_add(p15, p17)));
        const float2 sxy = p_sub(p7, p9);
        const float2 sxz = p_sub(p11, p13);
        const float2 syz = p_sub(p15, p17);
        const float2 iso = p_mul(drho, v2(1.0f / 3.0f));
        const float2 nrux = p_neg(p_mul(rho, ux)), nruy = p_neg(p_mul(rho, uy)), nruz = p_neg(p_mul(rho, uz));
        const float2 pxx = p_fma(nrux, ux, p_sub(sxx, iso));
        const float2 pyy = p_fma(nruy, uy, p_sub(syy, iso));
        const float2 pzz = p_fma(nruz, uz, p_sub(szz, iso));
        const float2 pxy = p_fma(nrux, uy, sxy);
        const float2 pxz = p_fma(nrux, uz, sxz);
        const float2 pyz = p_fma(nruy, uz, syz);
        const float2 diag = p_fma(pzz, pzz, p_fma(pyy, pyy, p_mul(pxx, pxx)));
        const float2 off = p_fma(pyz, pyz, p_fma(pxz, pxz, p_mul(pxy, pxy)));
        const float2 strain = p_sqrt(p_fma(v2(2.0f), off, diag));
        const float2 k = p_mul(p_mul(v2(r_mul(static_cast<float>(kSmagFactor), p.smag_c2)), strain), inv);
        const float2 tau = v2(p.tau);
        omega = p_rcp(p_mul(v2(0.5f), p_add(tau, p_sqrt(p_fma(tau, tau, k)))));
    } else {
        omega = v2(fast_rcp(p.tau));
    }
    const float2 base = p_fma(p_mul(v2(-1.5f), rho), uu, drho);
    const float2 rho45 = p_mul(v2(4.5f), rho);
    constexpr float w0 = 1.0f / 3.0f, w1 = 1.0f / 18.0f, w2 = 1.0f / 36.0f;
    f[0] = p_fma(omega, p_fma(v2(w0), base, p_neg(f[0])), f[0]);
    const float2 r3a = p_mul(v2(3.0f * w1), rho), r3b = p_mul(v2(3.0f * w2), rho);
    relax_opposite2(f[1], f[2], ux, w1, r3a, base, rho45, omega);
    relax_opposite2(f[3], f[4], uy, w1, r3a, base, rho45, omega);
    relax_opposite2(f[5], f[6], uz, w1, r3a, base, rho45, omega);
    relax_opposite2(f[7], f[8], p_add(ux, uy), w2, r3b, base, rho45, omega);
    relax_opposite2(f[9], f[10], p_sub(ux, uy), w2, r3b, base, rho45, omega);
    relax_opposite2(f[11], f[12], p_add(ux, uz), w2, r3b, base, rho45, omega);
    relax_opposite2(f[13], f[14], p_sub(ux, uz), w2, r3b, base, rho45, omega);
    relax_opposite2(f[15], f[16], p_add(uy, uz), w2, r3b, base, rho45, omega);
    relax_opposite2(f[17], f[18], p_sub(uy, uz), w2, r3b, base, rho45, omega);
    if (forced) {
        const float2 scale = p_fma(v2(-0.5f), omega, v2(1.0f));
#pragma unroll
        for (int i = 0; i < d3::Q; ++i) {
            const float ex = static_cast<float>(d3::cx(i)), ey = static_cast<float>(d3::cy(i)),
                        ez = static_cast<float>(d3::cz(i));
            const float2 cu = p_fma(v2(ez), uz, p_fma(v2(ey), uy, p_mul(v2(ex), ux)));
            const float cf = r_fma(ez, p.fz, r_fma(ey, p.fy, r_mul(ex, p.fx)));
            const float2 uf = p_fma(p_sub(v2(ez), uz), v2(p.fz),
                                    p_fma(p_sub(v2(ey), uy), v2(p.fy), p_mul(p_sub(v2(ex), ux), v2(p.fx))));
            const float2 term = p_fma(v2(3.0f), uf, p_mul(p_mul(v2(9.0f), cu), v2(cf)));
            f[i] = p_fma(p_mul(scale, v2(static_cast<float>(d3::w(i)))), term, f[i]);
        }
    }
}

// absorb3 for two nodes with their own layer rates (a node with rate 0 keeps
// its values, as absorb3 is then not applied to it).
__device__ __forceinline__ void absorb3_pair(float2 (&f)[d3::Q], float sa, float sb, const float* inlet) {
    const float ux = inlet[0], uy = inlet[1], uz = inlet[2];
    const float2 s = make_float2(sa, sb);
#pragma unroll
    for (int i = 0; i < d3::Q; ++i) {
        const float cu = r_add(r_add(r_mul(float(d3::cx(i)), ux), r_mul(float(d3::cy(i)), uy)),
                               r_mul(float(d3::cz(i)), uz));
        const float uu = r_add(r_add(r_mul(ux, ux), r_mul(uy, uy)), r_mul(uz, uz));
        const float quad = r_add(r_mul(3.0f, cu), r_mul(r_mul(4.5f, cu), cu));
        const float target = r_mul(float(d3::w(i)), r_sub(quad, r_mul(1.5f, uu)));
        const float2 r = p_sub(f[i], p_mul(s, p_sub(f[i], v2(target))));
        f[i] = make_float2(sa > 0.0f ? r.x : f[i].x, sb > 0.0f ? r.y : f[i].y);
    }
}

// Regularized Zou-He velocity inlet on the west face.
// Shifted: lbm3_inlet_west (glsl:105-162).  Unshifted binary64:
// velocity_inlet_west (lbm3d_internal.h:312-365), same operation order.
template <class A, bool kShifted>
__device__ __forceinline__ void inlet_west3(A (&f)[d3::Q], const A* inlet) {
    const A ux = inlet[0], uy = inlet[1], uz = inlet[2];
    A known = 0;
#pragma unroll
    for (int i = 0; i < d3::Q; ++i) {
        if (d3::cx(i) == 0) {
            known = r_add(known, f[i]);
        } else if (d3::cx(i) < 0) {
            known = r_add(known, r_mul(A(2), f[i]));
        }
    }
    A rho, drho;
    if constexpr (kShifted) {
        drho = r_div(r_add(known, ux), r_sub(A(1), ux));
        rho = r_add(A(1), drho);
    } else {
        rho = r_div(known, r_sub(A(1), ux));
        drho = 0;
    }
    if constexpr (kShifted) {
        // The five unknowns (c_x = +1): c.u written out per direction.
        const A r6a = r_mul(A(6) * A(1.0 / 18.0), rho), r6b = r_mul(A(6) * A(1.0 / 36.0), rho);
        f[1] = r_add(f[2], r_mul(r6a, ux));
        f[7] = r_add(f[8], r_mul(r6b, r_add(ux, uy)));
        f[9] = r_add(f[10], r_mul(r6b, r_sub(ux, uy)));
        f[11] = r_add(f[12], r_mul(r6b, r_add(ux, uz)));
        f[13] = r_add(f[14], r_mul(r6b, r_sub(ux, uz)));
    } else {
#pragma unroll
        for (int i = 0; i < d3::Q; ++i) {
            if (d3::cx(i) > 0) {
                const A cu = r_add(r_add(r_mul(A(d3::cx(i)), ux), r_mul(A(d3::cy(i)), uy)),
                                   r_mul(A(d3::cz(i)), uz));
                f[i] = r_add(f[d3::opposite(i)], r_mul(r_mul(A(6) * A(d3::w(i)), rho), cu));
            }
        }
    }
    const A uu = r_add(r_add(r_mul(ux, ux), r_mul(uy, uy)), r_mul(uz, uz));
    if constexpr (kShifted) {
        // Pi_neq from the second moments of the reconstructed set (sum c c f_eq
        // = rho (c_s^2 I + u u); shifted: drho c_s^2 I + rho u u), then
        // f = f_eq + 4.5 w (c c - c_s^2 I) : Pi_neq with f_eq formed on the fly.
        const auto sum = [](std::initializer_list<A> v) {
            A t = 0;
            bool first = true;
            for (A x : v) {
                t = first ? x : r_add(t, x);
                first = false;
            }
            return t;
        };
        const A iso = r_mul(drho, A(1.0 / 3.0));
        const A pxx = r_sub(r_sub(sum({f[1], f[2], f[7], f[8], f[9], f[10], f[11], f[12], f[13], f[14]}), iso),
                            r_mul(r_mul(rho, ux), ux));
        const A pyy = r_sub(r_sub(sum({f[3], f[4], f[7], f[8], f[9], f[10], f[15], f[16], f[17], f[18]}), iso),
                            r_mul(r_mul(rho, uy), uy));
        const A pzz = r_sub(r_sub(sum({f[5], f[6], f[11], f[12], f[13], f[14], f[15], f[16], f[17], f[18]}), iso),
                            r_mul(r_mul(rho, uz), uz));
        const A pxy = r_sub(r_sub(r_sub(r_add(f[7], f[8]), f[9]), f[10]), r_mul(r_mul(rho, ux), uy));
        const A pxz = r_sub(r_sub(r_sub(r_add(f[11], f[12]), f[13]), f[14]), r_mul(r_mul(rho, ux), uz));
        const A pyz = r_sub(r_sub(r_sub(r_add(f[15], f[16]), f[17]), f[18]), r_mul(r_mul(rho, uy), uz));
        // (c c - c_s^2 I) : Pi_neq by direction, the zero terms left out:
        // -tr/3 plus the diagonal entries of the axes c moves along, plus
        // 2 c_a c_b of the off-diagonal one; even in c, so shared by opposites.
        const A t0 = r_mul(A(-1.0 / 3.0), r_add(r_add(pxx, pyy), pzz));
        const A tx = r_add(pxx, t0), ty = r_add(pyy, t0), tz = r_add(pzz, t0);
        const A txy = r_add(tx, pyy), txz = r_add(tx, pzz), tyz = r_add(ty, pzz);
        const A p2xy = r_mul(A(2), pxy), p2xz = r_mul(A(2), pxz), p2yz = r_mul(A(2), pyz);
        // f_eq - w = w (drho + rho (3 c.u + 4.5 (c.u)^2 - 1.5 u.u)) for a pair of
        // opposite directions (c.u = +-cu): even part shared, odd part signed.
        const A uu15 = r_mul(A(1.5), uu);
        const auto pair = [&](int plus, int minus, A cu, A t, A w) {
            const A even = r_sub(r_mul(r_mul(A(4.5), cu), cu), uu15);
            const A odd = r_mul(A(3), cu);
            const A neq = r_mul(A(4.5) * w, t);
            f[plus] = r_add(r_mul(w, r_add(drho, r_mul(rho, r_add(even, odd)))), neq);
            f[minus] = r_add(r_mul(w, r_add(drho, r_mul(rho, r_sub(even, odd)))), neq);
        };
        constexpr A w0 = A(1.0 / 3.0), w1 = A(1.0 / 18.0), w2 = A(1.0 / 36.0);
        f[0] = r_add(r_mul(w0, r_add(drho, r_mul(rho, -uu15))), r_mul(A(4.5) * w0, t0));
        pair(1, 2, ux, tx, w1);
        pair(3, 4, uy, ty, w1);
        pair(5, 6, uz, tz, w1);
        pair(7, 8, r_add(ux, uy), r_add(txy, p2xy), w2);
        pair(9, 10, r_sub(ux, uy), r_sub(txy, p2xy), w2);
        pair(11, 12, r_add(ux, uz), r_add(txz, p2xz), w2);
        pair(13, 14, r_sub(ux, uz), r_sub(txz, p2xz), w2);
        pair(15, 16, r_add(uy, uz), r_add(tyz, p2yz), w2);
        pair(17, 18, r_sub(uy, uz), r_sub(tyz, p2yz), w2);
        return;
    }
    A feq[d3::Q];
    A pi0 = 0, pi1 = 0, pi2 = 0, pi3 = 0, pi4 = 0, pi5 = 0;
#pragma unroll
    for (int i = 0; i < d3::Q; ++i) {
        const A ex = A(d3::cx(i)), ey = A(d3::cy(i)), ez = A(d3::cz(i));
        const A cu = ex * ux + ey * uy + ez * uz;
        if constexpr (kShifted) {
            feq[i] = A(d3::w(i)) * (drho + rho * (A(3) * cu + A(4.5) * cu * cu - A(1.5) * uu));
        } else {
            feq[i] = A(d3::w(i)) * rho * (A(1) + A(3) * cu + A(4.5) * cu * cu - A(1.5) * uu);
        }
        const A neq = f[i] - feq[i];
        pi0 += ex * ex * neq;
        pi1 += ey * ey * neq;
        pi2 += ez * ez * neq;
        pi3 += ex * ey * neq;
        pi4 += ex * ez * neq;
        pi5 += ey * ez * neq;
    }
    const A cs2 = A(1.0 / 3.0);
#pragma unroll
    for (int i = 0; i < d3::Q; ++i) {
        const A ex = A(d3::cx(i)), ey = A(d3::cy(i)), ez = A(d3::cz(i));
        f[i] = feq[i] + A(4.5) * A(d3::w(i)) *
                            ((ex * ex - cs2) * pi0 + (ey * ey - cs2) * pi1 + (ez * ez - cs2) * pi2 +
                             A(2) * (ex * ey * pi3 + ex * ez * pi4 + ey * ez * pi5));
    }
}

// ------------------------------------------------------------------- step --

struct StepBuffers3D {
    const uint8_t* cls;      // node classes
    const uint32_t* nmask;   // per node, bit i: direction i bounces back (solid source)
    const int32_t* nslot;    // per node wall slot of the interpolated wall, -1 none (or null)
    const void* wall_q;      // 19 fractions per slot (arithmetic type)
    void* hist;              // convective-outlet history (arithmetic type)
    const void* inlet;       // imposed inlet velocity, 3 values (arithmetic type)
};

// The population `here` receives from the wall of its link i (reflected,
// lbm3d_internal.h:181-197; lbm3_reflected, glsl:164-181).
template <class S, int I>
__device__ __forceinline__ typename Storage<S>::A reflected3(const S* __restrict__ src,
                                                             uint64_t cells, uint64_t here,
                                                             int64_t farther_off,
                                                             typename Storage<S>::A q) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    constexpr int O = d3::opposite(I);
    const A leaving = T::load(src + static_cast<uint64_t>(O) * cells + here);
    if (q == A(0.5)) {
        return leaving;
    }
    const A q2 = r_mul(A(2), q);
    if (q < A(0.5)) {
        const uint64_t farther = static_cast<uint64_t>(static_cast<int64_t>(here) + farther_off);
        return r_add(r_mul(q2, leaving), r_mul(r_sub(A(1), q2), T::load(src + O * cells + farther)));
    }
    return r_div(r_add(leaving, r_mul(r_sub(q2, A(1)), T::load(src + static_cast<uint64_t>(I) * cells + here))),
                 q2);
}

// General gather of direction I at node (x, y, z) (resolve_source,
// lbm3d_internal.h:87-130, and the CPU's per-kind handling, lbm3d_cpu.cpp:281-312).
// Whether the source is solid comes from the plan's per-node mask (bit i),
// so no load waits on another; kSolid = false drops the test for nodes the
// plan knows have no solid source.
template <class S, int I, bool kSolid>
__device__ __forceinline__ void gather_one3(const Geom3D& g, const Phys3D<typename Storage<S>::A>& p,
                                            const S* __restrict__ src, const StepBuffers3D& b,
                                            int32_t slot, uint32_t mask, int x, int y, int z,
                                            uint64_t here,
                                            typename Storage<S>::A& wall_rho,
                                            typename Storage<S>::A& out) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    constexpr int CX = d3::cx(I), CY = d3::cy(I), CZ = d3::cz(I);
    constexpr int MY = d3::mirror_y(I);
    constexpr int MZ = d3::mirror_z(I);
    constexpr int MZY = d3::mirror_z(d3::mirror_y(I));
    const uint64_t cells = g.cells;
    int sx = x - CX, sy = y - CY, sz = z - CZ;
    bool ymir = false, zmir = false;
    int wall_side = -1;
    if (CY != 0 && (sy < 0 || sy >= static_cast<int>(g.ny))) {
        const int kind = sy < 0 ? g.y_lo : g.y_hi;
        if (kind == ORR_WALL_PERIODIC) {
            sy = sy < 0 ? static_cast<int>(g.ny) - 1 : 0;
        } else if (kind == ORR_WALL_SLIP) {
            sy = y;
            ymir = true;
        } else {
            wall_side = sy < 0 ? 0 : 1;
        }
    }
    if (wall_side < 0 && CZ != 0 && (sz < 0 || sz >= static_cast<int>(g.nz))) {
        const int kind = sz < 0 ? g.z_lo : g.z_hi;
        if (kind == ORR_WALL_PERIODIC) {
            sz = sz < 0 ? static_cast<int>(g.nz) - 1 : 0;
        } else if (kind == ORR_WALL_SLIP) {
            sz = z;
            zmir = true;
        } else {
            wall_side = sz < 0 ? 2 : 3;
        }
    }
    if (wall_side >= 0) {
        // No-slip domain wall: bounce-back plus the moving-wall term scaled
        // by the node's own density at the previous step.
        if (wall_rho < A(0)) {
            A r = 0;
#pragma unroll
            for (int k = 0; k < d3::Q; ++k) r += T::load(src + static_cast<uint64_t>(k) * cells + here);
            wall_rho = T::kShifted ? A(1) + r : r;
        }
        out = r_add(T::load(src + static_cast<uint64_t>(d3::opposite(I)) * cells + here),
                    r_mul(r_mul(r_mul(A(6) * A(d3::w(I)), wall_rho), A(CX)), p.wall_ux[wall_side]));
        return;
    }
    const int dir = zmir ? (ymir ? MZY : MZ) : (ymir ? MY : I);
    if (CX != 0 && (sx < 0 || sx >= static_cast<int>(g.nx))) {
        if (g.x_mode == ORR_X_PERIODIC) {
            sx = sx < 0 ? static_cast<int>(g.nx) - 1 : 0;
        } else if (sx < 0) {
            out = A(0); // reconstructed by the inlet
            return;
        } else {
            // Outlet: the zero-gradient value, blended with the node's
            // history by the convective outlet (outlet_value, lbm3d_cpu.cpp:239-250).
            const uint64_t face = (g.nx - 1u) + static_cast<uint64_t>(g.nx) *
                                                    (static_cast<uint64_t>(sy) + static_cast<uint64_t>(g.ny) * sz);
            const A up = T::load(src + static_cast<uint64_t>(dir) * cells + face);
            if (g.outlet_mode == ORR_OUTLET_EXTRAPOLATION) {
                out = up;
            } else {
                A* hist = static_cast<A*>(b.hist);
                const uint64_t k = static_cast<uint64_t>(d3::outlet_slot(I)) * g.ny * g.nz +
                                   static_cast<uint64_t>(y) + static_cast<uint64_t>(g.ny) * z;
                const A u = p.outlet_speed;
                const A v = r_div(r_add(hist[k], r_mul(u, up)), r_add(A(1), u));
                hist[k] = v;
                out = v;
            }
            return;
        }
    }
    const uint64_t source = static_cast<uint64_t>(sx) +
                            static_cast<uint64_t>(g.nx) * (static_cast<uint64_t>(sy) +
                                                           static_cast<uint64_t>(g.ny) * sz);
    if (kSolid && ((mask >> I) & 1u) != 0u) {
        const A q = slot >= 0 ? static_cast<const A*>(b.wall_q)[static_cast<uint64_t>(slot) * d3::Q + I]
                              : A(0.5);
        const int64_t farther_off = static_cast<int64_t>(CX) + static_cast<int64_t>(g.nx) * CY +
                                    static_cast<int64_t>(g.plane) * CZ;
        out = reflected3<S, I>(src, cells, here, farther_off, q);
        return;
    }
    out = T::load(src + static_cast<uint64_t>(dir) * cells + source);
}

template <class S, int I, bool kSolid>
__device__ __forceinline__ void gather_all3(const Geom3D& g, const Phys3D<typename Storage<S>::A>& p,
                                            const S* __restrict__ src, const StepBuffers3D& b,
                                            int32_t slot, uint32_t mask, int x, int y, int z,
                                            uint64_t here, typename Storage<S>::A& wall_rho,
                                            typename Storage<S>::A (&f)[d3::Q]) {
    if constexpr (I < d3::Q) {
        gather_one3<S, I, kSolid>(g, p, src, b, slot, mask, x, y, z, here, wall_rho, f[I]);
        gather_all3<S, I + 1, kSolid>(g, p, src, b, slot, mask, x, y, z, here, wall_rho, f);
    }
}

// Collision, absorbing layers and the 19 stores of one node.
template <class S, bool kSmag>
__device__ __forceinline__ void finish3(const Geom3D& g, const Phys3D<typename Storage<S>::A>& p,
                                        const StepBuffers3D& b, typename Storage<S>::A (&f)[d3::Q],
                                        uint32_t x, uint32_t y, uint32_t z, uint64_t here,
                                        S* __restrict__ dst) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    A ux, uy, uz;
    collide3<A, T::kShifted, kSmag>(f, p, g.forced, ux, uy, uz);
    if (g.sponge) {
        const A s = sponge_rate3<A>(g, p, x, y, z);
        if (s > A(0)) {
            absorb3<A, T::kShifted>(f, s, static_cast<const A*>(b.inlet));
        }
    }
    // Population i of the node at (dst + i * cells) + here: the first sum is
    // the same for every thread, the second one wide multiply-add of the
    // 32-bit node index (lattices hold fewer than 2^32 / 19 nodes).
    const uint32_t h = static_cast<uint32_t>(here);
#pragma unroll
    for (int i = 0; i < d3::Q; ++i) {
        T::store(dst + static_cast<uint64_t>(i) * g.cells + h, f[i]);
    }
}

// General gather of a lattice with g.flat set: the rules of gather_one3 for
// periodic / free-slip sides, the inlet unknowns, the outlet copy and
// halfway bounce-back, in which every direction's value is one stored
// population (or 0 for an inlet unknown).  At x = nx - 1 of an inflow /
// outflow lattice the caller applies convective_blend3 to the copies.  The source of each direction is
// resolved with integer selects first and the 19 loads are then independent,
// so a face or boundary node waits for one round trip instead of a chain.
template <class S>
__device__ __forceinline__ void gather_flat3(const Geom3D& g, const S* __restrict__ src, uint32_t mask,
                                             int x, int y, int z, uint64_t here,
                                             typename Storage<S>::A (&f)[d3::Q]) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    const int nx = static_cast<int>(g.nx), ny = static_cast<int>(g.ny), nz = static_cast<int>(g.nz);
#pragma unroll
    for (int i = 0; i < d3::Q; ++i) {
        int sx = x - d3::cx(i), sy = y - d3::cy(i), sz = z - d3::cz(i);
        int dir = i;
        if (d3::cy(i) != 0 && (sy < 0 || sy >= ny)) {
            const bool periodic = (sy < 0 ? g.y_lo : g.y_hi) == ORR_WALL_PERIODIC;
            sy = periodic ? (sy < 0 ? ny - 1 : 0) : y;
            dir = periodic ? dir : d3::mirror_y(i);
        }
        if (d3::cz(i) != 0 && (sz < 0 || sz >= nz)) {
            const bool periodic = (sz < 0 ? g.z_lo : g.z_hi) == ORR_WALL_PERIODIC;
            sz = periodic ? (sz < 0 ? nz - 1 : 0) : z;
            // Mirror of the (possibly already mirrored) direction.
            const int mz = dir == i ? d3::mirror_z(i) : d3::mirror_z(d3::mirror_y(i));
            dir = periodic ? dir : mz;
        }
        bool unknown = false, xside = false;
        if (d3::cx(i) != 0 && (sx < 0 || sx >= nx)) {
            if (g.x_mode == ORR_X_PERIODIC) {
                sx = sx < 0 ? nx - 1 : 0;
            } else {
                // Inlet unknown (reconstructed by the inlet) or the
                // zero-gradient outlet copy; neither takes the solid test.
                xside = true;
                unknown = sx < 0;
                sx = sx < 0 ? 0 : nx - 1;
            }
        }
        uint64_t at = static_cast<uint64_t>(dir) * g.cells + static_cast<uint64_t>(sx) +
                      static_cast<uint64_t>(nx) * (static_cast<uint64_t>(sy) + static_cast<uint64_t>(ny) * sz);
        if (!xside && ((mask >> i) & 1u) != 0u) {
            at = static_cast<uint64_t>(d3::opposite(i)) * g.cells + here; // halfway: f*_opp(x)
        }
        f[i] = unknown ? A(0) : T::load(src + at);
    }
}

// Convective outlet at x = nx - 1 (outlet_value, lbm3d_cpu.cpp:239-250): the
// zero-gradient copies in f (c_x < 0) are blended with the node's history;
// nothing for the extrapolation outlet.
template <class S>
__device__ __forceinline__ void convective_blend3(const Geom3D& g, const Phys3D<typename Storage<S>::A>& p,
                                                  const StepBuffers3D& b, uint32_t y, uint32_t z,
                                                  typename Storage<S>::A (&f)[d3::Q]) {
    using A = typename Storage<S>::A;
    if (g.outlet_mode != ORR_OUTLET_CONVECTIVE) {
        return;
    }
    A* hist = static_cast<A*>(b.hist);
    const A u = p.outlet_speed;
    const uint64_t at = static_cast<uint64_t>(y) + static_cast<uint64_t>(g.ny) * z;
    const uint64_t face = static_cast<uint64_t>(g.ny) * g.nz;
#pragma unroll
    for (int i = 0; i < d3::Q; ++i) {
        if (d3::cx(i) < 0) {
            const uint64_t k = static_cast<uint64_t>(d3::outlet_slot(i)) * face + at;
            const A v = r_div(r_add(hist[k], r_mul(u, f[i])), r_add(A(1), u));
            hist[k] = v;
            f[i] = v;
        }
    }
}

// Fix-ups of a bulk node after its 19 plain pulls f_i = f*_i(x - c_i).  The
// x-edge lanes of an interior row (two per row) read their c_x != 0 sources
// again: x = -1 wraps to nx - 1 (periodic) or is an inlet unknown, rebuilt by
// the inlet; x = nx wraps to 0 or copies the outlet node x = nx - 1.  The
// first reads stayed inside the lattice (neighbouring rows) and are
// discarded.
template <class S>
__device__ __forceinline__ void bulk_edges3(const Geom3D& g, const Phys3D<typename Storage<S>::A>& p,
                                            const S* __restrict__ src, const StepBuffers3D& b,
                                            uint32_t x, uint32_t y, uint32_t z, uint64_t here,
                                            typename Storage<S>::A (&f)[d3::Q]) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    const uint64_t cells = g.cells;
    const int64_t nx = g.nx, plane = g.plane;
    const bool xlo = x == 0u, xhi = x + 1u == g.nx;
    if (xlo && g.x_mode == ORR_X_PERIODIC) {
#pragma unroll
        for (int i = 0; i < d3::Q; ++i) {
            if (d3::cx(i) > 0) {
                const int64_t source = static_cast<int64_t>(here) + nx -
                                       (d3::cx(i) + nx * d3::cy(i) + plane * d3::cz(i));
                f[i] = T::load(src + static_cast<uint64_t>(i) * cells + static_cast<uint64_t>(source));
            }
        }
    }
    if (xhi) {
        const int64_t shift = g.x_mode == ORR_X_PERIODIC ? -nx : -1;
#pragma unroll
        for (int i = 0; i < d3::Q; ++i) {
            if (d3::cx(i) < 0) {
                const int64_t source = static_cast<int64_t>(here) + shift -
                                       (d3::cx(i) + nx * d3::cy(i) + plane * d3::cz(i));
                f[i] = T::load(src + static_cast<uint64_t>(i) * cells + static_cast<uint64_t>(source));
            }
        }
    }
    if (xhi && g.x_mode == ORR_X_INFLOW_OUTFLOW) {
        convective_blend3<S>(g, p, b, y, z, f);
    }
}

// One fused step src -> dst: one thread per node, one block per tile of a
// row (blockDim.x nodes along x), every row of the lattice.  Every lane of a
// row stores all 19 populations of its node in the same step, so each
// 32-byte sector of the destination is written whole while it sits in L2:
// a sector written in parts at different times costs the DRAM a
// read-modify-write (ECC), about a fifth of the bandwidth.  Per lane:
//   solid       stores its rest populations, which the reference never changes
//               (initial_populations puts solids at rest; the step skips them);
//   bulk        interior rows (y in [1, ny-2], z in [1, nz-2]) with no solid
//               source: 19 plain pulls f_i(x) = f*_i(x - c_i)
//               (lbm3d_cpu.cpp:272-276); the x-edge lanes shift their x
//               sources (periodic wrap, outlet copy) and then take the
//               convective-outlet blend or the inlet reconstruction;
//   face        a node of a y or z face row without a solid source: the general
//               gather, whose side rules are uniform along the row;
//   boundary    a node with a solid source (bounce-back / interpolated wall):
//               the general gather with the plan's per-node direction mask.
// The rules of a fluid node of a flat lattice once its plain pulls are in f
// (for an interior row; elsewhere f is filled here): x-edge, wall and outlet
// rules and the inlet, everything before the collision.
template <class S>
__device__ __forceinline__ void flat_fix3(const Geom3D& g, const Phys3D<typename Storage<S>::A>& p,
                                          const S* __restrict__ src, const StepBuffers3D& b,
                                          typename Storage<S>::A (&f)[d3::Q], uint8_t cls, bool interior,
                                          uint32_t x, uint32_t y, uint32_t z, uint64_t here) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    const uint64_t cells = g.cells;
    if (cls == kBulk) {
        bulk_edges3<S>(g, p, src, b, x, y, z, here, f);
    } else if (interior && x != 0u && x + 1u != g.nx) {
        // Boundary node of an interior row: halfway bounce-back replaces
        // the pulls of its solid-source directions by f*_opp at the node.
        const uint32_t mask = b.nmask[here];
#pragma unroll
        for (int i = 0; i < d3::Q; ++i) {
            if ((mask >> i) & 1u) {
                f[i] = T::load(src + static_cast<uint64_t>(d3::opposite(i)) * cells + here);
            }
        }
    } else {
        const uint32_t mask = cls == kBoundary ? b.nmask[here] : 0u;
        gather_flat3<S>(g, src, mask, static_cast<int>(x), static_cast<int>(y), static_cast<int>(z), here, f);
        if (x + 1u == g.nx && g.x_mode == ORR_X_INFLOW_OUTFLOW) {
            convective_blend3<S>(g, p, b, y, z, f);
        }
    }
    if (g.x_mode == ORR_X_INFLOW_OUTFLOW && x == 0u) {
        inlet_west3<A, T::kShifted>(f, static_cast<const A*>(b.inlet));
    }
}

// The rest of a node's step on a flat lattice once its pulls are in f (for
// an interior row; elsewhere f is filled here): class, edge and wall rules,
// the inlet, the collision and the 19 stores.
template <class S, bool kSmag>
__device__ __forceinline__ void flat_finish3(const Geom3D& g, const Phys3D<typename Storage<S>::A>& p,
                                             const S* __restrict__ src, S* __restrict__ dst,
                                             const StepBuffers3D& b, typename Storage<S>::A (&f)[d3::Q],
                                             uint8_t cls, bool interior, uint32_t x, uint32_t y, uint32_t z,
                                             uint64_t here) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    if (cls == kSolid) {
#pragma unroll
        for (int i = 0; i < d3::Q; ++i) {
            T::store(dst + static_cast<uint64_t>(i) * g.cells + here, T::kShifted ? A(0) : A(d3::w(i)));
        }
        return;
    }
    flat_fix3<S>(g, p, src, b, f, cls, interior, x, y, z, here);
    finish3<S, kSmag>(g, p, b, f, x, y, z, here, dst);
}

// The 19 plain pulls of node `here` (valid addresses for interior rows).
template <class S>
__device__ __forceinline__ void pull3(const Geom3D& g, const S* __restrict__ src, uint64_t here,
                                      typename Storage<S>::A (&f)[d3::Q]) {
    using T = Storage<S>;
    const int64_t nx = g.nx, plane = g.plane, cells = static_cast<int64_t>(g.cells);
    const uint32_t h = static_cast<uint32_t>(here);
#pragma unroll
    for (int i = 0; i < d3::Q; ++i) {
        // (src + i * cells - c_i . (1, nx, plane)) is the same for every
        // thread; the node index is added last as a 32-bit value.
        const int64_t shift = i * cells - (d3::cx(i) + nx * d3::cy(i) + plane * d3::cz(i));
        f[i] = T::load(src + shift + h);
    }
}

template <class S, bool kSmag, bool kFlat>
__device__ __forceinline__ void step_node3(const Geom3D& g, const Phys3D<typename Storage<S>::A>& p,
                                           const S* __restrict__ src, S* __restrict__ dst,
                                           const StepBuffers3D& b, uint32_t x, uint32_t y,
                                           uint32_t z) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    const uint64_t cells = g.cells;
    const uint64_t here = x + g.nx * (y + g.ny * z);   // below 2^32 / 19
    A f[d3::Q];
    if constexpr (kFlat) {
        // Interior rows: every plain pull address lies inside the lattice, so
        // the 19 pulls are issued together with the class load (no dependent
        // round trip) and then used, overridden or dropped by class.
        const bool interior = (y - 1u < g.ny - 2u) && (z - 1u < g.nz - 2u);
        if (interior) {
            pull3<S>(g, src, here, f);
        }
        flat_finish3<S, kSmag>(g, p, src, dst, b, f, b.cls[here], interior, x, y, z, here);
        return;
    } else {
        const uint8_t cls = b.cls[here];
        if (cls == kSolid) {
#pragma unroll
            for (int i = 0; i < d3::Q; ++i) {
                T::store(dst + static_cast<uint64_t>(i) * cells + here, T::kShifted ? A(0) : A(d3::w(i)));
            }
            return;
        }
        if (cls == kBulk) {
            pull3<S>(g, src, here, f);
            bulk_edges3<S>(g, p, src, b, x, y, z, here, f);
        } else {
            const uint32_t mask = cls == kBoundary ? b.nmask[here] : 0u;
            const int32_t slot = b.nslot != nullptr ? b.nslot[here] : -1;
            A wall_rho = A(-1);
            gather_all3<S, 0, true>(g, p, src, b, slot, mask, static_cast<int>(x), static_cast<int>(y),
                                    static_cast<int>(z), here, wall_rho, f);
        }
    }
    if (g.x_mode == ORR_X_INFLOW_OUTFLOW && x == 0u) {
        inlet_west3<A, T::kShifted>(f, static_cast<const A*>(b.inlet));
    }
    finish3<S, kSmag>(g, p, b, f, x, y, z, here, dst);
}

// Resident 256-thread blocks per SM the row step is compiled for: 48
// registers for the binary32 flat step, 40 for the flat step of the 2-byte
// storages, 64 for the general one, 128 for binary64.  The flat step fits 48
// without spills, and the extra resident warps hide more of the memory
// latency: 45.5 against 42.8 GLUPS for binary16 storage in 128-thread blocks,
// 41.4 against 39.9 for binary32 in 256-thread blocks (256 x 128 x 128 sphere
// channel).  The 2-byte forms, which issue more instructions per byte moved,
// gain again from 48 warps at 40 registers despite a few spilled values
// (binary16 88.1 against 92.1 us per step, bfloat16 89.8 against 93.1);
// binary32 loses there (105.2 against 101.1 us), so it keeps 48 registers.
template <class S, bool kFlat>
constexpr int kStepMinBlocks = sizeof(typename Storage<S>::A) == 8 ? 2
                               : !kFlat                        ? 4
                               : sizeof(S) == 2                ? 6
                                                               : 5;

// Grid (tiles along x, ny, nz): block (t, y, z) covers x in [t B, (t + 1) B)
// of row (y, z).
// kFlat: the lattice has g.flat set (the independent-load gather; the
// general one otherwise).
template <class S, bool kSmag, bool kFlat>
__global__ void __launch_bounds__(256, kStepMinBlocks<S, kFlat>) step3d_kernel(Geom3D g, Phys3D<typename Storage<S>::A> p,
                                                        const S* __restrict__ src,
                                                        S* __restrict__ dst, StepBuffers3D b) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= g.nx) {
        return;
    }
    step_node3<S, kSmag, kFlat>(g, p, src, dst, b, x, blockIdx.y, blockIdx.z);
}

// Row tiles of neighbouring node pairs, for the 2-byte storage forms of a
// flat lattice with even nx: thread t of block (k, y, z) takes the nodes
// x0 = 2 (k B + t) and x0 + 1 of row (y, z).  In an interior row each
// direction is one aligned 32-bit load per lane: the two values of the pair
// for c_x = 0; for c_x != 0 the pair's row word, whose missing half is the
// neighbouring lane's word (a warp shuffle; the first and last lanes of the
// warp load the word beyond the warp themselves).  A warp so moves 128 bytes
// per load and per store instruction instead of 64.  Both nodes then take the
// per-node rules (x edges, walls, inlet) on their own values and collide
// together in packed binary32 lanes (collide3_pair).  Face rows go node by
// node through step_node3.  Every value is rounded as in step3d_kernel: the
// same bits.
constexpr int kPairMinBlocks = 5;

template <class S, bool kSmag>
__global__ void __launch_bounds__(128, kPairMinBlocks) step3d_pair_kernel(Geom3D g, Phys3D<float> p,
                                                                          const S* __restrict__ src,
                                                                          S* __restrict__ dst, StepBuffers3D b) {
    using T = Storage<S>;
    static_assert(sizeof(S) == 2, "pairs of 2-byte values");
    const uint32_t x0 = 2u * (blockIdx.x * blockDim.x + threadIdx.x);
    const uint32_t y = blockIdx.y, z = blockIdx.z;
    if (y - 1u >= g.ny - 2u || z - 1u >= g.nz - 2u) {
        if (x0 < g.nx) {
            step_node3<S, kSmag, true>(g, p, src, dst, b, x0, y, z);
            step_node3<S, kSmag, true>(g, p, src, dst, b, x0 + 1u, y, z);
        }
        return;
    }
    // Interior row (uniform over the block): every lane loads and shuffles;
    // lanes past the row end load the row's last pair.
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t xl = min(x0, g.nx - 2u);
    const uint32_t h = xl + g.nx * (y + g.ny * z);
    const uint64_t here = h;
    const int64_t nx = g.nx, plane = g.plane, cells = static_cast<int64_t>(g.cells);
    uint32_t word[d3::Q], edge[d3::Q];
#pragma unroll
    for (int i = 0; i < d3::Q; ++i) {
        const int64_t shift = i * cells - (nx * d3::cy(i) + plane * d3::cz(i));
        const auto* at = reinterpret_cast<const uint32_t*>(src + shift + h);
        word[i] = __ldg(at);
        edge[i] = 0u;
        if (d3::cx(i) > 0 && lane == 0u) {
            edge[i] = __ldg(at - 1);
        }
        if (d3::cx(i) < 0 && lane == 31u) {
            edge[i] = __ldg(at + 1);
        }
    }
    const uint32_t cls2 = __ldg(reinterpret_cast<const uint16_t*>(b.cls + here));
    float fa[d3::Q], fb[d3::Q];
#pragma unroll
    for (int i = 0; i < d3::Q; ++i) {
        if (d3::cx(i) == 0) {
            fa[i] = T::lo(word[i]);
            fb[i] = T::hi(word[i]);
        } else if (d3::cx(i) > 0) {
            // sources x0 - 1 (the left lane's upper half) and x0
            uint32_t left = __shfl_up_sync(0xffffffffu, word[i], 1);
            left = lane == 0u ? edge[i] : left;
            fa[i] = T::hi(left);
            fb[i] = T::lo(word[i]);
        } else {
            // sources x0 + 1 and x0 + 2 (the right lane's lower half)
            uint32_t right = __shfl_down_sync(0xffffffffu, word[i], 1);
            right = lane == 31u ? edge[i] : right;
            fa[i] = T::hi(word[i]);
            fb[i] = T::lo(right);
        }
    }
    if (x0 >= g.nx) {
        return;
    }
    const uint8_t ca = static_cast<uint8_t>(cls2 & 0xffu), cb = static_cast<uint8_t>(cls2 >> 8);
    if (ca != kSolid && (ca != kBulk || x0 == 0u)) {
        flat_fix3<S>(g, p, src, b, fa, ca, true, x0, y, z, here);
    }
    if (cb != kSolid && (cb != kBulk || x0 + 2u == g.nx)) {
        flat_fix3<S>(g, p, src, b, fb, cb, true, x0 + 1u, y, z, here + 1u);
    }
    float2 f[d3::Q];
#pragma unroll
    for (int i = 0; i < d3::Q; ++i) {
        f[i] = make_float2(fa[i], fb[i]);
    }
    collide3_pair<kSmag>(f, p, g.forced);
    if (g.sponge) {
        const float sa = sponge_rate3<float>(g, p, x0, y, z);
        const float sb = sponge_rate3<float>(g, p, x0 + 1u, y, z);
        if (sa > 0.0f || sb > 0.0f) {
            absorb3_pair(f, sa, sb, static_cast<const float*>(b.inlet));
        }
    }
#pragma unroll
    for (int i = 0; i < d3::Q; ++i) {
        // solid nodes store 0 (f - w of the rest state)
        const float va = ca == kSolid ? 0.0f : f[i].x;
        const float vb = cb == kSolid ? 0.0f : f[i].y;
        *reinterpret_cast<uint32_t*>(dst + static_cast<uint64_t>(i) * g.cells + h) = T::pack(va, vb);
    }
}

// ------------------------------------------------------------ init / misc --

// Equilibrium of (rho, u) at every node, solids at rest (initial_populations,
// lbm3d_common.cpp:243-260); binary32 forms store f - w like the reference GPU
// driver (lbm3d_gpu.cpp:298-305).  The field arrays may live in the other
// population buffer (the solver stages them there), so they are read before
// the node's own entries are written and never alias them.
template <class S>
__global__ void init3d_kernel(Geom3D g, const uint8_t* __restrict__ cls, const double* rho,
                              const double* ux, const double* uy, const double* uz, double r0,
                              double u0x, double u0y, double u0z, S* __restrict__ f0) {
    using T = Storage<S>;
    const uint64_t c = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= g.cells) {
        return;
    }
    double r = 1.0, vx = 0.0, vy = 0.0, vz = 0.0;
    if (cls[c] != kSolid) {
        if (rho != nullptr) {
            r = rho[c];
            vx = ux[c];
            vy = uy[c];
            vz = uz[c];
        } else {
            r = r0;
            vx = u0x;
            vy = u0y;
            vz = u0z;
        }
    }
#pragma unroll
    for (int i = 0; i < d3::Q; ++i) {
        const double cu = static_cast<double>(d3::cx(i)) * vx + static_cast<double>(d3::cy(i)) * vy +
                          static_cast<double>(d3::cz(i)) * vz;
        const double uu = vx * vx + vy * vy + vz * vz;
        double feq = d3::w(i) * r * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * uu);
        if (T::kShifted) {
            feq -= d3::w(i);
        }
        f0[static_cast<uint64_t>(i) * g.cells + c] = T::encode(feq);
    }
}

// Convective-outlet history from the populations entering the outlet face
// (reset_outlet, lbm3d_cpu.cpp:225-237; lbm3d_gpu.cpp:311-323).
template <class S>
__global__ void history3d_kernel(Geom3D g, const S* __restrict__ f,
                                 typename Storage<S>::A* __restrict__ hist) {
    using T = Storage<S>;
    const uint32_t face = g.ny * g.nz;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= face) {
        return;
    }
    const uint32_t y = k % g.ny, z = k / g.ny;
    const uint64_t cell = (g.nx - 1u) + static_cast<uint64_t>(g.nx) * (y + static_cast<uint64_t>(g.ny) * z);
    constexpr int dirs[5] = {2, 8, 10, 12, 14};
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        hist[static_cast<uint64_t>(d3::outlet_slot(dirs[s])) * face + y + static_cast<uint64_t>(g.ny) * z] =
            T::load(f + static_cast<uint64_t>(dirs[s]) * g.cells + cell);
    }
}

// Moments of the stored post-collision populations: rho (rho - 1 for the
// shifted forms) and the velocity with the Guo half-force correction; solids
// report rest (lbm_d3q19_moments.comp.glsl; CpuLbm3D::macroscopic,
// lbm3d_cpu.cpp:154-186).
template <class S>
__global__ void moments3d_kernel(Geom3D g, Phys3D<typename Storage<S>::A> p,
                                 const uint8_t* __restrict__ cls, const S* __restrict__ f,
                                 typename Storage<S>::A* __restrict__ m) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    const uint64_t c = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= g.cells) {
        return;
    }
    A r = T::kShifted ? A(0) : A(1), ux = 0, uy = 0, uz = 0;
    if (cls[c] != kSolid) {
        A v[d3::Q];
#pragma unroll
        for (int i = 0; i < d3::Q; ++i) v[i] = T::load(f + static_cast<uint64_t>(i) * g.cells + c);
        A s = 0;
#pragma unroll
        for (int i = 0; i < d3::Q; ++i) s += v[i];
        const A jx = v[1] - v[2] + v[7] - v[8] + v[9] - v[10] + v[11] - v[12] + v[13] - v[14];
        const A jy = v[3] - v[4] + v[7] - v[8] - v[9] + v[10] + v[15] - v[16] + v[17] - v[18];
        const A jz = v[5] - v[6] + v[11] - v[12] - v[13] + v[14] + v[15] - v[16] - v[17] + v[18];
        const A rho = T::kShifted ? A(1) + s : s;
        r = s;
        ux = (jx - A(0.5) * p.fx) / rho;
        uy = (jy - A(0.5) * p.fy) / rho;
        uz = (jz - A(0.5) * p.fz) / rho;
    }
    m[c] = r;
    m[g.cells + c] = ux;
    m[2 * g.cells + c] = uy;
    m[3 * g.cells + c] = uz;
}

// Block-wide sum of N doubles per thread, then one atomicAdd per value per
// block into `out`.
template <int N>
__device__ __forceinline__ void block_reduce_add(double (&v)[N], double* out) {
    __shared__ double part[N][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int warps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < N; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) part[k][warp] = v[k];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            double s = lane < warps ? part[k][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) atomicAdd(out + k, s);
        }
    }
}

// One boundary link's momentum exchange c_o (f*_o(x) + f_j(x, t+1)) and its
// moment about the origin at the wall point x - q c_j, added to acc
// (CpuLbm3D::force, lbm3d_cpu.cpp:192-203; add_link_force and link_wall_point,
// lbm3d_common.cpp:213-241; lbm_d3q19_force.comp.glsl).  The one per-link
// routine of every force kernel (the solver's, the batched and the
// allocation-free one): the population arithmetic rounds explicitly in the
// storage's arithmetic type and the binary64 sums use unfused intrinsics, so
// no unit contracts them differently and every kernel sums the same terms.
// kChecked: the link comes from a caller's table, so a cell beyond the
// lattice, a direction outside 1..18 or an interpolation source outside the
// lattice skips the link and returns false (the plan's own links are in
// range by construction).
// Unfused binary64 forms of r_mul / r_sub / r_fma for the link arithmetic
// (the binary32 ones already round explicitly); the same bits in every unit,
// with or without FMA contraction.
__device__ __forceinline__ float lk_mul(float a, float b) { return r_mul(a, b); }
__device__ __forceinline__ float lk_sub(float a, float b) { return r_sub(a, b); }
__device__ __forceinline__ float lk_fma(float a, float b, float c) { return r_fma(a, b, c); }
__device__ __forceinline__ double lk_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double lk_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double lk_fma(double a, double b, double c) { return __dadd_rn(__dmul_rn(a, b), c); }

template <class S, bool kChecked = false>
__device__ __forceinline__ bool add_link3(uint64_t nx, uint64_t plane, uint64_t cells,
                                          const S* __restrict__ f, uint64_t h, int j, double q,
                                          double (&acc)[6]) {
    using A = typename Storage<S>::A;
    using T = Storage<S>;
    if constexpr (kChecked) {
        if (h >= cells || j < 1 || j >= d3::Q || !(q >= 0.0 && q <= 1.0)) {
            return false;
        }
    }
    const int o = opposite_rt(j);
    int jx, jy, jz;
    c_rt(j, jx, jy, jz);
    const A qa = static_cast<A>(q);
    const A leaving = T::load(f + static_cast<uint64_t>(o) * cells + h);
    A back;
    if (q == 0.5) {
        back = leaving;
    } else if (q < 0.5) {
        const int64_t farther = static_cast<int64_t>(h) + jx + static_cast<int64_t>(nx) * jy +
                                static_cast<int64_t>(plane) * jz;
        if constexpr (kChecked) {
            if (farther < 0 || static_cast<uint64_t>(farther) >= cells) {
                return false;
            }
        }
        const A t = lk_mul(A(2), qa);
        back = lk_fma(t, leaving,
                      lk_mul(lk_sub(A(1), t),
                             T::load(f + static_cast<uint64_t>(o) * cells + static_cast<uint64_t>(farther))));
    } else {
        const A t = lk_mul(A(2), qa);
        back = r_div(lk_fma(lk_sub(t, A(1)), T::load(f + static_cast<uint64_t>(j) * cells + h), leaving), t);
    }
    double ex = __dadd_rn(static_cast<double>(leaving), static_cast<double>(back));
    if (T::kShifted) {
        ex = __dadd_rn(ex, __dmul_rn(2.0, w_rt(o)));
    }
    // c_o = -c_j
    const double fx = -jx * ex, fy = -jy * ex, fz = -jz * ex;
    const uint64_t z = h / plane, rest = h - z * plane;
    const uint64_t y = rest / nx, x = rest - y * nx;
    const double rx = __dsub_rn(static_cast<double>(x), __dmul_rn(q, jx));
    const double ry = __dsub_rn(static_cast<double>(y), __dmul_rn(q, jy));
    const double rz = __dsub_rn(static_cast<double>(z), __dmul_rn(q, jz));
    acc[0] = __dadd_rn(acc[0], fx);
    acc[1] = __dadd_rn(acc[1], fy);
    acc[2] = __dadd_rn(acc[2], fz);
    acc[3] = __dadd_rn(acc[3], __dsub_rn(__dmul_rn(ry, fz), __dmul_rn(rz, fy)));
    acc[4] = __dadd_rn(acc[4], __dsub_rn(__dmul_rn(rz, fx), __dmul_rn(rx, fz)));
    acc[5] = __dadd_rn(acc[5], __dsub_rn(__dmul_rn(rx, fy), __dmul_rn(ry, fx)));
    return true;
}

// Momentum exchange over the boundary links, summed in binary64 (one thread
// per link, add_link3; warp shuffles, a block reduction and one atomic per
// value and block).
template <class S>
__global__ void force3d_kernel(Geom3D g, const S* __restrict__ f, const uint32_t* __restrict__ lcell,
                               const uint32_t* __restrict__ ldir, const double* __restrict__ lq,
                               uint64_t links, double* __restrict__ out) {
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (uint64_t k = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < links;
         k += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        add_link3<S>(g.nx, g.plane, g.cells, f, lcell[k], static_cast<int>(ldir[k]), lq[k], acc);
    }
    block_reduce_add<6>(acc, out);
}

// ------------------------------------------------------ batched forces --

// The links of one lattice for the batched force (device table entry).
struct ForceJob {
    const void* f;            // populations the force reads (the current buffer)
    const uint32_t* lcell;
    const uint32_t* ldir;
    const double* lq;
    uint64_t links;
    uint64_t chunk_begin;     // first global chunk of this lattice
    uint64_t nx, plane, cells;
};

constexpr uint32_t kForceThreads = 256;
constexpr uint64_t kForceChunk = 2048; // links per block of pass 1

// Sum of six doubles over the block in a fixed order; valid in thread 0.
__device__ __forceinline__ void block_sum6_fixed(double (&v)[6]) {
    __shared__ double part[6][kForceThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) part[k][warp] = v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            double t = 0.0;
            for (int w = 0; w < static_cast<int>(kForceThreads / 32); ++w) t += part[k][w];
            v[k] = t;
        }
    }
}

// Pass 1 of the batched force: block b sums global chunk b (kForceChunk
// links of one lattice) into partial[6 b .. 6 b + 5].
template <class S>
__global__ void __launch_bounds__(kForceThreads) force_batch_partials(const ForceJob* __restrict__ jobs,
                                                                      uint32_t n, double* __restrict__ partial) {
    const uint64_t chunk = blockIdx.x;
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (jobs[mid].chunk_begin <= chunk) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    const ForceJob& J = jobs[lo];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const uint64_t begin = (chunk - J.chunk_begin) * kForceChunk;
    const uint64_t end = begin + kForceChunk < J.links ? begin + kForceChunk : J.links;
    const S* f = static_cast<const S*>(J.f);
    for (uint64_t k = begin + threadIdx.x; k < end; k += kForceThreads) {
        add_link3<S>(J.nx, J.plane, J.cells, f, J.lcell[k], static_cast<int>(J.ldir[k]), J.lq[k], acc);
    }
    block_sum6_fixed(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int v = 0; v < 6; ++v) partial[chunk * 6 + v] = acc[v];
    }
}

// Pass 2: lattice blockIdx.x adds its chunks' partial sums in chunk order
// and adds (accumulate) or writes the six totals to out[6 l ..].
// (A template, instantiated per storage unit like the other kernels.)
template <class S>
__global__ void __launch_bounds__(kForceThreads) force_batch_totals(const ForceJob* __restrict__ jobs,
                                                                    const double* __restrict__ partial,
                                                                    double* __restrict__ out, int accumulate) {
    const ForceJob& J = jobs[blockIdx.x];
    const uint64_t chunks = (J.links + kForceChunk - 1) / kForceChunk;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (uint64_t c = threadIdx.x; c < chunks; c += kForceThreads) {
#pragma unroll
        for (int v = 0; v < 6; ++v) acc[v] += partial[(J.chunk_begin + c) * 6 + v];
    }
    block_sum6_fixed(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int v = 0; v < 6; ++v) {
            out[blockIdx.x * 6 + v] = accumulate ? out[blockIdx.x * 6 + v] + acc[v] : acc[v];
        }
    }
}

// Sum of the stored populations over fluid nodes in binary64 (the shifted
// forms add the node count on the host; CpuLbm3D::mass, lbm3d_cpu.cpp:205-215).
template <class S>
__global__ void mass3d_kernel(Geom3D g, const uint8_t* __restrict__ cls, const S* __restrict__ f,
                              double* __restrict__ out) {
    using T = Storage<S>;
    double acc[1] = {0.0};
    for (uint64_t c = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < g.cells;
         c += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (cls[c] != kSolid) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < d3::Q; ++i) s += static_cast<double>(T::load(f + static_cast<uint64_t>(i) * g.cells + c));
            acc[0] += s;
        }
    }
    block_reduce_add<1>(acc, out);
}

} // namespace orr
