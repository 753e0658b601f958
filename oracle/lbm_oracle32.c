/* Binary32 restatement of the reference's GPU step.  TEST INFRASTRUCTURE
 * ONLY: imported by tests/ and fixture scripts, never by the product.
 *
 * The reference runs its GPU solver as GLSL compute kernels that keep the
 * populations in binary32, shifted by their weights (f - w), and do every
 * operation in binary32 (src/render/shaders/lbm/lbm_d3q19_common.glsl:67-368,
 * lbm_d3q19_step.comp.glsl, lbm_d3q19_force.comp.glsl; driven by
 * src/aero/lbm3d/lbm3d_gpu.cpp).  That path cannot run here (no graphics
 * stack), so this file restates its arithmetic in C, statement for
 * statement, in binary32 with no contraction (built with
 * -ffp-contract=off; a GLSL compiler may fuse some multiply-adds, and its
 * division and square root may round differently, so this is one binary32
 * evaluation of the reference's GPU step, not its bits).  Its use: a
 * binary32 solver independent of the CUDA kernels, to tell binary32 rounding
 * from a kernel difference when the CUDA binary32 form is compared with the
 * binary64 reference.
 *
 * Every fluid node takes the general gather (lbm3_gather's boundary branch;
 * for a node whose sources are all in-range fluid nodes it performs the
 * plain pulls of the bulk branch, with the same arithmetic), so no node
 * classification is needed.  Initial state, outlet history and force follow
 * the driver: populations from the binary64 equilibrium minus the weight,
 * rounded once to binary32 (GpuLbm3D::initialize, lbm3d_gpu.cpp:298-331); the
 * force as the binary32 per-link sums of lbm_d3q19_force.comp.glsl, with the
 * weights added back and summed in binary64 (GpuLbm3D::force, :407-436;
 * add_link_force, lbm3d_common.cpp:213-241). */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "orrery_lbm.h"

#define Q 19

static const int CX[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const int CY[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
static const int CZ[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
static const int OPP[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
static const int MIRROR_Y[Q] = {0, 1, 2, 4, 3, 5, 6, 9, 10, 7, 8, 11, 12, 13, 14, 18, 17, 16, 15};
static const int MIRROR_Z[Q] = {0, 1, 2, 3, 4, 6, 5, 7, 8, 9, 10, 13, 14, 11, 12, 17, 18, 15, 16};
static const double WD[Q] = {1.0 / 3.0,  1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0,
                             1.0 / 18.0, 1.0 / 18.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                             1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                             1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};

typedef struct lo32 {
    int nx, ny, nz;
    size_t cells;
    /* the driver's uniforms, rounded once to binary32 */
    unsigned x_mode, outlet_mode, kind[4]; /* y low, y high, z low, z high: 0 periodic, 1 slip, 2 wall */
    float wall_ux[4], inlet[3], tau, c2, force[3], outlet_speed, sponge_strength;
    unsigned sponge_inlet, sponge_outlet, sponge_sides;
    float w[Q];
    uint8_t* solid;
    float* q;           /* 19 per cell wall fractions, or NULL (halfway everywhere) */
    float* f[2];
    float* history;     /* 5 * ny * nz */
    int cur;
    uint64_t steps;
} lo32;

static size_t idx(const lo32* s, int x, int y, int z) {
    return (size_t)x + (size_t)s->nx * ((size_t)y + (size_t)s->ny * (size_t)z);
}

static unsigned wall_code(int32_t kind) {
    return kind == ORR_WALL_PERIODIC ? 0u : (kind == ORR_WALL_SLIP ? 1u : 2u);
}

static unsigned outlet_slot(int i) {
    return i == 2 ? 0u : (i == 8 ? 1u : (i == 10 ? 2u : (i == 12 ? 3u : 4u)));
}

/* lbm3_side: true for a no-slip wall; s and the direction updated for the
 * periodic and free-slip rules. */
static int side(unsigned low, unsigned high, int* s, int n, int own, int* dir, int y_axis) {
    if (*s >= 0 && *s < n) {
        return 0;
    }
    const unsigned kind = *s < 0 ? low : high;
    if (kind == 0u) {
        *s = (*s + n) % n;
        return 0;
    }
    if (kind == 1u) {
        *s = own;
        *dir = y_axis ? MIRROR_Y[*dir] : MIRROR_Z[*dir];
        return 0;
    }
    return 1;
}

/* lbm3_reflected */
static float reflected(const lo32* s, const float* src, int i, size_t here, int x, int y, int z, float q) {
    const int o = OPP[i];
    const float leaving = src[(size_t)o * s->cells + here];
    if (q == 0.5f) {
        return leaving;
    }
    if (q < 0.5f) {
        const size_t farther = idx(s, x + CX[i], y + CY[i], z + CZ[i]);
        return 2.0f * q * leaving + (1.0f - 2.0f * q) * src[(size_t)o * s->cells + farther];
    }
    return (leaving + (2.0f * q - 1.0f) * src[(size_t)i * s->cells + here]) / (2.0f * q);
}

static float wall_fraction(const lo32* s, size_t here, int i) {
    return s->q != NULL ? s->q[here * Q + (size_t)i] : 0.5f;
}

/* lbm3_inlet_west */
static void inlet_west(const lo32* s, float f[Q]) {
    const float ux = s->inlet[0], uy = s->inlet[1], uz = s->inlet[2];
    float sum = 0.0f;
    for (int i = 0; i < Q; ++i) {
        if (CX[i] == 0) {
            sum += f[i];
        } else if (CX[i] < 0) {
            sum += 2.0f * f[i];
        }
    }
    const float drho = (sum + ux) / (1.0f - ux);
    const float rho = 1.0f + drho;
    for (int i = 0; i < Q; ++i) {
        if (CX[i] > 0) {
            const float cu = (float)CX[i] * ux + (float)CY[i] * uy + (float)CZ[i] * uz;
            f[i] = f[OPP[i]] + 6.0f * s->w[i] * rho * cu;
        }
    }
    const float uu = ux * ux + uy * uy + uz * uz;
    float feq[Q];
    float pxx = 0.0f, pyy = 0.0f, pzz = 0.0f, pxy = 0.0f, pxz = 0.0f, pyz = 0.0f;
    for (int i = 0; i < Q; ++i) {
        const float ex = (float)CX[i], ey = (float)CY[i], ez = (float)CZ[i];
        const float cu = ex * ux + ey * uy + ez * uz;
        feq[i] = s->w[i] * (drho + rho * (3.0f * cu + 4.5f * cu * cu - 1.5f * uu));
        const float neq = f[i] - feq[i];
        pxx += ex * ex * neq;
        pyy += ey * ey * neq;
        pzz += ez * ez * neq;
        pxy += ex * ey * neq;
        pxz += ex * ez * neq;
        pyz += ey * ez * neq;
    }
    for (int i = 0; i < Q; ++i) {
        const float ex = (float)CX[i], ey = (float)CY[i], ez = (float)CZ[i];
        f[i] = feq[i] + 4.5f * s->w[i] *
                            ((ex * ex - 1.0f / 3.0f) * pxx + (ey * ey - 1.0f / 3.0f) * pyy +
                             (ez * ez - 1.0f / 3.0f) * pzz + 2.0f * (ex * ey * pxy + ex * ez * pxz + ey * ez * pyz));
    }
}

/* lbm3_gather (every fluid node on the general branch) */
static void gather(lo32* s, const float* src, int x, int y, int z, float f[Q]) {
    const size_t here = idx(s, x, y, z);
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    float wall_rho = -1.0f;
    for (int i = 0; i < Q; ++i) {
        int sx = x - CX[i], sy = y - CY[i], sz = z - CZ[i];
        int dir = i;
        int wall = 0;
        float wall_ux = 0.0f;
        if (side(s->kind[0], s->kind[1], &sy, ny, y, &dir, 1)) {
            wall = 1;
            wall_ux = sy < 0 ? s->wall_ux[0] : s->wall_ux[1];
        } else if (side(s->kind[2], s->kind[3], &sz, nz, z, &dir, 0)) {
            wall = 1;
            wall_ux = sz < 0 ? s->wall_ux[2] : s->wall_ux[3];
        }
        if (wall) {
            if (wall_rho < 0.0f) {
                float drho = 0.0f;
                for (int k = 0; k < Q; ++k) {
                    drho += src[(size_t)k * s->cells + here];
                }
                wall_rho = 1.0f + drho;
            }
            f[i] = src[(size_t)OPP[i] * s->cells + here] + 6.0f * s->w[i] * wall_rho * (float)CX[i] * wall_ux;
            continue;
        }
        if (sx < 0 || sx >= nx) {
            if (s->x_mode == 0u) {
                sx = (sx + nx) % nx;
            } else if (sx < 0) {
                f[i] = 0.0f; /* reconstructed by the inlet */
                continue;
            } else {
                float upstream = src[(size_t)dir * s->cells + idx(s, nx - 1, sy, sz)];
                if (s->outlet_mode == 0u) {
                    const size_t slot = (size_t)outlet_slot(i) * (size_t)ny * (size_t)nz + (size_t)y +
                                        (size_t)ny * (size_t)z;
                    upstream = (s->history[slot] + s->outlet_speed * upstream) / (1.0f + s->outlet_speed);
                    s->history[slot] = upstream;
                }
                f[i] = upstream;
                continue;
            }
        }
        const size_t source = idx(s, sx, sy, sz);
        f[i] = s->solid[source] ? reflected(s, src, i, here, x, y, z, wall_fraction(s, here, i))
                                : src[(size_t)dir * s->cells + source];
    }
    if (s->x_mode == 1u && x == 0) {
        inlet_west(s, f);
    }
}

/* lbm3_collide */
static void collide(const lo32* s, float f[Q]) {
    float drho = 0.0f, jx = 0.0f, jy = 0.0f, jz = 0.0f;
    for (int i = 0; i < Q; ++i) {
        drho += f[i];
        jx += (float)CX[i] * f[i];
        jy += (float)CY[i] * f[i];
        jz += (float)CZ[i] * f[i];
    }
    const float rho = 1.0f + drho;
    const float ux = (jx + 0.5f * s->force[0]) / rho;
    const float uy = (jy + 0.5f * s->force[1]) / rho;
    const float uz = (jz + 0.5f * s->force[2]) / rho;
    const float uu = ux * ux + uy * uy + uz * uz;
    float feq[Q];
    for (int i = 0; i < Q; ++i) {
        const float cu = (float)CX[i] * ux + (float)CY[i] * uy + (float)CZ[i] * uz;
        feq[i] = s->w[i] * (drho + rho * (3.0f * cu + 4.5f * cu * cu - 1.5f * uu));
    }
    float tau = s->tau;
    if (s->c2 > 0.0f) {
        float pxx = 0.0f, pyy = 0.0f, pzz = 0.0f, pxy = 0.0f, pxz = 0.0f, pyz = 0.0f;
        for (int i = 0; i < Q; ++i) {
            const float ex = (float)CX[i], ey = (float)CY[i], ez = (float)CZ[i];
            const float neq = f[i] - feq[i];
            pxx += ex * ex * neq;
            pyy += ey * ey * neq;
            pzz += ez * ez * neq;
            pxy += ex * ey * neq;
            pxz += ex * ez * neq;
            pyz += ey * ez * neq;
        }
        const float strain = sqrtf(pxx * pxx + pyy * pyy + pzz * pzz + 2.0f * (pxy * pxy + pxz * pxz + pyz * pyz));
        tau = 0.5f * (tau + sqrtf(tau * tau + 25.455844122715710f * s->c2 * strain / rho));
    }
    const float omega = 1.0f / tau;
    const float scale = 1.0f - 0.5f * omega;
    const int forced = s->force[0] != 0.0f || s->force[1] != 0.0f || s->force[2] != 0.0f;
    for (int i = 0; i < Q; ++i) {
        float value = f[i] - omega * (f[i] - feq[i]);
        if (forced) {
            const float ex = (float)CX[i], ey = (float)CY[i], ez = (float)CZ[i];
            const float cu = ex * ux + ey * uy + ez * uz;
            value += scale * s->w[i] *
                     (3.0f * ((ex - ux) * s->force[0] + (ey - uy) * s->force[1] + (ez - uz) * s->force[2]) +
                      9.0f * cu * (ex * s->force[0] + ey * s->force[1] + ez * s->force[2]));
        }
        f[i] = value;
    }
}

static float sponge_layer(unsigned distance, unsigned thickness) {
    if (distance < thickness) {
        const float r = (float)(thickness - distance) / (float)thickness;
        return r * r;
    }
    return 0.0f;
}

/* lbm3_sponge */
static float sponge(const lo32* s, unsigned x, unsigned y, unsigned z) {
    if (!(s->sponge_strength > 0.0f) || s->x_mode != 1u) {
        return 0.0f;
    }
    float best = fmaxf(sponge_layer(x, s->sponge_inlet), sponge_layer((unsigned)s->nx - 1u - x, s->sponge_outlet));
    if (s->kind[0] != 0u) {
        best = fmaxf(best, fmaxf(sponge_layer(y, s->sponge_sides), sponge_layer((unsigned)s->ny - 1u - y, s->sponge_sides)));
    }
    if (s->kind[2] != 0u) {
        best = fmaxf(best, fmaxf(sponge_layer(z, s->sponge_sides), sponge_layer((unsigned)s->nz - 1u - z, s->sponge_sides)));
    }
    return s->sponge_strength * best;
}

/* lbm3_absorb */
static void absorb(const lo32* s, float f[Q], float rate) {
    const float ux = s->inlet[0], uy = s->inlet[1], uz = s->inlet[2];
    const float uu = ux * ux + uy * uy + uz * uz;
    for (int i = 0; i < Q; ++i) {
        const float cu = (float)CX[i] * ux + (float)CY[i] * uy + (float)CZ[i] * uz;
        const float target = s->w[i] * (3.0f * cu + 4.5f * cu * cu - 1.5f * uu);
        f[i] -= rate * (f[i] - target);
    }
}

/* ---- entry points ---- */

lo32* lo32_create(const orr_lbm3d_config* c, const uint8_t* solid, const float* wall_q) {
    lo32* s = (lo32*)calloc(1, sizeof(lo32));
    if (s == NULL) {
        return NULL;
    }
    s->nx = (int)c->nx;
    s->ny = (int)c->ny;
    s->nz = (int)c->nz;
    s->cells = (size_t)c->nx * c->ny * c->nz;
    s->x_mode = c->x_boundary == ORR_X_INFLOW_OUTFLOW ? 1u : 0u;
    s->outlet_mode = c->outlet == ORR_OUTLET_EXTRAPOLATION ? 1u : 0u;
    const orr_wall* walls[4] = {&c->y_low, &c->y_high, &c->z_low, &c->z_high};
    for (int k = 0; k < 4; ++k) {
        s->kind[k] = wall_code(walls[k]->kind);
        s->wall_ux[k] = (float)walls[k]->velocity_x;
    }
    s->inlet[0] = (float)c->inlet_ux;
    s->inlet[1] = (float)c->inlet_uy;
    s->inlet[2] = (float)c->inlet_uz;
    s->tau = (float)c->tau;
    const double k = c->smagorinsky_enabled ? c->smagorinsky_constant : 0.0;
    s->c2 = (float)(k * k);
    s->force[0] = (float)c->body_force_x;
    s->force[1] = (float)c->body_force_y;
    s->force[2] = (float)c->body_force_z;
    s->outlet_speed = (float)c->inlet_ux;
    s->sponge_strength = (float)c->sponge_strength;
    s->sponge_inlet = (unsigned)c->sponge_inlet;
    s->sponge_outlet = (unsigned)c->sponge_outlet;
    s->sponge_sides = (unsigned)c->sponge_sides;
    for (int i = 0; i < Q; ++i) {
        s->w[i] = i == 0 ? 1.0f / 3.0f : (i < 7 ? 1.0f / 18.0f : 1.0f / 36.0f);
    }
    s->solid = (uint8_t*)malloc(s->cells);
    s->f[0] = (float*)malloc(Q * s->cells * sizeof(float));
    s->f[1] = (float*)malloc(Q * s->cells * sizeof(float));
    s->history = (float*)calloc(5 * (size_t)s->ny * (size_t)s->nz, sizeof(float));
    if (wall_q != NULL) {
        s->q = (float*)malloc(Q * s->cells * sizeof(float));
        if (s->q) memcpy(s->q, wall_q, Q * s->cells * sizeof(float));
    }
    if (!s->solid || !s->f[0] || !s->f[1] || !s->history || (wall_q && !s->q)) {
        free(s->solid);
        free(s->f[0]);
        free(s->f[1]);
        free(s->history);
        free(s->q);
        free(s);
        return NULL;
    }
    memcpy(s->solid, solid, s->cells);
    return s;
}

void lo32_destroy(lo32* s) {
    if (s == NULL) {
        return;
    }
    free(s->solid);
    free(s->f[0]);
    free(s->f[1]);
    free(s->history);
    free(s->q);
    free(s);
}

/* GpuLbm3D::initialize: the binary64 equilibrium of (rho, u) at every fluid
 * node, rest at solid nodes (initial_populations, lbm3d_common.cpp:243-270),
 * minus the weight, rounded once; the outlet history from the same values;
 * the inlet velocity back to the configuration's. */
void lo32_initialize(lo32* s, const double* rho, const double* ux, const double* uy, const double* uz,
                     const double inlet[3]) {
    for (size_t c = 0; c < s->cells; ++c) {
        const int fluid = !s->solid[c];
        const double r = fluid ? rho[c] : 1.0;
        const double u[3] = {fluid ? ux[c] : 0.0, fluid ? uy[c] : 0.0, fluid ? uz[c] : 0.0};
        const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        for (int i = 0; i < Q; ++i) {
            const double cu = CX[i] * u[0] + CY[i] * u[1] + CZ[i] * u[2];
            const double feq = WD[i] * r * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * uu);
            const float v = (float)(feq - WD[i]);
            s->f[0][(size_t)i * s->cells + c] = v;
            s->f[1][(size_t)i * s->cells + c] = v;
        }
    }
    const size_t face = (size_t)s->ny * (size_t)s->nz;
    static const int outlet_dirs[5] = {2, 8, 10, 12, 14};
    for (int z = 0; z < s->nz; ++z) {
        for (int y = 0; y < s->ny; ++y) {
            const size_t c = idx(s, s->nx - 1, y, z);
            for (int k = 0; k < 5; ++k) {
                s->history[(size_t)k * face + (size_t)y + (size_t)s->ny * (size_t)z] =
                    s->f[0][(size_t)outlet_dirs[k] * s->cells + c];
            }
        }
    }
    for (int k = 0; k < 3; ++k) {
        s->inlet[k] = (float)inlet[k];
    }
    s->cur = 0;
    s->steps = 0;
}

void lo32_set_inlet(lo32* s, const double inlet[3]) {
    for (int k = 0; k < 3; ++k) {
        s->inlet[k] = (float)inlet[k];
    }
}

/* lbm_d3q19_step.comp.glsl: gather, collide, absorbing layers, store; solid
 * nodes untouched.  z-planes in parallel (each node writes only its own
 * values and its own history entries). */
void lo32_step(lo32* s, uint64_t count) {
    for (uint64_t n = 0; n < count; ++n) {
        const float* src = s->f[s->cur];
        float* dst = s->f[1 - s->cur];
#pragma omp parallel for schedule(static)
        for (int z = 0; z < s->nz; ++z) {
            float f[Q];
            for (int y = 0; y < s->ny; ++y) {
                for (int x = 0; x < s->nx; ++x) {
                    const size_t here = idx(s, x, y, z);
                    if (s->solid[here]) {
                        continue;
                    }
                    gather(s, src, x, y, z, f);
                    collide(s, f);
                    const float rate = sponge(s, (unsigned)x, (unsigned)y, (unsigned)z);
                    if (rate > 0.0f) {
                        absorb(s, f, rate);
                    }
                    for (int i = 0; i < Q; ++i) {
                        dst[(size_t)i * s->cells + here] = f[i];
                    }
                }
            }
        }
        s->cur = 1 - s->cur;
        ++s->steps;
    }
}

/* Unshifted populations (the driver's read-back adds w in binary64). */
void lo32_populations(const lo32* s, double* out) {
    const float* f = s->f[s->cur];
    for (int i = 0; i < Q; ++i) {
        for (size_t c = 0; c < s->cells; ++c) {
            out[(size_t)i * s->cells + c] = (double)f[(size_t)i * s->cells + c] + WD[i];
        }
    }
}

/* GpuLbm3D::force: per link the binary32 sum f*_o + reflected f_j of the
 * force kernel, the weights added back and the force and moment (about the
 * origin, at the wall point x - q c_j) summed in binary64 in link order
 * (add_link_force, lbm3d_common.cpp:213-241). */
void lo32_force(const lo32* s, const uint32_t* cell, const uint32_t* dir, const double* q, uint64_t links,
                double out[6]) {
    const float* src = s->f[s->cur];
    double fx = 0.0, fy = 0.0, fz = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
    for (uint64_t k = 0; k < links; ++k) {
        const size_t here = cell[k];
        const int j = (int)dir[k];
        const int o = OPP[j];
        const size_t plane = (size_t)s->nx * (size_t)s->ny;
        const int z = (int)(here / plane), y = (int)((here % plane) / (size_t)s->nx), x = (int)(here % (size_t)s->nx);
        const float back = reflected(s, src, j, here, x, y, z, wall_fraction(s, here, j));
        const float link_force = src[(size_t)o * s->cells + here] + back;
        const double exchanged = (double)link_force + 2.0 * WD[o];
        const double ex = -CX[j] * exchanged, ey = -CY[j] * exchanged, ez = -CZ[j] * exchanged;
        const double rx = x - q[k] * CX[j], ry = y - q[k] * CY[j], rz = z - q[k] * CZ[j];
        fx += ex;
        fy += ey;
        fz += ez;
        mx += ry * ez - rz * ey;
        my += rz * ex - rx * ez;
        mz += rx * ey - ry * ex;
    }
    out[0] = fx;
    out[1] = fy;
    out[2] = fz;
    out[3] = mx;
    out[4] = my;
    out[5] = mz;
}

uint64_t lo32_steps(const lo32* s) {
    return s->steps;
}
