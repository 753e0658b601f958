/*
 * lbm_oracle.c - binary64 CPU restatement of Orrery's D3Q19 and D2Q9 lattice
 * Boltzmann steps.  TEST INFRASTRUCTURE ONLY (see lbm_oracle.h).
 *
 * Each node is written by exactly one OpenMP iteration and reads only the
 * previous state, so results do not depend on the thread count (the same
 * property as the reference, src/aero/lbm3d/lbm3d_cpu.cpp:1-4).
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------------- common */

static int g_threads = 0;

void lo_set_threads(int threads) {
    g_threads = threads;
}

int lo_threads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

/* 18 sqrt(2): the Smagorinsky relaxation time is the positive root of
 * tau_eff^2 - tau tau_eff - (9 sqrt(2) / 2) C^2 Q / rho = 0
 * (lbm3d_cpu.cpp:23-26, 74-77). */
#define SMAG_FACTOR (18.0 * 1.4142135623730951)

/* --------------------------------------------------------------- D3Q19 --- */

/* Velocity set, weights and symmetry tables (d3q19.h:15-36). */
static const int C3X[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const int C3Y[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
static const int C3Z[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
static const int OPP3[19] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
static const int MIRY3[19] = {0, 1, 2, 4, 3, 5, 6, 9, 10, 7, 8, 11, 12, 13, 14, 18, 17, 16, 15};
static const int MIRZ3[19] = {0, 1, 2, 3, 4, 6, 5, 7, 8, 9, 10, 13, 14, 11, 12, 17, 18, 15, 16};
static const double W3[19] = {1.0 / 3.0,  1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0,
                              1.0 / 18.0, 1.0 / 18.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                              1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                              1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};

/* Outlet history slots of the populations entering at x = nx - 1 (c_x = -1):
 * directions 2, 8, 10, 12, 14 -> slots 0..4 (lbm3d_internal.h:30-46). */
static int outlet_slot3(int i) {
    switch (i) {
        case 2: return 0;
        case 8: return 1;
        case 10: return 2;
        case 12: return 3;
        default: return 4;
    }
}

enum { CLS_SOLID = 0, CLS_BULK = 1, CLS_BOUNDARY = 2 };
enum { SRC_NODE, SRC_BOUNCE, SRC_WALL, SRC_INLET, SRC_OUTLET };

struct lo3 {
    orr_lbm3d_config c;
    long nx, ny, nz;
    size_t cells;
    uint8_t* solid;
    double* distance;   /* NULL when the mask has none */
    uint8_t* cls;
    long off[19];       /* linear offset of the pull source x - c_i */
    /* boundary links in scan order */
    size_t nlinks;
    uint32_t* lcell;
    uint32_t* ldir;
    double* lq;
    /* wall fractions of the interpolated wall: slot per cell (-1 none), 19 q per slot */
    int32_t* slot;
    double* wq;
    double* f;
    double* g;
    double* hist;
    double inlet[3];
    uint64_t steps;
};

static size_t idx3(const lo3* o, long x, long y, long z) {
    return (size_t)(x + o->nx * (y + o->ny * z));
}

/* Second-order equilibrium (d3q19.h:49-58). */
static double feq3(int i, double rho, double ux, double uy, double uz) {
    const double cu = C3X[i] * ux + C3Y[i] * uy + C3Z[i] * uz;
    const double uu = ux * ux + uy * uy + uz * uz;
    return W3[i] * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * uu);
}

/* Source of population i of fluid node (x, y, z) in the pull step
 * (resolve_source + apply_side, lbm3d_internal.h:57-130): the y sides first,
 * then z, then x, then the solid check. */
typedef struct {
    int kind;
    size_t cell;
    int dir;
    double wall_ux;
} source3;

static int side_rule(const orr_wall* low, const orr_wall* high, long* s, long n, long own,
                     int* dir, const int* mirror, double* wall_ux) {
    if (*s >= 0 && *s < n) {
        return 0;
    }
    const orr_wall* w = *s < 0 ? low : high;
    if (w->kind == ORR_WALL_PERIODIC) {
        *s = (*s + n) % n;
        return 0;
    }
    if (w->kind == ORR_WALL_SLIP) {
        *s = own;
        *dir = mirror[*dir];
        return 0;
    }
    *wall_ux = w->velocity_x;
    return 1;
}

static source3 resolve3(const lo3* o, long x, long y, long z, int i) {
    source3 s;
    const size_t here = idx3(o, x, y, z);
    long sx = x - C3X[i];
    long sy = y - C3Y[i];
    long sz = z - C3Z[i];
    int dir = i;
    double wall_ux = 0.0;
    if (side_rule(&o->c.y_low, &o->c.y_high, &sy, o->ny, y, &dir, MIRY3, &wall_ux) ||
        side_rule(&o->c.z_low, &o->c.z_high, &sz, o->nz, z, &dir, MIRZ3, &wall_ux)) {
        s.kind = SRC_WALL;
        s.cell = here;
        s.dir = OPP3[i];
        s.wall_ux = wall_ux;
        return s;
    }
    s.wall_ux = 0.0;
    if (sx < 0 || sx >= o->nx) {
        if (o->c.x_boundary == ORR_X_PERIODIC) {
            sx = (sx + o->nx) % o->nx;
        } else if (sx < 0) {
            s.kind = SRC_INLET;
            s.cell = here;
            s.dir = i;
            return s;
        } else {
            s.kind = SRC_OUTLET;
            s.cell = idx3(o, o->nx - 1, sy, sz);
            s.dir = dir;
            return s;
        }
    }
    const size_t cell = idx3(o, sx, sy, sz);
    if (o->solid[cell]) {
        s.kind = SRC_BOUNCE;
        s.cell = here;
        s.dir = OPP3[i];
        return s;
    }
    s.kind = SRC_NODE;
    s.cell = cell;
    s.dir = dir;
    return s;
}

static int inside3(const lo3* o, long x, long y, long z) {
    return x >= 0 && y >= 0 && z >= 0 && x < o->nx && y < o->ny && z < o->nz;
}

/* Wall fraction of the link from (x, y, z) towards its solid source x - c_i
 * (link_fraction, lbm3d_internal.h:132-179). */
static double link_q3(const lo3* o, long x, long y, long z, int i) {
    if (o->c.solid_wall != ORR_SOLID_INTERPOLATED || o->distance == NULL) {
        return 0.5;
    }
    const long sx = x - C3X[i], sy = y - C3Y[i], sz = z - C3Z[i];
    if (!inside3(o, sx, sy, sz)) {
        return 0.5;
    }
    const double df = o->distance[idx3(o, x, y, z)];
    const double ds = o->distance[idx3(o, sx, sy, sz)];
    if (!isfinite(df) || !isfinite(ds) || df < 0.0 || ds > 0.0 || (df == 0.0 && ds == 0.0)) {
        return 0.5;
    }
    const double span = df - ds;
    const double ratio = isfinite(span) ? df / span : 0.5 * df / (0.5 * df - 0.5 * ds);
    const double q = ratio < 1.0 ? ratio : 1.0;
    if (q < 0.5) {
        const long fx = x + C3X[i], fy = y + C3Y[i], fz = z + C3Z[i];
        if (!inside3(o, fx, fy, fz) || o->solid[idx3(o, fx, fy, fz)]) {
            return 0.5;
        }
    }
    return q;
}

/* Population the node `here` receives from the wall of its link i, from the
 * post-collision state f (reflected, lbm3d_internal.h:181-197). */
static double reflect3(const lo3* o, const double* f, size_t here, int i, double q) {
    const size_t cells = o->cells;
    const int op = OPP3[i];
    const double leaving = f[(size_t)op * cells + here];
    if (q == 0.5) {
        return leaving;
    }
    if (q < 0.5) {
        const size_t farther = (size_t)((long)here - o->off[i]);
        return 2.0 * q * leaving + (1.0 - 2.0 * q) * f[(size_t)op * cells + farther];
    }
    return (leaving + (2.0 * q - 1.0) * f[(size_t)i * cells + here]) / (2.0 * q);
}

/* Regularized Zou-He velocity inlet on the west face
 * (velocity_inlet_west, lbm3d_internal.h:312-365). */
static void inlet_west3(double* f, double ux, double uy, double uz) {
    double known = 0.0;
    for (int i = 0; i < 19; ++i) {
        if (C3X[i] == 0) {
            known += f[i];
        } else if (C3X[i] < 0) {
            known += 2.0 * f[i];
        }
    }
    const double rho = known / (1.0 - ux);
    for (int i = 0; i < 19; ++i) {
        if (C3X[i] > 0) {
            const double cu = C3X[i] * ux + C3Y[i] * uy + C3Z[i] * uz;
            f[i] = f[OPP3[i]] + 6.0 * W3[i] * rho * cu;
        }
    }
    double eq[19];
    double pi[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 19; ++i) {
        eq[i] = feq3(i, rho, ux, uy, uz);
        const double neq = f[i] - eq[i];
        const double ex = C3X[i], ey = C3Y[i], ez = C3Z[i];
        pi[0] += ex * ex * neq;
        pi[1] += ey * ey * neq;
        pi[2] += ez * ez * neq;
        pi[3] += ex * ey * neq;
        pi[4] += ex * ez * neq;
        pi[5] += ey * ez * neq;
    }
    for (int i = 0; i < 19; ++i) {
        const double ex = C3X[i], ey = C3Y[i], ez = C3Z[i];
        f[i] = eq[i] + 4.5 * W3[i] *
                           ((ex * ex - 1.0 / 3.0) * pi[0] + (ey * ey - 1.0 / 3.0) * pi[1] +
                            (ez * ez - 1.0 / 3.0) * pi[2] +
                            2.0 * (ex * ey * pi[3] + ex * ez * pi[4] + ey * ez * pi[5]));
    }
}

/* Absorbing-layer rate at a node (sponge_sigma, lbm3d_internal.h:255-281). */
static double layer(long d, uint64_t thickness) {
    if (d >= 0 && (uint64_t)d < thickness) {
        const double r = (double)(thickness - (uint64_t)d) / (double)thickness;
        return r * r;
    }
    return 0.0;
}

static double sponge3(const lo3* o, long x, long y, long z) {
    const orr_lbm3d_config* c = &o->c;
    if (!(c->sponge_strength > 0.0) || c->x_boundary != ORR_X_INFLOW_OUTFLOW) {
        return 0.0;
    }
    double best = 0.0, v;
    v = layer(x, c->sponge_inlet); best = v > best ? v : best;
    v = layer(o->nx - 1 - x, c->sponge_outlet); best = v > best ? v : best;
    if (c->y_low.kind != ORR_WALL_PERIODIC) {
        v = layer(y, c->sponge_sides); best = v > best ? v : best;
        v = layer(o->ny - 1 - y, c->sponge_sides); best = v > best ? v : best;
    }
    if (c->z_low.kind != ORR_WALL_PERIODIC) {
        v = layer(z, c->sponge_sides); best = v > best ? v : best;
        v = layer(o->nz - 1 - z, c->sponge_sides); best = v > best ? v : best;
    }
    return c->sponge_strength * best;
}

/* BGK with Guo forcing and the optional Smagorinsky closure, then the
 * absorbing-layer relaxation towards f_eq(1, stream) (collide,
 * lbm3d_cpu.cpp:28-100). */
static void collide3(double* f, const orr_lbm3d_config* c, double sponge, const double* stream) {
    double rho = 0.0;
    for (int i = 0; i < 19; ++i) {
        rho += f[i];
    }
    const double jx = f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[11] - f[12] + f[13] - f[14];
    const double jy = f[3] - f[4] + f[7] - f[8] - f[9] + f[10] + f[15] - f[16] + f[17] - f[18];
    const double jz = f[5] - f[6] + f[11] - f[12] - f[13] + f[14] + f[15] - f[16] - f[17] + f[18];
    const double fx = c->body_force_x, fy = c->body_force_y, fz = c->body_force_z;
    const double ux = (jx + 0.5 * fx) / rho;
    const double uy = (jy + 0.5 * fy) / rho;
    const double uz = (jz + 0.5 * fz) / rho;
    const double base = 1.0 - 1.5 * (ux * ux + uy * uy + uz * uz);
    const double cu[19] = {0.0,     ux,       -ux,      uy,      -uy,     uz,       -uz,
                           ux + uy, -ux - uy, ux - uy,  uy - ux, ux + uz, -ux - uz, ux - uz,
                           uz - ux, uy + uz,  -uy - uz, uy - uz, uz - uy};
    double eq[19];
    for (int i = 0; i < 19; ++i) {
        eq[i] = W3[i] * rho * (base + cu[i] * (3.0 + 4.5 * cu[i]));
    }
    double tau = c->tau;
    if (c->smagorinsky_enabled) {
        double pi[6] = {0, 0, 0, 0, 0, 0};
        for (int i = 0; i < 19; ++i) {
            const double neq = f[i] - eq[i];
            const double ex = C3X[i], ey = C3Y[i], ez = C3Z[i];
            pi[0] += ex * ex * neq;
            pi[1] += ey * ey * neq;
            pi[2] += ez * ez * neq;
            pi[3] += ex * ey * neq;
            pi[4] += ex * ez * neq;
            pi[5] += ey * ez * neq;
        }
        const double strain = sqrt(pi[0] * pi[0] + pi[1] * pi[1] + pi[2] * pi[2] +
                                   2.0 * (pi[3] * pi[3] + pi[4] * pi[4] + pi[5] * pi[5]));
        const double k = c->smagorinsky_constant;
        tau = 0.5 * (tau + sqrt(tau * tau + SMAG_FACTOR * k * k * strain / rho));
    }
    const double omega = 1.0 / tau;
    const int forced = fx != 0.0 || fy != 0.0 || fz != 0.0;
    const double scale = 1.0 - 0.5 * omega;
    for (int i = 0; i < 19; ++i) {
        double v = f[i] - omega * (f[i] - eq[i]);
        if (forced) {
            const double ex = C3X[i], ey = C3Y[i], ez = C3Z[i];
            v += scale * W3[i] *
                 (3.0 * ((ex - ux) * fx + (ey - uy) * fy + (ez - uz) * fz) +
                  9.0 * cu[i] * (ex * fx + ey * fy + ez * fz));
        }
        f[i] = v;
    }
    if (sponge > 0.0) {
        for (int i = 0; i < 19; ++i) {
            f[i] -= sponge * (f[i] - feq3(i, 1.0, stream[0], stream[1], stream[2]));
        }
    }
}

static void reset_history3(lo3* o) {
    const size_t face = (size_t)(o->ny * o->nz);
    static const int dirs[5] = {2, 8, 10, 12, 14};
    for (long z = 0; z < o->nz; ++z) {
        for (long y = 0; y < o->ny; ++y) {
            const size_t cell = idx3(o, o->nx - 1, y, z);
            for (int k = 0; k < 5; ++k) {
                const int i = dirs[k];
                o->hist[(size_t)outlet_slot3(i) * face + (size_t)(y + o->ny * z)] =
                    o->f[(size_t)i * o->cells + cell];
            }
        }
    }
}

lo3* lo3_create(const orr_lbm3d_config* config, const uint8_t* solid, const double* distance) {
    lo3* o = (lo3*)calloc(1, sizeof(lo3));
    o->c = *config;
    o->nx = (long)config->nx;
    o->ny = (long)config->ny;
    o->nz = (long)config->nz;
    o->cells = (size_t)(o->nx * o->ny * o->nz);
    o->solid = (uint8_t*)malloc(o->cells);
    memcpy(o->solid, solid, o->cells);
    if (distance != NULL) {
        o->distance = (double*)malloc(o->cells * sizeof(double));
        memcpy(o->distance, distance, o->cells * sizeof(double));
    }
    const long plane = o->nx * o->ny;
    for (int i = 0; i < 19; ++i) {
        o->off[i] = -C3X[i] - o->nx * C3Y[i] - plane * C3Z[i];
    }
    /* Node classes (classify_nodes, lbm3d_internal.h:214-248). */
    o->cls = (uint8_t*)malloc(o->cells);
    for (long z = 0; z < o->nz; ++z) {
        for (long y = 0; y < o->ny; ++y) {
            for (long x = 0; x < o->nx; ++x) {
                const size_t h = idx3(o, x, y, z);
                if (o->solid[h]) {
                    o->cls[h] = CLS_SOLID;
                    continue;
                }
                uint8_t k = CLS_BULK;
                if (x == 0 || y == 0 || z == 0 || x + 1 == o->nx || y + 1 == o->ny ||
                    z + 1 == o->nz) {
                    k = CLS_BOUNDARY;
                } else {
                    for (int i = 1; i < 19; ++i) {
                        if (o->solid[(size_t)((long)h + o->off[i])]) {
                            k = CLS_BOUNDARY;
                            break;
                        }
                    }
                }
                o->cls[h] = k;
            }
        }
    }
    /* Boundary links in scan order (boundary_links, lbm3d_common.cpp:176-198). */
    size_t cap = 1024, n = 0;
    o->lcell = (uint32_t*)malloc(cap * sizeof(uint32_t));
    o->ldir = (uint32_t*)malloc(cap * sizeof(uint32_t));
    o->lq = (double*)malloc(cap * sizeof(double));
    for (long z = 0; z < o->nz; ++z) {
        for (long y = 0; y < o->ny; ++y) {
            for (long x = 0; x < o->nx; ++x) {
                const size_t h = idx3(o, x, y, z);
                if (o->solid[h]) {
                    continue;
                }
                for (int i = 1; i < 19; ++i) {
                    if (resolve3(o, x, y, z, i).kind != SRC_BOUNCE) {
                        continue;
                    }
                    if (n == cap) {
                        cap *= 2;
                        o->lcell = (uint32_t*)realloc(o->lcell, cap * sizeof(uint32_t));
                        o->ldir = (uint32_t*)realloc(o->ldir, cap * sizeof(uint32_t));
                        o->lq = (double*)realloc(o->lq, cap * sizeof(double));
                    }
                    o->lcell[n] = (uint32_t)h;
                    o->ldir[n] = (uint32_t)i;
                    o->lq[n] = link_q3(o, x, y, z, i);
                    ++n;
                }
            }
        }
    }
    o->nlinks = n;
    /* Wall table of the interpolated wall (wall_table, lbm3d_internal.h:283-310). */
    if (config->solid_wall == ORR_SOLID_INTERPOLATED) {
        o->slot = (int32_t*)malloc(o->cells * sizeof(int32_t));
        for (size_t k = 0; k < o->cells; ++k) {
            o->slot[k] = -1;
        }
        size_t slots = 0;
        for (size_t k = 0; k < n; ++k) {
            if (o->slot[o->lcell[k]] < 0) {
                o->slot[o->lcell[k]] = (int32_t)slots++;
            }
        }
        o->wq = (double*)malloc((slots > 0 ? slots : 1) * 19 * sizeof(double));
        for (size_t k = 0; k < slots * 19; ++k) {
            o->wq[k] = 0.5;
        }
        for (size_t k = 0; k < n; ++k) {
            o->wq[(size_t)o->slot[o->lcell[k]] * 19 + o->ldir[k]] = o->lq[k];
        }
    }
    o->f = (double*)malloc(19 * o->cells * sizeof(double));
    o->g = (double*)malloc(19 * o->cells * sizeof(double));
    o->hist = (double*)malloc(5 * (size_t)(o->ny * o->nz) * sizeof(double));
    lo3_initialize(o, NULL, NULL, NULL, NULL);
    return o;
}

void lo3_destroy(lo3* o) {
    if (o == NULL) {
        return;
    }
    free(o->solid);
    free(o->distance);
    free(o->cls);
    free(o->lcell);
    free(o->ldir);
    free(o->lq);
    free(o->slot);
    free(o->wq);
    free(o->f);
    free(o->g);
    free(o->hist);
    free(o);
}

/* Equilibrium of the given fields, solids at rest (initial_populations and
 * uniform_inlet_state, lbm3d_common.cpp:243-270); the step count and the
 * inlet velocity are reset (lbm3d_cpu.cpp:129-136). */
void lo3_initialize(lo3* o, const double* rho, const double* ux, const double* uy,
                    const double* uz) {
    const int inflow = o->c.x_boundary == ORR_X_INFLOW_OUTFLOW;
    const double u0x = inflow ? o->c.inlet_ux : 0.0;
    const double u0y = inflow ? o->c.inlet_uy : 0.0;
    const double u0z = inflow ? o->c.inlet_uz : 0.0;
    for (size_t h = 0; h < o->cells; ++h) {
        double r = 1.0, vx = 0.0, vy = 0.0, vz = 0.0;
        if (!o->solid[h]) {
            if (rho != NULL) {
                r = rho[h];
                vx = ux[h];
                vy = uy[h];
                vz = uz[h];
            } else {
                vx = u0x;
                vy = u0y;
                vz = u0z;
            }
        }
        for (int i = 0; i < 19; ++i) {
            o->f[(size_t)i * o->cells + h] = feq3(i, r, vx, vy, vz);
        }
    }
    memcpy(o->g, o->f, 19 * o->cells * sizeof(double));
    reset_history3(o);
    o->inlet[0] = o->c.inlet_ux;
    o->inlet[1] = o->c.inlet_uy;
    o->inlet[2] = o->c.inlet_uz;
    o->steps = 0;
}

void lo3_set_inlet(lo3* o, const double velocity[3]) {
    o->inlet[0] = velocity[0];
    o->inlet[1] = velocity[1];
    o->inlet[2] = velocity[2];
}

/* One row of constant (y, z) (update_row, lbm3d_cpu.cpp:261-322). */
static void row3(lo3* o, long y, long z) {
    const size_t cells = o->cells;
    const double* f = o->f;
    double* g = o->g;
    const size_t face = (size_t)(o->ny * o->nz);
    const int inflow = o->c.x_boundary == ORR_X_INFLOW_OUTFLOW;
    for (long x = 0; x < o->nx; ++x) {
        const size_t h = idx3(o, x, y, z);
        const uint8_t k = o->cls[h];
        if (k == CLS_SOLID) {
            continue;
        }
        double p[19];
        if (k == CLS_BULK) {
            for (int i = 0; i < 19; ++i) {
                p[i] = f[(size_t)i * cells + (size_t)((long)h + o->off[i])];
            }
        } else {
            double wall_rho = -1.0;
            for (int i = 0; i < 19; ++i) {
                const source3 s = resolve3(o, x, y, z, i);
                switch (s.kind) {
                    case SRC_NODE:
                        p[i] = f[(size_t)s.dir * cells + s.cell];
                        break;
                    case SRC_BOUNCE:
                        if (o->slot != NULL && o->slot[h] >= 0) {
                            p[i] = reflect3(o, f, h, i, o->wq[(size_t)o->slot[h] * 19 + i]);
                        } else {
                            p[i] = f[(size_t)s.dir * cells + s.cell];
                        }
                        break;
                    case SRC_WALL:
                        if (wall_rho < 0.0) {
                            wall_rho = 0.0;
                            for (int j = 0; j < 19; ++j) {
                                wall_rho += f[(size_t)j * cells + h];
                            }
                        }
                        p[i] = f[(size_t)s.dir * cells + s.cell] +
                               6.0 * W3[i] * wall_rho * C3X[i] * s.wall_ux;
                        break;
                    case SRC_INLET:
                        p[i] = 0.0;
                        break;
                    default: { /* SRC_OUTLET (outlet_value, lbm3d_cpu.cpp:239-250) */
                        const double up = f[(size_t)s.dir * cells + s.cell];
                        if (o->c.outlet == ORR_OUTLET_EXTRAPOLATION) {
                            p[i] = up;
                        } else {
                            const double u = o->c.inlet_ux;
                            double* prev =
                                &o->hist[(size_t)outlet_slot3(i) * face + (size_t)(y + o->ny * z)];
                            *prev = (*prev + u * up) / (1.0 + u);
                            p[i] = *prev;
                        }
                        break;
                    }
                }
            }
            if (inflow && x == 0) {
                inlet_west3(p, o->inlet[0], o->inlet[1], o->inlet[2]);
            }
        }
        collide3(p, &o->c, sponge3(o, x, y, z), o->inlet);
        for (int i = 0; i < 19; ++i) {
            g[(size_t)i * cells + h] = p[i];
        }
    }
}

void lo3_step(lo3* o, uint64_t count) {
    const long rows = o->ny * o->nz;
    for (uint64_t n = 0; n < count; ++n) {
#pragma omp parallel for schedule(static) num_threads(lo_threads())
        for (long r = 0; r < rows; ++r) {
            row3(o, r % o->ny, r / o->ny);
        }
        double* t = o->f;
        o->f = o->g;
        o->g = t;
        ++o->steps;
    }
}

void lo3_populations(const lo3* o, double* f) {
    memcpy(f, o->f, 19 * o->cells * sizeof(double));
}

/* Momentum exchange over the boundary links (CpuLbm3D::force,
 * lbm3d_cpu.cpp:192-203; add_link_force and link_wall_point,
 * lbm3d_common.cpp:213-241). */
void lo3_force(const lo3* o, double out[6]) {
    double F[3] = {0, 0, 0}, M[3] = {0, 0, 0};
    const size_t plane = (size_t)(o->nx * o->ny);
    for (size_t k = 0; k < o->nlinks; ++k) {
        const size_t h = o->lcell[k];
        const int j = (int)o->ldir[k];
        const int op = OPP3[j];
        const double q = o->lq[k];
        const double ex = o->f[(size_t)op * o->cells + h] + reflect3(o, o->f, h, j, q);
        const double fl[3] = {C3X[op] * ex, C3Y[op] * ex, C3Z[op] * ex};
        const size_t z = h / plane, rest = h % plane;
        const size_t y = rest / (size_t)o->nx, x = rest % (size_t)o->nx;
        const double r[3] = {(double)x - q * C3X[j], (double)y - q * C3Y[j],
                             (double)z - q * C3Z[j]};
        F[0] += fl[0];
        F[1] += fl[1];
        F[2] += fl[2];
        M[0] += r[1] * fl[2] - r[2] * fl[1];
        M[1] += r[2] * fl[0] - r[0] * fl[2];
        M[2] += r[0] * fl[1] - r[1] * fl[0];
    }
    out[0] = F[0];
    out[1] = F[1];
    out[2] = F[2];
    out[3] = M[0];
    out[4] = M[1];
    out[5] = M[2];
}

/* Moments with the Guo half-force correction; solids at rest
 * (CpuLbm3D::macroscopic, lbm3d_cpu.cpp:154-186). */
void lo3_macroscopic(const lo3* o, double* rho, double* ux, double* uy, double* uz) {
    for (size_t h = 0; h < o->cells; ++h) {
        if (o->solid[h]) {
            rho[h] = 1.0;
            ux[h] = uy[h] = uz[h] = 0.0;
            continue;
        }
        double r = 0, jx = 0, jy = 0, jz = 0;
        for (int i = 0; i < 19; ++i) {
            const double v = o->f[(size_t)i * o->cells + h];
            r += v;
            jx += C3X[i] * v;
            jy += C3Y[i] * v;
            jz += C3Z[i] * v;
        }
        rho[h] = r;
        ux[h] = (jx - 0.5 * o->c.body_force_x) / r;
        uy[h] = (jy - 0.5 * o->c.body_force_y) / r;
        uz[h] = (jz - 0.5 * o->c.body_force_z) / r;
    }
}

double lo3_mass(const lo3* o) {
    double total = 0.0;
    for (size_t h = 0; h < o->cells; ++h) {
        if (!o->solid[h]) {
            for (int i = 0; i < 19; ++i) {
                total += o->f[(size_t)i * o->cells + h];
            }
        }
    }
    return total;
}

uint64_t lo3_link_count(const lo3* o) {
    return o->nlinks;
}

void lo3_links(const lo3* o, uint32_t* cell, uint32_t* direction, double* q) {
    for (size_t k = 0; k < o->nlinks; ++k) {
        cell[k] = o->lcell[k];
        direction[k] = o->ldir[k];
        q[k] = o->lq[k];
    }
}

uint64_t lo3_boundary_count(const lo3* o) {
    uint64_t n = 0;
    for (size_t h = 0; h < o->cells; ++h) {
        n += o->cls[h] == CLS_BOUNDARY;
    }
    return n;
}

/* ---------------------------------------------------------------- D2Q9 --- */

/* d2q9.h:12-23: 0 rest, 1 E, 2 N, 3 W, 4 S, 5 NE, 6 NW, 7 SW, 8 SE. */
static const int C2X[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
static const int C2Y[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
static const int OPP2[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
static const int MIRY2[9] = {0, 1, 4, 3, 2, 8, 7, 6, 5};
static const double W2[9] = {4.0 / 9.0,  1.0 / 9.0,  1.0 / 9.0,  1.0 / 9.0, 1.0 / 9.0,
                             1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};

struct lo2 {
    orr_lbm2d_config c;
    long nx, ny;
    size_t cells;
    uint8_t* solid;
    uint8_t* cls;
    long off[9];
    size_t nlinks;
    uint32_t* lcell;
    uint32_t* ldir;
    double* f;
    double* g;
    double* hist;
    uint64_t steps;
};

static double feq2(int i, double rho, double ux, double uy) {
    const double cu = C2X[i] * ux + C2Y[i] * uy;
    const double uu = ux * ux + uy * uy;
    return W2[i] * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * uu);
}

/* Outlet history slot of directions 3, 6, 7 (lbm2d_internal.h:24-27). */
static int outlet_slot2(int i) {
    return i == 3 ? 0 : (i == 6 ? 1 : 2);
}

typedef struct {
    int kind;
    size_t cell;
    int dir;
    double wall_ux;
} source2;

/* resolve_source (lbm2d_internal.h:36-75). */
static source2 resolve2(const lo2* o, long x, long y, int i) {
    source2 s;
    const size_t here = (size_t)(x + o->nx * y);
    long sx = x - C2X[i];
    long sy = y - C2Y[i];
    int dir = i;
    s.wall_ux = 0.0;
    if (sy < 0 || sy >= o->ny) {
        const orr_wall* w = sy < 0 ? &o->c.bottom : &o->c.top;
        if (w->kind == ORR_WALL_PERIODIC) {
            sy = (sy + o->ny) % o->ny;
        } else if (w->kind == ORR_WALL_SLIP) {
            sy = y;
            dir = MIRY2[i];
        } else {
            s.kind = SRC_WALL;
            s.cell = here;
            s.dir = OPP2[i];
            s.wall_ux = w->velocity_x;
            return s;
        }
    }
    if (sx < 0 || sx >= o->nx) {
        if (o->c.x_boundary == ORR_X_PERIODIC) {
            sx = (sx + o->nx) % o->nx;
        } else if (sx < 0) {
            s.kind = SRC_INLET;
            s.cell = here;
            s.dir = i;
            return s;
        } else {
            s.kind = SRC_OUTLET;
            s.cell = (size_t)(o->nx - 1 + o->nx * sy);
            s.dir = dir;
            return s;
        }
    }
    const size_t cell = (size_t)(sx + o->nx * sy);
    if (o->solid[cell]) {
        s.kind = SRC_BOUNCE;
        s.cell = here;
        s.dir = OPP2[i];
        return s;
    }
    s.kind = SRC_NODE;
    s.cell = cell;
    s.dir = dir;
    return s;
}

/* Zou-He west inlet, then regularized (zou_he_west, lbm2d_internal.h:77-111). */
static void inlet_west2(double* f, double ux, double uy) {
    const double rho = (f[0] + f[2] + f[4] + 2.0 * (f[3] + f[6] + f[7])) / (1.0 - ux);
    f[1] = f[3] + (2.0 / 3.0) * rho * ux;
    f[5] = f[7] - 0.5 * (f[2] - f[4]) + (1.0 / 6.0) * rho * ux + 0.5 * rho * uy;
    f[8] = f[6] + 0.5 * (f[2] - f[4]) + (1.0 / 6.0) * rho * ux - 0.5 * rho * uy;
    double eq[9];
    double pxx = 0.0, pyy = 0.0, pxy = 0.0;
    for (int i = 0; i < 9; ++i) {
        eq[i] = feq2(i, rho, ux, uy);
        const double neq = f[i] - eq[i];
        const double ex = C2X[i], ey = C2Y[i];
        pxx += ex * ex * neq;
        pyy += ey * ey * neq;
        pxy += ex * ey * neq;
    }
    for (int i = 0; i < 9; ++i) {
        const double ex = C2X[i], ey = C2Y[i];
        f[i] = eq[i] + 4.5 * W2[i] *
                           ((ex * ex - 1.0 / 3.0) * pxx + (ey * ey - 1.0 / 3.0) * pyy +
                            2.0 * ex * ey * pxy);
    }
}

/* collide (lbm2d_cpu.cpp:26-75). */
static void collide2(double* f, const orr_lbm2d_config* c) {
    const double rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
    const double jx = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
    const double jy = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
    const double fx = c->body_force_x, fy = c->body_force_y;
    const double ux = (jx + 0.5 * fx) / rho;
    const double uy = (jy + 0.5 * fy) / rho;
    const double base = 1.0 - 1.5 * (ux * ux + uy * uy);
    const double cu[9] = {0.0, ux, uy, -ux, -uy, ux + uy, uy - ux, -ux - uy, ux - uy};
    double eq[9];
    for (int i = 0; i < 9; ++i) {
        eq[i] = W2[i] * rho * (base + cu[i] * (3.0 + 4.5 * cu[i]));
    }
    double tau = c->tau;
    if (c->smagorinsky_enabled) {
        double pxx = 0.0, pyy = 0.0, pxy = 0.0;
        for (int i = 0; i < 9; ++i) {
            const double neq = f[i] - eq[i];
            const double ex = C2X[i], ey = C2Y[i];
            pxx += ex * ex * neq;
            pyy += ey * ey * neq;
            pxy += ex * ey * neq;
        }
        const double strain = sqrt(pxx * pxx + pyy * pyy + 2.0 * pxy * pxy);
        const double k = c->smagorinsky_constant;
        tau = 0.5 * (tau + sqrt(tau * tau + SMAG_FACTOR * k * k * strain / rho));
    }
    const double omega = 1.0 / tau;
    const int forced = fx != 0.0 || fy != 0.0;
    const double scale = 1.0 - 0.5 * omega;
    for (int i = 0; i < 9; ++i) {
        double v = f[i] - omega * (f[i] - eq[i]);
        if (forced) {
            const double ex = C2X[i], ey = C2Y[i];
            v += scale * W2[i] * (3.0 * ((ex - ux) * fx + (ey - uy) * fy) + 9.0 * cu[i] * (ex * fx + ey * fy));
        }
        f[i] = v;
    }
}

static void reset_history2(lo2* o) {
    for (long y = 0; y < o->ny; ++y) {
        const size_t cell = (size_t)(o->nx - 1 + o->nx * y);
        static const int dirs[3] = {3, 6, 7};
        for (int k = 0; k < 3; ++k) {
            o->hist[(size_t)outlet_slot2(dirs[k]) * (size_t)o->ny + (size_t)y] =
                o->f[(size_t)dirs[k] * o->cells + cell];
        }
    }
}

lo2* lo2_create(const orr_lbm2d_config* config, const uint8_t* solid) {
    lo2* o = (lo2*)calloc(1, sizeof(lo2));
    o->c = *config;
    o->nx = (long)config->nx;
    o->ny = (long)config->ny;
    o->cells = (size_t)(o->nx * o->ny);
    o->solid = (uint8_t*)malloc(o->cells);
    memcpy(o->solid, solid, o->cells);
    for (int i = 0; i < 9; ++i) {
        o->off[i] = -C2X[i] - o->nx * C2Y[i];
    }
    /* Node classes (CpuLbm2D::classify_nodes, lbm2d_cpu.cpp:312-341). */
    o->cls = (uint8_t*)malloc(o->cells);
    for (long y = 0; y < o->ny; ++y) {
        for (long x = 0; x < o->nx; ++x) {
            const size_t h = (size_t)(x + o->nx * y);
            if (o->solid[h]) {
                o->cls[h] = CLS_SOLID;
                continue;
            }
            uint8_t k = CLS_BULK;
            if (x == 0 || y == 0 || x + 1 == o->nx || y + 1 == o->ny) {
                k = CLS_BOUNDARY;
            } else {
                for (int i = 1; i < 9; ++i) {
                    if (o->solid[(size_t)((long)h + o->off[i])]) {
                        k = CLS_BOUNDARY;
                        break;
                    }
                }
            }
            o->cls[h] = k;
        }
    }
    /* boundary_links (lbm2d_common.cpp:79-97). */
    size_t cap = 256, n = 0;
    o->lcell = (uint32_t*)malloc(cap * sizeof(uint32_t));
    o->ldir = (uint32_t*)malloc(cap * sizeof(uint32_t));
    for (long y = 0; y < o->ny; ++y) {
        for (long x = 0; x < o->nx; ++x) {
            const size_t h = (size_t)(x + o->nx * y);
            if (o->solid[h]) {
                continue;
            }
            for (int i = 1; i < 9; ++i) {
                if (resolve2(o, x, y, i).kind != SRC_BOUNCE) {
                    continue;
                }
                if (n == cap) {
                    cap *= 2;
                    o->lcell = (uint32_t*)realloc(o->lcell, cap * sizeof(uint32_t));
                    o->ldir = (uint32_t*)realloc(o->ldir, cap * sizeof(uint32_t));
                }
                o->lcell[n] = (uint32_t)h;
                o->ldir[n] = (uint32_t)i;
                ++n;
            }
        }
    }
    o->nlinks = n;
    o->f = (double*)malloc(9 * o->cells * sizeof(double));
    o->g = (double*)malloc(9 * o->cells * sizeof(double));
    o->hist = (double*)malloc(3 * (size_t)o->ny * sizeof(double));
    lo2_initialize(o, NULL, NULL, NULL);
    return o;
}

void lo2_destroy(lo2* o) {
    if (o == NULL) {
        return;
    }
    free(o->solid);
    free(o->cls);
    free(o->lcell);
    free(o->ldir);
    free(o->f);
    free(o->g);
    free(o->hist);
    free(o);
}

/* initial_populations / uniform_inlet_state (lbm2d_common.cpp:178-199). */
void lo2_initialize(lo2* o, const double* rho, const double* ux, const double* uy) {
    const int inflow = o->c.x_boundary == ORR_X_INFLOW_OUTFLOW;
    const double u0x = inflow ? o->c.inlet_ux : 0.0;
    const double u0y = inflow ? o->c.inlet_uy : 0.0;
    for (size_t h = 0; h < o->cells; ++h) {
        double r = 1.0, vx = 0.0, vy = 0.0;
        if (!o->solid[h]) {
            if (rho != NULL) {
                r = rho[h];
                vx = ux[h];
                vy = uy[h];
            } else {
                vx = u0x;
                vy = u0y;
            }
        }
        for (int i = 0; i < 9; ++i) {
            o->f[(size_t)i * o->cells + h] = feq2(i, r, vx, vy);
        }
    }
    memcpy(o->g, o->f, 9 * o->cells * sizeof(double));
    reset_history2(o);
    o->steps = 0;
}

/* update_row (lbm2d_cpu.cpp:352-404). */
static void row2(lo2* o, long y) {
    const size_t cells = o->cells;
    const double* f = o->f;
    double* g = o->g;
    const int inflow = o->c.x_boundary == ORR_X_INFLOW_OUTFLOW;
    for (long x = 0; x < o->nx; ++x) {
        const size_t h = (size_t)(x + o->nx * y);
        const uint8_t k = o->cls[h];
        if (k == CLS_SOLID) {
            continue;
        }
        double p[9];
        if (k == CLS_BULK) {
            for (int i = 0; i < 9; ++i) {
                p[i] = f[(size_t)i * cells + (size_t)((long)h + o->off[i])];
            }
        } else {
            double wall_rho = -1.0;
            for (int i = 0; i < 9; ++i) {
                const source2 s = resolve2(o, x, y, i);
                switch (s.kind) {
                    case SRC_NODE:
                    case SRC_BOUNCE:
                        p[i] = f[(size_t)s.dir * cells + s.cell];
                        break;
                    case SRC_WALL:
                        if (wall_rho < 0.0) {
                            wall_rho = 0.0;
                            for (int j = 0; j < 9; ++j) {
                                wall_rho += f[(size_t)j * cells + h];
                            }
                        }
                        p[i] = f[(size_t)s.dir * cells + s.cell] +
                               6.0 * W2[i] * wall_rho * C2X[i] * s.wall_ux;
                        break;
                    case SRC_INLET:
                        p[i] = 0.0;
                        break;
                    default: {
                        const double up = f[(size_t)s.dir * cells + s.cell];
                        if (o->c.outlet == ORR_OUTLET_EXTRAPOLATION) {
                            p[i] = up;
                        } else {
                            const double u = o->c.inlet_ux;
                            double* prev = &o->hist[(size_t)outlet_slot2(i) * (size_t)o->ny + (size_t)y];
                            *prev = (*prev + u * up) / (1.0 + u);
                            p[i] = *prev;
                        }
                        break;
                    }
                }
            }
            if (inflow && x == 0) {
                inlet_west2(p, o->c.inlet_ux, o->c.inlet_uy);
            }
        }
        collide2(p, &o->c);
        for (int i = 0; i < 9; ++i) {
            g[(size_t)i * cells + h] = p[i];
        }
    }
}

void lo2_step(lo2* o, uint64_t count) {
    for (uint64_t n = 0; n < count; ++n) {
#pragma omp parallel for schedule(static) num_threads(lo_threads())
        for (long y = 0; y < o->ny; ++y) {
            row2(o, y);
        }
        double* t = o->f;
        o->f = o->g;
        o->g = t;
        ++o->steps;
    }
}

void lo2_populations(const lo2* o, double* f) {
    memcpy(f, o->f, 9 * o->cells * sizeof(double));
}

/* Force2D over the links, 2 c_o f*_o at the halfway wall point
 * (CpuLbm2D::force, lbm2d_cpu.cpp:265-272; add_link_force, lbm2d.h:145-155). */
void lo2_force(const lo2* o, double out[3]) {
    double fx = 0.0, fy = 0.0, m = 0.0;
    for (size_t k = 0; k < o->nlinks; ++k) {
        const size_t h = o->lcell[k];
        const int j = (int)o->ldir[k];
        const int op = OPP2[j];
        const double v = o->f[(size_t)op * o->cells + h];
        const double ax = 2.0 * C2X[op] * v;
        const double ay = 2.0 * C2Y[op] * v;
        const double rx = (double)(h % (size_t)o->nx) - 0.5 * C2X[j];
        const double ry = (double)(h / (size_t)o->nx) - 0.5 * C2Y[j];
        fx += ax;
        fy += ay;
        m += rx * ay - ry * ax;
    }
    out[0] = fx;
    out[1] = fy;
    out[2] = m;
}

void lo2_macroscopic(const lo2* o, double* rho, double* ux, double* uy) {
    for (size_t h = 0; h < o->cells; ++h) {
        if (o->solid[h]) {
            rho[h] = 1.0;
            ux[h] = uy[h] = 0.0;
            continue;
        }
        double r = 0, jx = 0, jy = 0;
        for (int i = 0; i < 9; ++i) {
            const double v = o->f[(size_t)i * o->cells + h];
            r += v;
            jx += C2X[i] * v;
            jy += C2Y[i] * v;
        }
        rho[h] = r;
        ux[h] = (jx - 0.5 * o->c.body_force_x) / r;
        uy[h] = (jy - 0.5 * o->c.body_force_y) / r;
    }
}

double lo2_mass(const lo2* o) {
    double total = 0.0;
    for (size_t h = 0; h < o->cells; ++h) {
        if (!o->solid[h]) {
            for (int i = 0; i < 9; ++i) {
                total += o->f[(size_t)i * o->cells + h];
            }
        }
    }
    return total;
}

uint64_t lo2_link_count(const lo2* o) {
    return o->nlinks;
}

void lo2_links(const lo2* o, uint32_t* cell, uint32_t* direction) {
    for (size_t k = 0; k < o->nlinks; ++k) {
        cell[k] = o->lcell[k];
        direction[k] = o->ldir[k];
    }
}
