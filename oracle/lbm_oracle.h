/*
 * lbm_oracle.h - CPU restatement of Orrery's lattice Boltzmann step, in plain
 * C and binary64.  TEST INFRASTRUCTURE ONLY: tests, the smoke check and the
 * benchmark's CPU-baseline leg use it as the checker; the product never links
 * or loads it.
 *
 * It restates, in its own code, the algorithm of the reference's CPU solvers
 *   src/aero/lbm3d/lbm3d_cpu.cpp, src/aero/lbm3d/lbm3d_internal.h,
 *   src/aero/lbm3d/lbm3d_common.cpp  (D3Q19)
 *   src/aero/lbm/lbm2d_cpu.cpp, src/aero/lbm/lbm2d_internal.h,
 *   src/aero/lbm/lbm2d_common.cpp, src/aero/lbm/include/orrery/aero/lbm/lbm2d.h (D2Q9)
 * and is pinned against that reference compiled in place (oracle/_ref) and
 * against the reference's own known-answer tests (tests/aero/lbm3d/
 * test_lbm3d_flows.cpp, tests/aero/lbm/test_lbm2d_flows.cpp).
 *
 * No validation is done here: callers pass configurations the reference
 * accepts.  Configurations use the structs of include/orrery_lbm.h.
 */
#ifndef ORRERY_LBM_ORACLE_H
#define ORRERY_LBM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/orrery_lbm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lo3 lo3;
typedef struct lo2 lo2;

void lo_set_threads(int threads);
int lo_threads(void);

lo3* lo3_create(const orr_lbm3d_config* config, const uint8_t* solid, const double* distance);
void lo3_destroy(lo3* o);
void lo3_initialize(lo3* o, const double* rho, const double* ux, const double* uy, const double* uz);
void lo3_step(lo3* o, uint64_t count);
void lo3_set_inlet(lo3* o, const double velocity[3]);
void lo3_populations(const lo3* o, double* f);
void lo3_force(const lo3* o, double out[6]);
void lo3_macroscopic(const lo3* o, double* rho, double* ux, double* uy, double* uz);
double lo3_mass(const lo3* o);
uint64_t lo3_link_count(const lo3* o);
void lo3_links(const lo3* o, uint32_t* cell, uint32_t* direction, double* q);
uint64_t lo3_boundary_count(const lo3* o);

lo2* lo2_create(const orr_lbm2d_config* config, const uint8_t* solid);
void lo2_destroy(lo2* o);
void lo2_initialize(lo2* o, const double* rho, const double* ux, const double* uy);
void lo2_step(lo2* o, uint64_t count);
void lo2_populations(const lo2* o, double* f);
void lo2_force(const lo2* o, double out[3]);
void lo2_macroscopic(const lo2* o, double* rho, double* ux, double* uy);
double lo2_mass(const lo2* o);
uint64_t lo2_link_count(const lo2* o);
void lo2_links(const lo2* o, uint32_t* cell, uint32_t* direction);

#ifdef __cplusplus
}
#endif

#endif
