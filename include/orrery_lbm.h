/*
 * orrery_lbm.h - C ABI of the B200 lattice Boltzmann solvers (D3Q19 and D2Q9).
 *
 * This is the drop-in boundary for Orrery's LBM hot path.  Every entry point
 * below replaces one member of the reference's solver seam
 *   class Lbm3DSolver          src/aero/lbm3d/include/orrery/aero/lbm3d/lbm3d.h:196-232
 *   make_gpu_solver (3D)       src/aero/lbm3d/include/orrery/aero/lbm3d/lbm3d.h:246-247
 *   class Lbm2DSolver          src/aero/lbm/include/orrery/aero/lbm/lbm2d.h:173-202
 *   make_gpu_solver (2D)       src/aero/lbm/include/orrery/aero/lbm/lbm2d.h:211-212
 * and is cited at its declaration.  The signatures carry plain C types only:
 * host pointers, sizes and opaque handles.
 *
 * Conventions
 *   - Every call returns an orr_status; 0 is success.  The text of the last
 *     failure is available from orr_lbm3d_last_error(handle) (per handle) or
 *     orr_last_error() (per thread; also set by failed create calls).  Error
 *     texts follow the reference's wording (lbm3d_common.cpp:74-155,
 *     lbm3d_gpu.cpp:94-149) so callers that match on them keep working.
 *   - Nothing throws across this boundary.  Creation refuses a configuration
 *     before allocating anything on the device (lbm3d_gpu.cpp:488-513).
 *   - Node (x, y, z) has the linear index x + nx (y + ny z); populations are
 *     reported structure-of-arrays, f[i * cells + cell], in the reference's
 *     D3Q19 / D2Q9 direction order (d3q19.h:15-36, d2q9.h:12-23), unshifted.
 *   - The library copies every caller array it is given; callers keep
 *     ownership.  A handle owns one CUDA stream and is not thread-safe.
 */
#ifndef ORRERY_LBM_H
#define ORRERY_LBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define ORR_API __attribute__((visibility("default")))
#else
#define ORR_API
#endif

typedef int32_t orr_status;
enum {
    ORR_OK = 0,
    ORR_ERR_INVALID = 1,   /* configuration, mask or argument refused */
    ORR_ERR_MEMORY = 2,    /* device memory refused or exhausted */
    ORR_ERR_CUDA = 3,      /* a CUDA call failed */
    ORR_ERR_STATE = 4,     /* call not valid in the handle's state */
    ORR_ERR_TIMEOUT = 5,   /* a bounded device wait gave up */
    ORR_ERR_DIVERGED = 6,  /* non-finite coefficients detected */
    ORR_ERR_NO_DEVICE = 7  /* no CUDA device of compute capability 10.0 */
};

/* Wall kinds of the y and z sides (WallKind, lbm2d.h:51). */
enum { ORR_WALL_PERIODIC = 0, ORR_WALL_SLIP = 1, ORR_WALL_NO_SLIP = 2 };
/* x boundary (XBoundary, lbm2d.h:43). */
enum { ORR_X_PERIODIC = 0, ORR_X_INFLOW_OUTFLOW = 1 };
/* Outlet treatment (Outlet, lbm2d.h:50). */
enum { ORR_OUTLET_CONVECTIVE = 0, ORR_OUTLET_EXTRAPOLATION = 1 };
/* Solid wall treatment (SolidWall, lbm3d.h:81). */
enum { ORR_SOLID_HALFWAY = 0, ORR_SOLID_INTERPOLATED = 1 };
/* Population storage on the device.  All forms collide in binary32 except
 * F64, which computes in binary64 throughout (the FP64 device oracle).
 * F32, F16 and BF16 hold f - w. */
enum { ORR_STORAGE_F32 = 0, ORR_STORAGE_F16 = 1, ORR_STORAGE_BF16 = 2, ORR_STORAGE_F64 = 3 };

/* Wall (lbm2d.h:53-56). velocity_x is the tangential speed of a no-slip wall. */
typedef struct orr_wall {
    int32_t kind;
    int32_t pad_;
    double velocity_x;
} orr_wall;

/* Lbm3DConfig (lbm3d.h:83-103), field for field; Smagorinsky and Sponge
 * (lbm2d.h:60-63, lbm3d.h:61-66) are flattened. */
typedef struct orr_lbm3d_config {
    uint64_t nx, ny, nz;
    double tau;
    int32_t x_boundary;
    int32_t outlet;
    orr_wall y_low, y_high, z_low, z_high;
    double inlet_ux, inlet_uy, inlet_uz;
    double body_force_x, body_force_y, body_force_z;
    int32_t smagorinsky_enabled;
    int32_t solid_wall;
    double smagorinsky_constant;
    double sponge_strength;
    uint64_t sponge_inlet, sponge_outlet, sponge_sides;
} orr_lbm3d_config;

/* Lbm2DConfig (lbm2d.h:65-78). */
typedef struct orr_lbm2d_config {
    uint64_t nx, ny;
    double tau;
    int32_t x_boundary;
    int32_t outlet;
    orr_wall bottom, top;
    double inlet_ux, inlet_uy;
    double body_force_x, body_force_y;
    int32_t smagorinsky_enabled;
    int32_t pad_;
    double smagorinsky_constant;
} orr_lbm2d_config;

/* Options of the device solver that have no counterpart in Lbm3DConfig. */
typedef struct orr_solver_options {
    int32_t storage;          /* ORR_STORAGE_* */
    int32_t allow_high_mach;  /* 1: skip the lattice Mach guard (opt-in; off by default) */
    int32_t device;           /* CUDA device ordinal */
    int32_t block_x;          /* threads per block of the step kernel; 0 = tuned default */
    int32_t kernel;           /* ORR_KERNEL_*: the D3Q19 step kernel (0 = automatic: the row kernel) */
    int32_t stages;           /* pipeline stages of ORR_KERNEL_STAGED; 0 = tuned default */
    int32_t nodes_per_thread; /* STAGED: 1 or 2 nodes per thread of a span; ROWS: 1, or 2
                                 neighbouring nodes per thread (2-byte storage, periodic or
                                 free-slip sides, halfway walls, even nx, block_x <= 128 only);
                                 0 = default */
} orr_solver_options;

/* D3Q19 step kernels.  ROWS: one block per row tile, every population read
 * straight from global memory.  STAGED: a persistent kernel whose interior
 * row spans receive their 19 source segments through a shared-memory
 * pipeline of bulk asynchronous copies (rows of lattices whose nx is a
 * multiple of 16; other rows take the per-node path); it serves lattices with
 * periodic or free-slip sides and halfway walls (and refuses others).  TILED:
 * a persistent kernel fed by tensor-map tile copies, for the same lattices.
 * AUTO picks ROWS for every storage.  All give the same result bit for bit. */
enum { ORR_KERNEL_AUTO = 0, ORR_KERNEL_ROWS = 1, ORR_KERNEL_STAGED = 2, ORR_KERNEL_TILED = 3 };

typedef struct orr_lbm3d orr_lbm3d;
typedef struct orr_lbm2d orr_lbm2d;

/* ---- library ----------------------------------------------------------- */

/* Text of the last failure on the calling thread ("" if none). */
ORR_API const char* orr_last_error(void);
/* Library version string. */
ORR_API const char* orr_version(void);
/* Number of CUDA devices the library can use (0 when none). */
ORR_API orr_status orr_device_count(int32_t* count);

/* ---- D3Q19 ------------------------------------------------------------- */

/* validate() (lbm3d.h:113-114; lbm3d_common.cpp:74-161), plus the checks of
 * make_gpu_solver (lbm3d_gpu.cpp:94-127, 492-500) for the chosen storage.
 * `distance` may be NULL (a mask without distances).  Writes the reason into
 * `message` (capacity `capacity`, always NUL-terminated) and returns
 * ORR_ERR_INVALID when refused, ORR_OK otherwise.  No device is touched. */
ORR_API orr_status orr_lbm3d_validate(const orr_lbm3d_config* config, const uint8_t* solid,
                                      const double* distance, const orr_solver_options* options,
                                      char* message, size_t capacity);

/* make_gpu_solver (lbm3d.h:246-247; lbm3d_gpu.cpp:487-513): validates, counts
 * the boundary tables, checks device memory and only then allocates; the
 * state starts at uniform_inlet_state (lbm3d_common.cpp:262-270).
 * `options` may be NULL (FP32 storage, Mach guard on, device 0). */
ORR_API orr_status orr_lbm3d_create(const orr_lbm3d_config* config, const uint8_t* solid,
                                    const double* distance, const orr_solver_options* options,
                                    orr_lbm3d** out);
ORR_API void orr_lbm3d_destroy(orr_lbm3d* solver);
ORR_API const char* orr_lbm3d_last_error(const orr_lbm3d* solver);

/* The step kernel a solver runs and its launch shape (no counterpart in the
 * reference, whose GL backend has one dispatch shape): kernel ORR_KERNEL_ROWS,
 * ORR_KERNEL_STAGED or ORR_KERNEL_TILED, threads per CTA (consumer threads of
 * the persistent steps), pipeline stages and shared bytes per CTA, CTAs per
 * launch, resident CTAs per SM, registers per thread, nodes per consumer
 * thread of a staged span or tile, and the staged spans or tiles and the
 * per-node work items. */
typedef struct orr_kernel_info {
    int32_t kernel;
    uint32_t block;
    uint32_t stages;
    uint32_t grid;
    int32_t ctas_per_sm;
    int32_t registers;
    uint32_t shared_bytes;
    uint32_t nodes_per_thread;
    uint64_t staged_items;
    uint64_t direct_items;
} orr_kernel_info;
ORR_API orr_status orr_lbm3d_kernel_info(const orr_lbm3d* solver, orr_kernel_info* info);

/* Lbm3DSolver::initialize (lbm3d.h:211): equilibrium of the given fields at
 * every fluid node (solids at rest), step count reset, inlet velocity back to
 * the configuration's.  Each of rho, ux, uy, uz is an array of nx*ny*nz
 * doubles; all four NULL gives uniform_inlet_state. */
ORR_API orr_status orr_lbm3d_initialize(orr_lbm3d* solver, const double* rho, const double* ux,
                                        const double* uy, const double* uz);
/* Lbm3DSolver::step (lbm3d.h:212). */
ORR_API orr_status orr_lbm3d_step(orr_lbm3d* solver, uint64_t count);
/* Lbm3DSolver::steps (lbm3d.h:207). */
ORR_API orr_status orr_lbm3d_steps(const orr_lbm3d* solver, uint64_t* steps);
/* Lbm3DSolver::set_inlet_velocity / inlet_velocity (lbm3d.h:218-219;
 * check_inlet_velocity, lbm3d_common.cpp:163-174). */
ORR_API orr_status orr_lbm3d_set_inlet_velocity(orr_lbm3d* solver, const double velocity[3]);
ORR_API orr_status orr_lbm3d_inlet_velocity(const orr_lbm3d* solver, double velocity[3]);
/* Lbm3DSolver::force (lbm3d.h:227; lbm3d_gpu.cpp:407-436): force[0..2] and
 * moment about the lattice origin [3..5], summed in binary64 on the device. */
ORR_API orr_status orr_lbm3d_force(orr_lbm3d* solver, double force_moment[6]);
/* Lbm3DSolver::macroscopic (lbm3d.h:221; lbm3d_gpu.cpp:357-392): density and
 * velocity with the Guo half-force correction; solids report 1 and 0.  Any
 * output pointer may be NULL. */
ORR_API orr_status orr_lbm3d_macroscopic(orr_lbm3d* solver, double* rho, double* ux, double* uy,
                                         double* uz);
/* Lbm3DSolver::populations (lbm3d.h:222): 19 * cells doubles, unshifted. */
ORR_API orr_status orr_lbm3d_populations(orr_lbm3d* solver, double* f);
/* Lbm3DSolver::mass (lbm3d.h:229): sum of populations over fluid nodes,
 * accumulated in binary64 on the device. */
ORR_API orr_status orr_lbm3d_mass(orr_lbm3d* solver, double* mass);
/* Lbm3DSolver::links (lbm3d.h:231; boundary_links, lbm3d_common.cpp:176-198),
 * in the reference's scan order.  Query the count first. */
ORR_API orr_status orr_lbm3d_link_count(const orr_lbm3d* solver, uint64_t* count);
ORR_API orr_status orr_lbm3d_links(const orr_lbm3d* solver, uint32_t* cell, uint32_t* direction,
                                   double* q);
/* gpu_memory_bytes(config, links, wall_slots) (lbm3d.h:188-189) for this
 * library's layout and the chosen storage: what create() checks against the
 * free device memory.  Empty result (ORR_ERR_INVALID) when it overflows. */
ORR_API orr_status orr_lbm3d_memory_bytes(const orr_lbm3d_config* config, uint64_t links,
                                          uint64_t boundary_nodes, int32_t storage,
                                          uint64_t* bytes);
/* Host-only planning of an accepted configuration, no device involved:
 * boundary_links (lbm3d.h:124-125; lbm3d_common.cpp:176-198) with their wall
 * fractions (link_fraction, lbm3d_internal.h:132-179), and the node counts.
 * Pass NULL arrays to query the counts; then arrays of `links` entries.
 * Any count pointer may be NULL. */
ORR_API orr_status orr_lbm3d_plan(const orr_lbm3d_config* config, const uint8_t* solid,
                                  const double* distance, uint64_t* links, uint64_t* fluid,
                                  uint64_t* boundary_nodes, uint32_t* cell, uint32_t* direction,
                                  double* q);
/* Number of boundary (non-bulk fluid) nodes the step kernel handles on its
 * general path, and of fluid nodes. */
ORR_API orr_status orr_lbm3d_node_counts(const orr_lbm3d* solver, uint64_t* fluid,
                                         uint64_t* boundary);
/* The cudaStream_t the handle launches on (for event timing by the caller). */
ORR_API orr_status orr_lbm3d_stream(const orr_lbm3d* solver, void** stream);
/* Kernels launched by this handle since creation (step, force, moments, ...). */
ORR_API orr_status orr_lbm3d_launch_count(const orr_lbm3d* solver, uint64_t* launches);
/* Test hook of the staged step's bounded waits (no counterpart in the
 * reference, whose GL kernels do not wait on copies): the next staged launch's
 * CTA `cta` withholds the copies of its first span, so its consumers' wait
 * runs out (about 1.3 s), the launch ends early and the next read-back returns
 * ORR_ERR_TIMEOUT, as after a copy that never lands; the populations are then
 * invalid until orr_lbm3d_initialize, which also cancels a request no launch
 * has taken.  Refused (ORR_ERR_INVALID) unless the solver runs the staged step
 * and that CTA has a staged span. */
ORR_API orr_status orr_lbm3d_request_stall(orr_lbm3d* solver, uint32_t cta);

/* ---- D3Q19 batches ------------------------------------------------------ */

/* A batch advances several D3Q19 solvers together.  The reference has no
 * counterpart: it steps one lattice per solver (Lbm3DSolver::step,
 * lbm3d.h:213), and a drag table or sweep runs its lattices one after
 * another.  Members are ordinary solver handles created with
 * orr_lbm3d_create; they keep every read-back entry point (force,
 * macroscopic, populations, mass), while orr_lbm3d_step is refused for a
 * member.  Members share the device, the storage form and the collision
 * model (Smagorinsky on or off); their sizes, boundaries and parameters may
 * all differ.  A batch step gives every member exactly the populations its
 * own steps would give (bit for bit), whatever the schedule and the mix.
 * Not thread-safe; one batch per thread. */
typedef struct orr_batch3d orr_batch3d;

/* How a batch step runs.  kernel ORR_KERNEL_STAGED: one launch of the
 * persistent staged kernel over every member's row tiles (block 128 or 256,
 * stages 0 = tuned default); ORR_KERNEL_ROWS: one row-tile launch per member
 * (block 32..256).  Steps run as CUDA graphs.  grid and ms_per_step are
 * outputs (CTAs of the staged launch; the time per batch step a tuning trial
 * measured). */
typedef struct orr_batch_schedule {
    int32_t kernel;
    uint32_t block;
    uint32_t stages;
    uint32_t grid;
    uint32_t nodes_per_thread;   /* staged: 1 or 2 nodes per thread of a span (0 = default);
                                    rows: 2 takes two neighbouring nodes per thread on the
                                    members that allow it (as orr_solver_options), 1 elsewhere */
    uint32_t branches;           /* 0: as above; n > 0: each member runs its own single-lattice
                                    launches (staged: a grid proportional to its nodes), the
                                    members spread over n parallel graph branches */
    double ms_per_step;
} orr_batch_schedule;

ORR_API orr_status orr_batch3d_create(int32_t device, orr_batch3d** out);
/* Destroys the batch; its members become ordinary solvers again. */
ORR_API void orr_batch3d_destroy(orr_batch3d* batch);
ORR_API const char* orr_batch3d_last_error(const orr_batch3d* batch);
ORR_API orr_status orr_batch3d_add(orr_batch3d* batch, orr_lbm3d* solver);
ORR_API orr_status orr_batch3d_remove(orr_batch3d* batch, orr_lbm3d* solver);
/* Members and their total nodes. */
ORR_API orr_status orr_batch3d_size(const orr_batch3d* batch, uint32_t* members, uint64_t* cells);
ORR_API orr_status orr_batch3d_set_schedule(orr_batch3d* batch, const orr_batch_schedule* schedule);
ORR_API orr_status orr_batch3d_schedule(const orr_batch3d* batch, orr_batch_schedule* schedule);
/* `count` steps of every member (asynchronous on the batch stream). */
ORR_API orr_status orr_batch3d_step(orr_batch3d* batch, uint64_t count);
/* `count` steps of every member with the momentum-exchange force and moment
 * summed after every `sample_every` steps (even, dividing count) - the
 * reference adapter's sampling (lbm_aero_solver3d.cpp:385-441).  `sums`
 * (6 doubles per member, in the order members were added; may be NULL)
 * receives the sums over the samples, added in a fixed order. */
ORR_API orr_status orr_batch3d_step_sampled(orr_batch3d* batch, uint64_t count, uint32_t sample_every,
                                            double* sums);
/* Force and moment (about the lattice origin) of every member now, 6 doubles
 * per member, summed in a fixed order (after an even number of batch steps). */
ORR_API orr_status orr_batch3d_forces(orr_batch3d* batch, double* force_moment);
/* Autotuner: times every candidate schedule on the batch itself for
 * `graphs_per_trial` graphs of 16 steps (after one untimed graph) and keeps
 * the fastest.  The trial steps are real steps of every member.  The
 * candidates' timings go to `trials` (up to `capacity`), their number to
 * `count`. */
ORR_API orr_status orr_batch3d_tune(orr_batch3d* batch, uint32_t graphs_per_trial,
                                    orr_batch_schedule* trials, uint32_t capacity, uint32_t* count);
ORR_API orr_status orr_batch3d_synchronize(orr_batch3d* batch);
ORR_API orr_status orr_batch3d_stream(const orr_batch3d* batch, void** stream);
ORR_API orr_status orr_batch3d_launch_count(const orr_batch3d* batch, uint64_t* launches);

/* ---- D3Q19 serving ------------------------------------------------------ */

/* A server runs drag solves of any lattice size as they arrive, with
 * continuous batching on one device: each round advances every admitted
 * lattice by `chunk_steps` steps in one batch (orr_batch3d_*), admits queued
 * requests in arrival order while a slot is free and the admitted lattices'
 * device memory (orr_lbm3d_memory_bytes) stays within `memory_budget` - the
 * planning, allocation and upload of new solves overlap the running chunk -
 * and retires the solves that are done.  A solve samples its force every
 * `sample_every` steps (the reference adapter's sampling,
 * lbm_aero_solver3d.cpp:385-441) and is done when the mean Cd of its last
 * window of `window` steps differs from the previous window's by less than
 * `tolerance` (converged), at `max_steps` (capped), or when the force stops
 * being finite (failed).  A solve's result is the same alone and in any mix.
 * The reference has no counterpart: atmo::sample_cd_table
 * (src/atmo/cd_sampling.cpp:98-120) runs its solves one after another.
 * Entry points are thread-safe; results are kept until the server is
 * destroyed. */
typedef struct orr_server orr_server;

typedef struct orr_serve_options {
    int32_t storage;          /* ORR_STORAGE_* of every solve */
    int32_t device;
    uint64_t memory_budget;   /* bytes of device memory the admitted lattices may hold */
    uint32_t max_active;      /* lattices on the device at once */
    uint32_t chunk_steps;     /* steps per round (a multiple of sample_every) */
    uint32_t sample_every;    /* force sampling interval, even */
    int32_t kernel;           /* batch schedule: ORR_KERNEL_AUTO (the row kernel, each lattice on its
                                 own graph branch, up to 64), ORR_KERNEL_ROWS or ORR_KERNEL_STAGED */
    uint32_t block;           /* 0: the schedule's default */
    uint32_t stages;          /* 0: tuned default */
    uint32_t branches;        /* as orr_batch_schedule::branches: 0 one launch (staged) or one stream
                                 (rows) for all lattices; n > 0 each lattice its own launches, the
                                 lattices spread over n parallel graph branches */
} orr_serve_options;

typedef struct orr_solve_request {
    const orr_lbm3d_config* config;   /* inflow / outflow x with a non-zero inlet speed */
    const uint8_t* solid;             /* nx*ny*nz flags, copied */
    const double* distance;           /* signed distances or NULL, copied */
    const double* rho;                /* initial fields (all four or none), copied */
    const double* ux;
    const double* uy;
    const double* uz;
    int32_t allow_high_mach;
    uint32_t sample_every;            /* 0 or the server's */
    uint32_t window;                  /* steps per window, a multiple of chunk_steps */
    uint32_t mode;                    /* ORR_RUN_UNTIL_SETTLED or ORR_RUN_FIXED_STEPS */
    double tolerance;                 /* on |delta Cd| between consecutive window means (until settled) */
    uint64_t max_steps;               /* step cap (0: none); the run's length when fixed */
    double reference_area;            /* Cd = Fx / (1/2 rho U^2 A) */
    double reference_length;          /* Cm = Mz / (1/2 rho U^2 A L) */
    double moment_centre[3];
    /* Gradual start (LbmAeroSolver3D::step, src/aero/lbm3d/lbm_aero_solver3d.cpp:
     * 398-412): when positive the solve starts at rest (rho 1, u 0, initial
     * fields not allowed) and its inlet velocity is the configured one times
     * (1 - cos(pi s / ramp_steps)) / 2 while s < ramp_steps, where s is the
     * first step of each sampling interval (held over the interval), and the
     * configured one after.  0: no ramp. */
    double ramp_steps;
    /* Steady test of the settle rule (until settled only): when positive, a
     * window settles only if, besides |delta Cd| < tolerance, the ranges
     * (max - min) of the x, y and z force samples over the window are each
     * within steady_range times |mean x force| - the reference adapter's
     * steady criterion (forces_settled_3d, src/aero/lbm3d/
     * lbm_aero_solver3d.cpp:61-80, kSteadyResidual = 1e-3 at :25), so that
     * an oscillating wake is not taken as settled when two window means
     * happen to agree.  The ranges are of the lattice-axis components, the
     * wind axes for an inlet along x.  0: off. */
    double steady_range;
} orr_solve_request;

/* Run modes of a served solve.  Until settled: windows of `window` steps
 * until |delta Cd| < tolerance or max_steps.  Fixed steps: exactly max_steps
 * steps (max_steps and max_steps - window multiples of chunk_steps), the
 * result the means over the last `window` steps, as the reference adapter's
 * moving average over a run of fixed duration (lbm_aero_solver3d.cpp:464-481);
 * the tolerance is not used. */
enum {
    ORR_RUN_UNTIL_SETTLED = 0,
    ORR_RUN_FIXED_STEPS = 1
};

enum {
    ORR_SOLVE_QUEUED = 0,
    ORR_SOLVE_RUNNING = 1,
    ORR_SOLVE_CONVERGED = 2,
    ORR_SOLVE_CAPPED = 3,
    ORR_SOLVE_FAILED = 4,
    ORR_SOLVE_COMPLETED = 5           /* a fixed-steps solve ran its steps */
};

typedef struct orr_solve_result {
    int32_t state;                    /* ORR_SOLVE_* */
    int32_t reserved;
    uint64_t steps;
    double cd, cl, cm;                /* means of the last window (lift along +y, moment about z) */
    double delta_cd;                  /* |Cd difference| of the last two windows */
    double force[3], moment[3];       /* window means, moment about the lattice origin */
    double arrival_s, admitted_s, finished_s; /* seconds since the server started */
    uint64_t device_bytes;
    char message[160];
} orr_solve_result;

typedef struct orr_serve_statistics {
    uint64_t submitted, completed, failed, queued, active;
    double latency_p50_s, latency_p99_s, latency_mean_s; /* arrival to result, completed solves */
    double solves_per_second;         /* completed / (last finish - first arrival) */
    double lattice_updates;           /* sum over rounds of active nodes x steps */
    double busy_seconds;              /* time with lattices on the device */
    uint64_t peak_device_bytes;
    double mean_active;               /* lattices per round */
    uint64_t chunks;
    int32_t worker_failed;
    char message[160];
} orr_serve_statistics;

ORR_API orr_status orr_serve_create(const orr_serve_options* options, orr_server** out);
/* Stops the worker (solves still queued or running are abandoned). */
ORR_API void orr_serve_destroy(orr_server* server);
ORR_API const char* orr_serve_last_error(const orr_server* server);
ORR_API orr_status orr_serve_submit(orr_server* server, const orr_solve_request* request, uint64_t* id);
ORR_API orr_status orr_serve_poll(orr_server* server, uint64_t id, orr_solve_result* result);
/* Blocks until the solve is done or the timeout passes (ORR_ERR_TIMEOUT). */
ORR_API orr_status orr_serve_wait(orr_server* server, uint64_t id, double timeout_s, orr_solve_result* result);
/* Blocks until every submitted solve is done or the timeout passes. */
ORR_API orr_status orr_serve_drain(orr_server* server, double timeout_s);
ORR_API orr_status orr_serve_stats(orr_server* server, orr_serve_statistics* stats);

/* Inputs of orr_lbm3d_force_static: device pointers the caller owns. */
typedef struct orr_force_links {
    uint64_t nx, ny, nz;        /* lattice dimensions */
    int32_t storage;            /* ORR_STORAGE_* of `populations` */
    int32_t device;             /* CUDA device the pointers belong to */
    const void* populations;    /* 19 * nx*ny*nz values, layout of orr_lbm3d_populations,
                                   stored as the storage form holds them (f - w for the
                                   binary32, binary16 and bfloat16 forms, f for binary64) */
    const uint32_t* link_cell;  /* per link: node index x + nx (y + ny z) */
    const uint32_t* link_dir;   /* per link: direction j (its source x - c_j is solid) */
    const double* link_q;       /* per link: wall fraction q */
    uint64_t links;             /* number of links, at most ORR_FORCE_STATIC_MAX_LINKS */
    void* stream;               /* cudaStream_t to run on; NULL is the legacy default stream */
} orr_force_links;

#define ORR_FORCE_STATIC_MAX_LINKS 8388608u

/* No counterpart in the reference: an allocation-free twin of
 * orr_lbm3d_force for callers that may not allocate device memory (a host
 * application whose device memory belongs to another allocator or pool, a
 * real-time loop that must not call into the allocator, a process that has
 * reserved all device memory up front).  It computes the same momentum-
 * exchange force and moment over links the caller already holds on the
 * device, using as scratch a fixed 192 KiB array compiled into the library
 * (held by every GPU that loads the library until exit), so it calls no
 * cudaMalloc or cudaFree.  More than ORR_FORCE_STATIC_MAX_LINKS links are
 * refused with ORR_ERR_INVALID, and so is a call whose tables hold a link
 * outside the lattice (a cell beyond nx*ny*nz, a direction outside 1..18 or
 * an interpolation source beyond the lattice: the caller owns the tables,
 * and such links are skipped on the device, never read through).  The
 * first call on a device looks up the
 * array's device address (make it before any stream capture).  All calls
 * share the array: calls whose work overlaps on the GPU race and must be
 * serialised by the caller.  Blocks until the result is in force_moment. */
ORR_API orr_status orr_lbm3d_force_static(const orr_force_links* args, double force_moment[6]);

/* ---- The reference's compute-backend kernels --------------------------- */

/* The three D3Q19 kernels the reference's GPU driver, GpuLbm3D, dispatches
 * through its IComputeBackend (lbm_d3q19_step, lbm_d3q19_moments,
 * lbm_d3q19_force: src/aero/lbm3d/lbm3d_gpu.cpp:37-44, 158-189, 333-436,
 * IComputeBackend::dispatch of compute_backend.h:94-129), run on device
 * buffers in that driver's layout: binary32 populations shifted by their
 * weights (19 * nx*ny*nz, the layout of ORR_STORAGE_F32), node codes (uint32:
 * 0 solid, 1 bulk, 2 boundary, 3 + wall slot), 19 binary32 wall fractions per
 * slot, the convective-outlet history (5 * ny*nz), the moments (rho - 1, ux,
 * uy, uz planes) and the links (cell, direction pairs).  A CUDA
 * IComputeBackend (orrery_b200/adapter/compute_backend_cuda.cpp) maps the
 * driver's dispatches onto these calls.  Population buffers need
 * orr_gl3d_buffer_slack() bytes of addressable slack before and after them
 * (the step reads past the lattice at its edges and never uses those values).
 * Calls are ordered on `stream` (a cudaStream_t; NULL is the legacy stream). */
typedef struct orr_gl3d_params {   /* the driver's uniforms (lbm3d_gpu.cpp:158-189) */
    uint32_t nx, ny, nz;           /* u_nx, u_ny, u_nz */
    uint32_t x_mode;               /* u_x_mode: 1 inflow / outflow, 0 periodic */
    uint32_t wall_kind[4];         /* u_{y_low,y_high,z_low,z_high}_kind: 0 periodic, 1 slip, 2 no-slip */
    float wall_ux[4];              /* u_{y_low,y_high,z_low,z_high}_ux */
    float inlet[3];                /* u_inlet_ux, u_inlet_uy, u_inlet_uz */
    float tau;                     /* u_tau */
    float smagorinsky_c2;          /* u_smagorinsky_c2: the closure is on when positive */
    float force[3];                /* u_force_x, u_force_y, u_force_z */
    uint32_t outlet_mode;          /* u_outlet_mode: 1 extrapolation, 0 convective */
    float outlet_speed;            /* u_outlet_speed */
    float sponge_strength;         /* u_sponge_strength */
    uint32_t sponge_inlet, sponge_outlet, sponge_sides; /* u_sponge_* */
    uint32_t link_count;           /* u_link_count */
} orr_gl3d_params;

typedef struct orr_gl3d orr_gl3d;  /* the tables derived from one node-code buffer */

/* Bytes of slack a population buffer needs before and after it. */
ORR_API uint64_t orr_gl3d_buffer_slack(void);
/* Tables for the lattice of `params` whose node codes are `class_codes` (host,
 * nx*ny*nz values): this library's node classes, bounce-back masks and wall
 * slots, on `device`.  The lattice is validated as the driver's make_gpu_solver
 * validates it. */
ORR_API orr_status orr_gl3d_create(const orr_gl3d_params* params, const uint32_t* class_codes, int32_t device,
                                   orr_gl3d** out);
ORR_API void orr_gl3d_destroy(orr_gl3d* tables);
ORR_API const char* orr_gl3d_last_error(const orr_gl3d* tables);
/* lbm_d3q19_step: binding 0 (src) -> binding 2 (dst), binding 6 (outlet
 * history, updated), binding 7 (wall fractions; may be NULL without slots). */
ORR_API orr_status orr_gl3d_step(orr_gl3d* tables, const orr_gl3d_params* params, const float* src, float* dst,
                                 float* outlet, const float* wall, void* stream);
/* lbm_d3q19_moments: binding 0 (src) -> binding 3 (moments). */
ORR_API orr_status orr_gl3d_moments(orr_gl3d* tables, const orr_gl3d_params* params, const float* src,
                                    float* moments, void* stream);
/* lbm_d3q19_force: binding 0 (src), 4 (links), 7 (wall) -> binding 5 (per link
 * the shifted sum f*_o + f_j; a link outside the lattice gives 0). */
ORR_API orr_status orr_gl3d_link_force(orr_gl3d* tables, const orr_gl3d_params* params, const float* src,
                                       const uint32_t* links, float* link_force, const float* wall, void* stream);

/* The D2Q9 twins: the three kernels the reference's GpuLbm2D dispatches
 * (lbm_d2q9_step, lbm_d2q9_moments, lbm_d2q9_force: src/aero/lbm/
 * lbm2d_gpu.cpp:36-44, 104-124, 220-300), on buffers in that driver's
 * layout: binary32 populations shifted by their weights (9 * nx*ny), solid
 * flags (uint32: 1 solid, 0 fluid), the moments (rho - 1, ux, uy planes), the
 * convective-outlet history (3 * ny: directions 3, 6, 7, slot * ny + y) and
 * the links (cell, direction pairs).  No slack is needed around the
 * population buffers. */
typedef struct orr_gl2d_params {   /* the driver's uniforms (lbm2d_gpu.cpp:104-124) */
    uint32_t nx, ny;               /* u_nx, u_ny */
    uint32_t x_mode;               /* u_x_mode: 1 inflow / outflow, 0 periodic */
    uint32_t bottom_kind, top_kind; /* u_bottom_kind, u_top_kind: 0 periodic, 1 slip, 2 no-slip */
    float bottom_ux, top_ux;       /* u_bottom_ux, u_top_ux */
    float inlet[2];                /* u_inlet_ux, u_inlet_uy */
    float tau;                     /* u_tau */
    float smagorinsky_c2;          /* u_smagorinsky_c2: the closure is on when positive */
    float force[2];                /* u_force_x, u_force_y */
    uint32_t outlet_mode;          /* u_outlet_mode: 1 extrapolation, 0 convective */
    float outlet_speed;            /* u_outlet_speed */
    uint32_t link_count;           /* u_link_count */
} orr_gl2d_params;

typedef struct orr_gl2d orr_gl2d;  /* the tables derived from one solid-flag buffer */

/* Tables for the lattice of `params` whose solid flags are `solid_flags`
 * (host, nx*ny values): this library's node classes and bounce-back masks,
 * on `device`.  The lattice is validated as the 2D make_gpu_solver
 * validates it. */
ORR_API orr_status orr_gl2d_create(const orr_gl2d_params* params, const uint32_t* solid_flags, int32_t device,
                                   orr_gl2d** out);
ORR_API void orr_gl2d_destroy(orr_gl2d* tables);
ORR_API const char* orr_gl2d_last_error(const orr_gl2d* tables);
/* lbm_d2q9_step: binding 0 (src) -> binding 2 (dst), binding 6 (outlet
 * history, updated). */
ORR_API orr_status orr_gl2d_step(orr_gl2d* tables, const orr_gl2d_params* params, const float* src, float* dst,
                                 float* outlet, void* stream);
/* lbm_d2q9_moments: binding 0 (src) -> binding 3 (moments). */
ORR_API orr_status orr_gl2d_moments(orr_gl2d* tables, const orr_gl2d_params* params, const float* src,
                                    float* moments, void* stream);
/* lbm_d2q9_force: binding 0 (src), 4 (links) -> binding 5 (per link the two
 * components of 2 c_o fs_o, fs_o the shifted population leaving towards the
 * wall; a link outside the lattice gives 0).  `tables` may be NULL (the
 * kernel needs the lattice size only; it then runs on the current device). */
ORR_API orr_status orr_gl2d_link_force(orr_gl2d* tables, const orr_gl2d_params* params, const float* src,
                                       const uint32_t* links, float* link_force, void* stream);

/* ---- D2Q9 -------------------------------------------------------------- */

/* validate (lbm2d.h:85-86; lbm2d_common.cpp:31-77) plus the binary32 checks
 * of the 2D make_gpu_solver (lbm2d.h:205-212). */
ORR_API orr_status orr_lbm2d_validate(const orr_lbm2d_config* config, const uint8_t* solid,
                                      const orr_solver_options* options, char* message,
                                      size_t capacity);
/* make_gpu_solver (lbm2d.h:211-212). */
ORR_API orr_status orr_lbm2d_create(const orr_lbm2d_config* config, const uint8_t* solid,
                                    const orr_solver_options* options, orr_lbm2d** out);
ORR_API void orr_lbm2d_destroy(orr_lbm2d* solver);
ORR_API const char* orr_lbm2d_last_error(const orr_lbm2d* solver);
/* Lbm2DSolver::initialize (lbm2d.h:187); rho, ux, uy arrays of nx*ny doubles
 * or all NULL for uniform_inlet_state. */
ORR_API orr_status orr_lbm2d_initialize(orr_lbm2d* solver, const double* rho, const double* ux,
                                        const double* uy);
ORR_API orr_status orr_lbm2d_step(orr_lbm2d* solver, uint64_t count);
ORR_API orr_status orr_lbm2d_steps(const orr_lbm2d* solver, uint64_t* steps);
/* Lbm2DSolver::force (lbm2d.h:196): x, y and the z moment about the origin. */
ORR_API orr_status orr_lbm2d_force(orr_lbm2d* solver, double force_moment[3]);
ORR_API orr_status orr_lbm2d_macroscopic(orr_lbm2d* solver, double* rho, double* ux, double* uy);
ORR_API orr_status orr_lbm2d_populations(orr_lbm2d* solver, double* f);
ORR_API orr_status orr_lbm2d_mass(orr_lbm2d* solver, double* mass);
ORR_API orr_status orr_lbm2d_link_count(const orr_lbm2d* solver, uint64_t* count);
ORR_API orr_status orr_lbm2d_links(const orr_lbm2d* solver, uint32_t* cell, uint32_t* direction);
ORR_API orr_status orr_lbm2d_stream(const orr_lbm2d* solver, void** stream);
ORR_API orr_status orr_lbm2d_launch_count(const orr_lbm2d* solver, uint64_t* launches);

/* ---- mesh voxelization (solid masks and wall distances) ------------------
 *
 * The adapter builds every lattice's solid mask and wall distances from the
 * body's triangle mesh (lbm_aero_solver3d.cpp:249-258) with geom::voxelize and
 * geom::signed_distance_band (src/geom/include/orrery/geom/voxel_grid.h:35-69).
 * These entry points compute the same arrays on the device; inputs and
 * outputs are host arrays.  Cell (i, j, k) has its centre at
 * origin + spacing (i + 1/2, j + 1/2, k + 1/2) and index i + nx (j + ny k). */
typedef struct orr_grid_spec {     /* geom::GridSpec (voxel_grid.h:14-27) */
    double origin[3];
    double spacing;
    uint64_t nx, ny, nz;
} orr_grid_spec;

typedef struct orr_mesh {           /* geom::TriangleMesh (triangle_mesh.h:15-19) */
    const double* vertices;         /* 3 per vertex */
    uint64_t vertex_count;
    const uint32_t* triangles;      /* 3 corner indices per triangle, counter-clockwise seen from outside */
    uint64_t triangle_count;
} orr_mesh;

/* geom::grid_around (voxel_grid.h:31-33): the grid covering the box with
 * `padding` extra cells on every side, centred on it. */
ORR_API orr_status orr_grid_around(const double box_min[3], const double box_max[3], double spacing,
                                   uint64_t padding, orr_grid_spec* out);
/* geom::voxelize (voxel_grid.h:47-52): solid[c] = winding number at the cell
 * centre >= threshold (0.5 in the reference); `winding` (nx*ny*nz doubles) may
 * be NULL.  Refusals carry the reference's texts.  *device_ms (may be NULL)
 * receives the kernel time. */
ORR_API orr_status orr_voxelize(const orr_mesh* mesh, const orr_grid_spec* spec, double threshold,
                                int32_t device, uint8_t* solid, double* winding, double* device_ms);
/* geom::signed_distance_band (voxel_grid.h:54-69) for the solid flags of
 * orr_voxelize: distance to the closest triangle within band_cells * spacing
 * (negative in solid cells, +-band outside the band), in_band flags, and the
 * band width in *band (may be NULL). */
ORR_API orr_status orr_signed_distance_band(const orr_mesh* mesh, const orr_grid_spec* spec,
                                            const uint8_t* solid, uint64_t solid_count, double band_cells,
                                            int32_t device, double* distance, uint8_t* in_band, double* band,
                                            double* device_ms);

#ifdef __cplusplus
}
#endif

#endif /* ORRERY_LBM_H */
