// The reference's own 3D adapter, LbmAeroSolver3D (src/aero/lbm3d/
// lbm_aero_solver3d.cpp), compiled unmodified from the reference sources in
// place by oracle/Makefile into oracle/_ref/libref_adapter.so, with its GPU
// branch on the CUDA solver: the adapter calls make_gpu_solver when
// LbmSolver3DOptions::backend is set (lbm_aero_solver3d.cpp:312), and the
// definition below returns the CUDA solver of orrery_b200/adapter/lbm3d_cuda.cpp
// (a null compute backend only selects that branch).  Without a backend the
// adapter runs the reference's CPU solver.
//
// TEST INFRASTRUCTURE ONLY: the end-to-end check of the solver seam (the
// reference's "3D IAeroSolver adapter runs on the GPU backend" test with the
// CUDA solver in place of the GL one).  The product never links or loads it.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <numbers>
#include <string>
#include <vector>

#include "lbm3d_cuda.h"
#include "orrery/aero/compute/null_compute_backend.h"
#include "orrery/aero/lbm3d/lbm_aero_solver3d.h"
#include "orrery/atmo/aero_table.h"

namespace orrery::aero::lbm {

namespace {
std::int32_t g_storage = ORR_STORAGE_F32;
}

core::Result<std::unique_ptr<Lbm3DSolver>, std::string> make_gpu_solver(compute::IComputeBackend& /*backend*/,
                                                                         const Lbm3DConfig& config,
                                                                         SolidMask3D mask) {
    return make_cuda_solver(config, std::move(mask), g_storage, 0);
}

} // namespace orrery::aero::lbm

namespace {

// Wall pressure coefficients and the velocity field (3 per node, m/s) of the
// last solve, for ref_adapter_fields.
std::vector<double> g_cp;
std::vector<double> g_velocity;

void copy_message(const std::string& text, char* message, size_t capacity) {
    if (message == nullptr || capacity == 0) {
        return;
    }
    const size_t n = text.size() < capacity - 1 ? text.size() : capacity - 1;
    std::memcpy(message, text.data(), n);
    message[n] = '\0';
}

orrery::aero::AeroGeometry geometry_of(const double* vertices, uint64_t nv, const uint32_t* triangles, uint64_t nt,
                                       const double* p) {
    orrery::aero::AeroGeometry geometry;
    geometry.mesh.vertices.resize(nv);
    for (uint64_t i = 0; i < nv; ++i) {
        geometry.mesh.vertices[i] = {vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]};
    }
    geometry.mesh.triangles.resize(nt);
    for (uint64_t t = 0; t < nt; ++t) {
        geometry.mesh.triangles[t] = {triangles[3 * t], triangles[3 * t + 1], triangles[3 * t + 2]};
    }
    geometry.reference.length = p[0];
    geometry.reference.area = p[1];
    return geometry;
}

orrery::aero::FlowConditions conditions_of(const double* p) {
    orrery::aero::FlowConditions conditions;
    conditions.speed = p[2];
    conditions.density = p[3];
    conditions.viscosity = p[4];
    conditions.angle_of_attack = p[5];
    conditions.sideslip = p[6];
    return conditions;
}

orrery::aero::lbm::LbmSolver3DOptions options_of(const double* p) {
    namespace lbm = orrery::aero::lbm;
    lbm::LbmSolver3DOptions options;
    options.resolution = lbm::LatticeResolution{p[7], p[8]};
    options.upstream = p[9];
    options.downstream = p[10];
    options.width = p[11];
    options.duration = p[12];
    options.average_window = p[13];
    options.steps_per_call = static_cast<std::size_t>(p[14]);
    options.wall = p[15] != 0.0 ? lbm::SolidWall::interpolated : lbm::SolidWall::halfway;
    options.sponge_strength = p[16];
    options.start_ramp = p[17];
    options.les = p[18] == 1.0 ? lbm::LesMode::on : (p[18] == 2.0 ? lbm::LesMode::off : lbm::LesMode::automatic);
    options.sample_every = static_cast<std::size_t>(p[19]);
    return options;
}

// The free stream of a drag-table point: the template with its speed set to
// Mach times the speed of sound (sample_point, src/atmo/cd_sampling.cpp:63-64).
orrery::aero::FlowConditions table_flow(const double* p, double temperature, double mach) {
    orrery::aero::FlowConditions flow = conditions_of(p);
    flow.temperature = temperature;
    flow.speed = mach * flow.speed_of_sound();
    return flow;
}

} // namespace

extern "C" {

// One adapter solve, stepped until LbmAeroSolver3D::step() reports it done.
// p: reference length, reference area, speed, density, viscosity, angle of
// attack, sideslip, cells per length, lattice velocity, upstream, downstream,
// width, duration, average window, steps per call, wall (0 halfway, 1
// interpolated), sponge strength, start ramp, LES (0 automatic, 1 on, 2 off),
// sample_every.  backend: 0 the reference CPU solver, 1 the CUDA solver with
// `storage`.  out: cd, cl, cy, cm, force x y z, moment x y z, iterations,
// converged, seconds, nx, ny, nz, lattice steps.  0 on success; -1 with the
// exception's text.  The wall pressure coefficients and the velocity field
// (update_result, lbm_aero_solver3d.cpp:489-550) are kept for
// ref_adapter_fields.
int ref_adapter_run(const double* vertices, uint64_t nv, const uint32_t* triangles, uint64_t nt, const double* p,
                    int backend, int storage, double* out, char* message, size_t capacity) {
    namespace lbm = orrery::aero::lbm;
    try {
        const orrery::aero::AeroGeometry geometry = geometry_of(vertices, nv, triangles, nt, p);
        const orrery::aero::FlowConditions conditions = conditions_of(p);
        lbm::LbmSolver3DOptions options = options_of(p);
        orrery::aero::compute::NullComputeBackend null_backend;
        if (backend == 1) {
            lbm::g_storage = storage;
            options.backend = &null_backend;
        }
        const auto t0 = std::chrono::steady_clock::now();
        lbm::LbmAeroSolver3D solver(options);
        solver.setup(geometry, conditions);
        while (!solver.step()) {
        }
        const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        const orrery::aero::AeroResult& r = solver.result();
        g_cp = r.surface.cp;
        g_velocity.clear();
        if (r.velocity) {
            g_velocity.reserve(3 * r.velocity->values.size());
            for (const auto& v : r.velocity->values) {
                g_velocity.insert(g_velocity.end(), {v.x, v.y, v.z});
            }
        }
        const double v[] = {r.cd,
                            r.cl,
                            r.cy,
                            r.cm,
                            r.force.x,
                            r.force.y,
                            r.force.z,
                            r.moment.x,
                            r.moment.y,
                            r.moment.z,
                            static_cast<double>(r.iterations),
                            r.converged ? 1.0 : 0.0,
                            seconds,
                            static_cast<double>(solver.lattice()->config().nx),
                            static_cast<double>(solver.lattice()->config().ny),
                            static_cast<double>(solver.lattice()->config().nz),
                            static_cast<double>(solver.total_steps())};
        std::memcpy(out, v, sizeof v);
        return 0;
    } catch (const std::exception& e) {
        copy_message(e.what(), message, capacity);
        return -1;
    }
}

// The reference's drag-table client, atmo::sample_cd_table
// (src/atmo/cd_sampling.cpp:98-120), with the lattice Boltzmann solver forced
// (CdSamplingRequest::solver_override) and a factory that returns the
// reference's LbmAeroSolver3D on the CUDA solver (`storage`): one solve per
// Mach number, one after another.  p: the ref_adapter_run parameter block
// (its speed is unused: each point sets Mach times the speed of sound of
// `temperature`).  out, 8 per point: Mach, Cd, IAeroSolver::step calls,
// converged, within the solver's envelope, seconds of the point, the table's
// Cd at that Mach, seconds of the whole table.  0 on success; -1 with the error's text.
int ref_cd_table(const double* vertices, uint64_t nv, const uint32_t* triangles, uint64_t nt, const double* p,
                 double temperature, const double* mach, uint64_t n, uint64_t max_steps, int storage, double* out,
                 char* message, size_t capacity) {
    namespace lbm = orrery::aero::lbm;
    namespace atmo = orrery::atmo;
    try {
        atmo::CdSamplingRequest request;
        request.geometry = geometry_of(vertices, nv, triangles, nt, p);
        request.mach_numbers.assign(mach, mach + n);
        request.freestream = conditions_of(p);
        request.freestream.temperature = temperature;
        request.solver_override = orrery::aero::SolverKind::lattice_boltzmann;
        request.max_steps = max_steps;
        orrery::aero::compute::NullComputeBackend null_backend;
        lbm::g_storage = storage;
        lbm::LbmSolver3DOptions options = options_of(p);
        options.backend = &null_backend;
        // Start time of each point: the factory is called once per point.
        std::vector<std::chrono::steady_clock::time_point> starts;
        const atmo::AeroSolverFactory factory =
            [&](orrery::aero::SolverKind kind) -> std::unique_ptr<orrery::aero::IAeroSolver> {
            starts.push_back(std::chrono::steady_clock::now());
            if (kind != orrery::aero::SolverKind::lattice_boltzmann) {
                return nullptr;
            }
            return std::make_unique<lbm::LbmAeroSolver3D>(options);
        };
        const auto t0 = std::chrono::steady_clock::now();
        auto sampled = atmo::sample_cd_table(request, factory);
        const auto t1 = std::chrono::steady_clock::now();
        const double total = std::chrono::duration<double>(t1 - t0).count();
        starts.push_back(t1);
        if (!sampled) {
            copy_message(sampled.error().message, message, capacity);
            return -1;
        }
        const atmo::CdSamplingResult& r = sampled.value();
        for (uint64_t k = 0; k < n; ++k) {
            const atmo::CdSamplingPoint& pt = r.points[k];
            double* o = out + 8 * k;
            o[0] = pt.mach;
            o[1] = pt.cd;
            o[2] = static_cast<double>(pt.steps);
            o[3] = pt.converged ? 1.0 : 0.0;
            o[4] = pt.within_envelope ? 1.0 : 0.0;
            o[5] = k + 1 < starts.size() ? std::chrono::duration<double>(starts[k + 1] - starts[k]).count() : 0.0;
            o[6] = r.table.cd(pt.mach);
            o[7] = total;
        }
        return 0;
    } catch (const std::exception& e) {
        copy_message(e.what(), message, capacity);
        return -1;
    }
}

// The lattice problem LbmAeroSolver3D::setup builds for the Mach `mach` point
// of such a table (the same free stream as ref_cd_table, the CUDA solver
// behind it), for a served run of the same solve: the configuration, and
// when `solid` is not null the solid flags and (`distance` not null, the
// interpolated wall) the wall distances.  meta (12): nx, ny, nz, lattice
// steps of the run (total_steps), samples in the averaging window
// (lbm_aero_solver3d.cpp:333-341), lattice steps of the gradual start, dx (m),
// the reference area and length in lattice units, the lattice velocity,
// sample_every, whether the mask has distances.  0 on success; -1 with the
// error's text.
int ref_cd_point_problem(const double* vertices, uint64_t nv, const uint32_t* triangles, uint64_t nt,
                         const double* p, double temperature, double mach, orr_lbm3d_config* config,
                         uint8_t* solid, double* distance, double* meta, char* message, size_t capacity) {
    namespace lbm = orrery::aero::lbm;
    try {
        const orrery::aero::AeroGeometry geometry = geometry_of(vertices, nv, triangles, nt, p);
        const orrery::aero::FlowConditions flow = table_flow(p, temperature, mach);
        orrery::aero::compute::NullComputeBackend null_backend;
        lbm::g_storage = ORR_STORAGE_F32;
        lbm::LbmSolver3DOptions options = options_of(p);
        options.backend = &null_backend;
        lbm::LbmAeroSolver3D solver(options);
        solver.setup(geometry, flow);
        const lbm::Lbm3DSolver& lattice = *solver.lattice();
        const lbm::SolidMask3D& mask = lattice.mask();
        const lbm::LatticeUnits& units = *solver.units();
        *config = lbm::c_config(lattice.config());
        if (solid != nullptr) {
            std::memcpy(solid, mask.solid.data(), mask.solid.size());
        }
        if (distance != nullptr && !mask.distance.empty()) {
            std::memcpy(distance, mask.distance.data(), mask.distance.size() * sizeof(double));
        }
        // Run lengths of LbmAeroSolver3D::setup (lbm_aero_solver3d.cpp:264-271,
        // 319, 340-341): steps per convective time = cells per length / lattice
        // velocity.
        const double steps_per_time = units.cells_per_length() / units.lattice_velocity();
        const double window_real =
            options.average_window * steps_per_time / static_cast<double>(options.sample_every);
        const double dx = units.dx();
        const double m[] = {static_cast<double>(mask.nx),
                            static_cast<double>(mask.ny),
                            static_cast<double>(mask.nz),
                            static_cast<double>(solver.total_steps()),
                            std::max(1.0, std::floor(window_real)),
                            options.start_ramp * steps_per_time,
                            dx,
                            geometry.reference.area / (dx * dx),
                            geometry.reference.length / dx,
                            units.lattice_velocity(),
                            static_cast<double>(options.sample_every),
                            mask.distance.empty() ? 0.0 : 1.0};
        std::memcpy(meta, m, sizeof m);
        return 0;
    } catch (const std::exception& e) {
        copy_message(e.what(), message, capacity);
        return -1;
    }
}

// The reference's AeroCoefficientTable (src/atmo/aero_table.cpp:47-83):
// create() from n samples (Mach, Cd) with `area`, then lookup() at m query
// Mach numbers (Cd and whether it was clamped).  0 on success; -1 with the
// refusal's text.
int ref_cd_table_lookup(const double* mach, const double* cd, uint64_t n, double area, const double* query,
                        uint64_t m, double* out_cd, uint8_t* clamped, char* message, size_t capacity) {
    namespace atmo = orrery::atmo;
    std::vector<atmo::CdSample> samples;
    for (uint64_t k = 0; k < n; ++k) {
        samples.push_back(atmo::CdSample{mach[k], cd[k]});
    }
    auto table = atmo::AeroCoefficientTable::create(std::move(samples), orrery::core::si::Area(area));
    if (!table) {
        copy_message(table.error().message, message, capacity);
        return -1;
    }
    for (uint64_t k = 0; k < m; ++k) {
        const atmo::CdLookup r = table.value().lookup(query[k]);
        out_cd[k] = r.cd;
        clamped[k] = r.clamped ? 1 : 0;
    }
    return 0;
}

// Sizes (cp values, velocity doubles) of the last solve's fields, and a copy
// of them when the pointers are not null.
void ref_adapter_fields(uint64_t* cp_count, uint64_t* velocity_count, double* cp, double* velocity) {
    *cp_count = g_cp.size();
    *velocity_count = g_velocity.size();
    if (cp != nullptr) {
        std::memcpy(cp, g_cp.data(), g_cp.size() * sizeof(double));
    }
    if (velocity != nullptr) {
        std::memcpy(velocity, g_velocity.data(), g_velocity.size() * sizeof(double));
    }
}

} // extern "C"
