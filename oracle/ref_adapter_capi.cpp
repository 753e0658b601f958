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
        orrery::aero::FlowConditions conditions;
        conditions.speed = p[2];
        conditions.density = p[3];
        conditions.viscosity = p[4];
        conditions.angle_of_attack = p[5];
        conditions.sideslip = p[6];
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
